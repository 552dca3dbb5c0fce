// io.cu -- results out of the device state, and restart.
//
//  - mgm_write_solution: Solution.csv as mg_NS_solver.c:83-88 writes it
//    ("%lf, " x, y, z, u, v, w and a pressure, one node per line, level 0 in
//    the order the set-up left the nodes).
//  - mgm_checkpoint_save / mgm_checkpoint_load: every field a time step reads
//    from the previous one (each level's p, source and residual; level 0's
//    velocities, their intermediate and old copies, dp/dn, grad p, the TIMPLE
//    pressure), in one binary file with the levels' sizes and a fingerprint of
//    their coordinates, so that a run continued from a checkpoint repeats the
//    uninterrupted run bit for bit.  The reference has no restart; its
//    operators, clouds and parameters are rebuilt by mgm_setup / set on the
//    context as usual, and a checkpoint only loads into a context whose levels
//    match.
#include "ctx.cuh"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace mgm {
namespace {

constexpr char kMagic[8] = {'M', 'G', 'M', 'C', 'K', 'P', 'T', '1'};
constexpr int kVersion = 1;

uint64_t fnv1a(const void *data, size_t bytes, uint64_t h = 1469598103934665603ULL)
{
    const unsigned char *p = (const unsigned char *)data;
    for (size_t i = 0; i < bytes; i++) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}

// the fields a step carries over: per level, then level 0's
std::vector<DBuf<double> *> level_state(Level &L) { return {&L.p, &L.src, &L.res}; }
std::vector<DBuf<double> *> field_state(mgm_ctx *c)
{
    return {&c->u,     &c->v,     &c->w,    &c->u_new, &c->v_new, &c->w_new, &c->u_old, &c->v_old,
            &c->w_old, &c->dpdn,  &c->dpdx, &c->dpdy,  &c->dpdz,  &c->p_old};
}

uint64_t geometry_hash(mgm_ctx *c, int l)
{
    Level &L = c->L[l];
    std::vector<double> a(L.n);
    uint64_t h = fnv1a(&L.n, sizeof(int));
    for (DBuf<double> *b : {&L.x, &L.y, &L.z}) {
        b->download(a.data(), L.n, c->s);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        h = fnv1a(a.data(), sizeof(double) * L.n, h);
    }
    return h;
}

struct File {
    std::FILE *f = nullptr;
    ~File()
    {
        if (f) std::fclose(f);
    }
};

void write_all(std::FILE *f, const void *p, size_t bytes, uint64_t *sum)
{
    MGM_REQUIRE(std::fwrite(p, 1, bytes, f) == bytes, "checkpoint: write failed");
    if (sum) *sum = fnv1a(p, bytes, *sum);
}

void read_all(std::FILE *f, void *p, size_t bytes, uint64_t *sum)
{
    MGM_REQUIRE(std::fread(p, 1, bytes, f) == bytes, "checkpoint: file truncated");
    if (sum) *sum = fnv1a(p, bytes, *sum);
}

void save(mgm_ctx *c, const char *path)
{
    File F;
    F.f = std::fopen(path, "wb");
    MGM_REQUIRE(F.f != nullptr, std::string("mgm_checkpoint_save: unable to open ") + path);
    int hdr[3] = {kVersion, c->dim, c->nl};
    write_all(F.f, kMagic, sizeof(kMagic), nullptr);
    write_all(F.f, hdr, sizeof(hdr), nullptr);
    for (int l = 0; l < c->nl; l++) {
        int sz[2] = {c->L[l].n, c->L[l].k};
        uint64_t h = geometry_hash(c, l);
        write_all(F.f, sz, sizeof(sz), nullptr);
        write_all(F.f, &h, sizeof(h), nullptr);
    }
    uint64_t sum = 1469598103934665603ULL;
    std::vector<double> buf;
    auto put = [&](DBuf<double> *b, int n) {
        buf.assign(n, 0.0);
        if (b->p) b->download(buf.data(), n, c->s);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        write_all(F.f, buf.data(), sizeof(double) * n, &sum);
    };
    for (int l = 0; l < c->nl; l++)
        for (DBuf<double> *b : level_state(c->L[l])) put(b, c->L[l].n);
    for (DBuf<double> *b : field_state(c)) put(b, c->L[0].n);
    write_all(F.f, &sum, sizeof(sum), nullptr);
    MGM_REQUIRE(std::fflush(F.f) == 0, "mgm_checkpoint_save: write failed");
}

void load(mgm_ctx *c, const char *path)
{
    File F;
    F.f = std::fopen(path, "rb");
    MGM_REQUIRE(F.f != nullptr, std::string("mgm_checkpoint_load: unable to open ") + path);
    char magic[8];
    int hdr[3];
    read_all(F.f, magic, sizeof(magic), nullptr);
    MGM_REQUIRE(std::memcmp(magic, kMagic, sizeof(kMagic)) == 0, "mgm_checkpoint_load: not a checkpoint file");
    read_all(F.f, hdr, sizeof(hdr), nullptr);
    MGM_REQUIRE(hdr[0] == kVersion, "mgm_checkpoint_load: unsupported checkpoint version");
    MGM_REQUIRE(hdr[1] == c->dim && hdr[2] == c->nl,
                "mgm_checkpoint_load: checkpoint does not match this context's levels");
    for (int l = 0; l < c->nl; l++) {
        int sz[2];
        uint64_t h;
        read_all(F.f, sz, sizeof(sz), nullptr);
        read_all(F.f, &h, sizeof(h), nullptr);
        MGM_REQUIRE(sz[0] == c->L[l].n && sz[1] == c->L[l].k && h == geometry_hash(c, l),
                    "mgm_checkpoint_load: checkpoint does not match this context's levels (level " +
                        std::to_string(l) + ")");
    }
    // read everything first, check the sum, then upload
    uint64_t sum = 1469598103934665603ULL;
    std::vector<std::vector<double>> data;
    std::vector<DBuf<double> *> dst;
    for (int l = 0; l < c->nl; l++)
        for (DBuf<double> *b : level_state(c->L[l])) {
            data.emplace_back(c->L[l].n);
            read_all(F.f, data.back().data(), sizeof(double) * c->L[l].n, &sum);
            dst.push_back(b);
        }
    for (DBuf<double> *b : field_state(c)) {
        data.emplace_back(c->L[0].n);
        read_all(F.f, data.back().data(), sizeof(double) * c->L[0].n, &sum);
        dst.push_back(b);
    }
    uint64_t want;
    read_all(F.f, &want, sizeof(want), nullptr);
    MGM_REQUIRE(want == sum, "mgm_checkpoint_load: checksum mismatch (corrupt file)");
    for (size_t t = 0; t < dst.size(); t++) {
        MGM_REQUIRE(dst[t]->p != nullptr, "mgm_checkpoint_load: call mgm_setup first");
        dst[t]->upload(data[t].data(), data[t].size(), c->s);
    }
    MGM_CUDA(cudaStreamSynchronize(c->s));
}

void write_solution(mgm_ctx *c, const char *path, int pressure_field)
{
    Level &L = c->L[0];
    const int n = L.n;
    DBuf<double> *pb = nullptr;
    if (pressure_field == MGM_FIELD_P) pb = &L.p;
    else if (pressure_field == MGM_FIELD_P_OLD) pb = &c->p_old;
    MGM_REQUIRE(pb != nullptr, "mgm_write_solution: pressure_field must be MGM_FIELD_P or MGM_FIELD_P_OLD");
    std::vector<std::vector<double>> a(7, std::vector<double>(n));
    DBuf<double> *src[7] = {&L.x, &L.y, &L.z, &c->u, &c->v, &c->w, pb};
    for (int t = 0; t < 7; t++) src[t]->download(a[t].data(), n, c->s);
    MGM_CUDA(cudaStreamSynchronize(c->s));
    File F;
    F.f = std::fopen(path, "w");
    MGM_REQUIRE(F.f != nullptr, std::string("mgm_write_solution: unable to open ") + path);
    for (int i = 0; i < n; i++)
        std::fprintf(F.f, "%lf, %lf, %lf, %lf, %lf, %lf, %lf\n", a[0][i], a[1][i], a[2][i], a[3][i], a[4][i], a[5][i],
                     a[6][i]);
    MGM_REQUIRE(std::fflush(F.f) == 0, "mgm_write_solution: write failed");
}

template <class F>
int ioguard(F &&f)
{
    try {
        f();
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    } catch (const std::exception &e) {
        set_error(MGM_ERR_ARG, e.what());
        return MGM_ERR_ARG;
    }
}

}  // namespace
}  // namespace mgm

using namespace mgm;

extern "C" {

int mgm_write_solution(mgm_ctx *c, const char *path, int pressure_field)
{
    return ioguard([&] {
        MGM_REQUIRE(c != nullptr && path != nullptr, "mgm_write_solution: null argument");
        MGM_CUDA(cudaSetDevice(c->device));
        MGM_REQUIRE(c->setup_done, "mgm_write_solution: call mgm_setup first");
        MGM_CUDA(cudaStreamSynchronize(c->s));
        write_solution(c, path, pressure_field);
    });
}

int mgm_checkpoint_save(mgm_ctx *c, const char *path)
{
    return ioguard([&] {
        MGM_REQUIRE(c != nullptr && path != nullptr, "mgm_checkpoint_save: null argument");
        MGM_CUDA(cudaSetDevice(c->device));
        MGM_REQUIRE(c->setup_done, "mgm_checkpoint_save: call mgm_setup first");
        MGM_CUDA(cudaStreamSynchronize(c->s));
        save(c, path);
    });
}

int mgm_checkpoint_load(mgm_ctx *c, const char *path)
{
    return ioguard([&] {
        MGM_REQUIRE(c != nullptr && path != nullptr, "mgm_checkpoint_load: null argument");
        MGM_CUDA(cudaSetDevice(c->device));
        MGM_REQUIRE(c->setup_done, "mgm_checkpoint_load: call mgm_setup first");
        MGM_CUDA(cudaStreamSynchronize(c->s));
        load(c, path);
        // the pressure history of the initial guesses belongs to the run
        // that was interrupted, not to the loaded state
        if (c->hist_ok.p) {
            c->hist_ok.zero(c->s);
            MGM_CUDA(cudaStreamSynchronize(c->s));
        }
    });
}

}  // extern "C"
