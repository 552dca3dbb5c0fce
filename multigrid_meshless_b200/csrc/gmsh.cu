// gmsh.cu -- read_PointStructure (header_files/mesh_functions.h:172-476)
// behind the C ABI: a Gmsh 2.2 ASCII mesh becomes one multigrid level's nodes
// in the state the reference's reader leaves them.
//
// What the reference does, and what this file reproduces:
//  - nodes from $Nodes ("id x y z" lines, ids 1..N in order); the bounding box
//    with min/max started at +1e6 / -1e6;
//  - $Elements: every element line is "id type t1 t2 t3 nodes..." (three
//    integers between the type and the nodes, whatever the tag count says);
//    2D: 2-node lines (type 1) tag both nodes as boundary and add the line's
//    normal (-dy, dx) to both; 3D: 3-node triangles (2) and 4-node quads (3)
//    tag their nodes and add the cross product of the element's edges
//    1->2 and 1->3 to every node; 1-node points (15), and in 3D both ends of
//    2-node lines, are corner nodes; any other line is skipped to its end;
//  - d_avg = sqrt(Lx Ly / num_elem) in 2D, cbrt(Lx Ly Lz / num_elem) in 3D;
//  - the first num_corners nodes are dropped (Gmsh numbers geometric points
//    and curve nodes first) and num_boundary_nodes -= num_corners.
// The normals are left unnormalised, as the reference leaves them
// (correct_normal_directions normalises and orients them later).
//
// The file is scanned on the host (integers as fscanf's %i, i.e. strtol with
// base 0; reals as %lf, i.e. strtod).  The normals are summed on the GPU: each
// node walks its boundary elements in element order, every product and sum
// rounded separately, so the sums are those of the reference's loop.
#include "mgm_internal.cuh"
#include "mgm.h"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

struct mgm_mesh {
    int n = 0, nb = 0, num_elem = 0;
    double d_avg = 0;
    std::vector<double> x, y, z, nx, ny, nz;
    std::vector<unsigned char> btag, corner;
};

namespace mgm {
namespace {

// A cursor over the file's bytes with fscanf's directive semantics.
struct Scan {
    const char *p, *end;
    void ws()
    {
        while (p < end && std::isspace((unsigned char)*p)) p++;
    }
    // "%s " : one whitespace-delimited word
    bool word(std::string &w)
    {
        ws();
        const char *b = p;
        while (p < end && !std::isspace((unsigned char)*p)) p++;
        if (p == b) return false;
        w.assign(b, p);
        ws();
        return true;
    }
    // "%i "
    bool integer(long &v)
    {
        ws();
        if (p >= end) return false;
        char *e = nullptr;
        v = std::strtol(p, &e, 0);
        if (e == p) return false;
        p = e;
        ws();
        return true;
    }
    // "%lf "
    bool real(double &v)
    {
        ws();
        if (p >= end) return false;
        char *e = nullptr;
        v = std::strtod(p, &e);
        if (e == p) return false;
        p = e;
        ws();
        return true;
    }
    // "%*[^\n]\n": the rest of the line (nothing when it is empty), then whitespace
    void rest_of_line()
    {
        if (p >= end || *p == '\n') return;
        while (p < end && *p != '\n') p++;
        ws();
    }
    bool seek(const char *key)
    {
        std::string w;
        while (word(w))
            if (w == key) return true;
        return false;
    }
};

// boundary element: type 1 (2D line), 2 (triangle) or 3 (quad), nodes 0-based
struct BElem {
    int type;
    int v[4];
};

// Sum of the boundary elements' normal contributions at each node, in element order
__global__ void k_mesh_normals(int n, const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const int4 *__restrict__ ev,
                               const int *__restrict__ etype, const int *__restrict__ rowptr,
                               const int *__restrict__ elist, double *__restrict__ nx, double *__restrict__ ny,
                               double *__restrict__ nz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int t = rowptr[i]; t < rowptr[i + 1]; t++) {
        const int e = elist[t];
        const int4 v = ev[e];
        if (etype[e] == 1) {
            const double dx = MGM_SUB(x[v.y], x[v.x]), dy = MGM_SUB(y[v.y], y[v.x]);
            sx = MGM_ADD(sx, -dy);
            sy = MGM_ADD(sy, dx);
        } else {
            const double dx = MGM_SUB(x[v.y], x[v.x]), dy = MGM_SUB(y[v.y], y[v.x]), dz = MGM_SUB(z[v.y], z[v.x]);
            const double dx1 = MGM_SUB(x[v.z], x[v.x]), dy1 = MGM_SUB(y[v.z], y[v.x]),
                         dz1 = MGM_SUB(z[v.z], z[v.x]);
            sx = MGM_ADD(sx, MGM_SUB(MGM_MUL(dy, dz1), MGM_MUL(dz, dy1)));
            sy = MGM_ADD(sy, MGM_SUB(MGM_MUL(dz, dx1), MGM_MUL(dx, dz1)));
            sz = MGM_ADD(sz, MGM_SUB(MGM_MUL(dx, dy1), MGM_MUL(dy, dx1)));
        }
    }
    nx[i] = sx;
    ny[i] = sy;
    nz[i] = sz;
}

mgm_mesh *read_mesh(const char *path, int dim)
{
    MGM_REQUIRE(path != nullptr, "mgm_mesh_read: null path");
    MGM_REQUIRE(dim == 2 || dim == 3, "mgm_mesh_read: dim must be 2 or 3");
    std::FILE *f = std::fopen(path, "rb");
    MGM_REQUIRE(f != nullptr, std::string("mgm_mesh_read: unable to open ") + path);
    std::string buf;
    {
        char chunk[1 << 16];
        size_t got;
        while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.append(chunk, got);
        std::fclose(f);
    }
    Scan sc{buf.c_str(), buf.c_str() + buf.size()};
    const std::string bad = std::string("mgm_mesh_read: ") + path + ": ";
    MGM_REQUIRE(sc.seek("$Nodes"), bad + "no $Nodes section");
    long nn = 0;
    MGM_REQUIRE(sc.integer(nn) && nn > 0 && nn < (1L << 31), bad + "bad node count");
    std::vector<double> X(nn), Y(nn), Z(nn);
    double lo[3] = {1e6, 1e6, 1e6}, hi[3] = {-1e6, -1e6, -1e6};
    for (long i = 0; i < nn; i++) {
        long id;
        double v[3];
        MGM_REQUIRE(sc.integer(id) && sc.real(v[0]) && sc.real(v[1]) && sc.real(v[2]), bad + "truncated $Nodes");
        X[i] = v[0]; Y[i] = v[1]; Z[i] = v[2];
        for (int d = 0; d < 3; d++) {
            if (v[d] < lo[d]) lo[d] = v[d];
            if (v[d] > hi[d]) hi[d] = v[d];
        }
    }
    MGM_REQUIRE(sc.seek("$Elements"), bad + "no $Elements section");
    long ne = 0;
    MGM_REQUIRE(sc.integer(ne) && ne > 0, bad + "bad element count");
    std::vector<unsigned char> BT(nn, 0), CT(nn, 0);
    std::vector<BElem> be;
    auto node = [&](long &v) {
        MGM_REQUIRE(sc.integer(v) && v >= 1 && v <= nn, bad + "element node out of range");
        return (int)(v - 1);
    };
    for (long e = 0; e < ne; e++) {
        long id, type, t;
        MGM_REQUIRE(sc.integer(id) && sc.integer(type), bad + "truncated $Elements");
        const bool line2 = dim == 2 && type == 1, tri = dim == 3 && type == 2, quad = dim == 3 && type == 3;
        const bool line3 = dim == 3 && type == 1, point = type == 15;
        if (!(line2 || tri || quad || line3 || point)) {
            sc.rest_of_line();
            continue;
        }
        for (int q = 0; q < 3; q++) MGM_REQUIRE(sc.integer(t), bad + "truncated element tags");
        long v;
        if (point) {
            CT[node(v)] = 1;
        } else if (line3) {
            const int a = node(v), b = node(v);
            CT[a] = 1;
            CT[b] = 1;
        } else {
            BElem el{line2 ? 1 : (tri ? 2 : 3), {-1, -1, -1, -1}};
            const int cnt = line2 ? 2 : (tri ? 3 : 4);
            for (int q = 0; q < cnt; q++) {
                el.v[q] = node(v);
                BT[el.v[q]] = 1;
            }
            be.push_back(el);
        }
    }
    // element-ordered incidence lists of the boundary elements' nodes
    std::vector<int> rowptr(nn + 1, 0), elist;
    for (const BElem &el : be)
        for (int q = 0; q < 4; q++)
            if (el.v[q] >= 0) rowptr[el.v[q] + 1]++;
    for (long i = 0; i < nn; i++) rowptr[i + 1] += rowptr[i];
    elist.resize(rowptr[nn]);
    {
        std::vector<int> fill(rowptr.begin(), rowptr.end() - 1);
        for (size_t e = 0; e < be.size(); e++)
            for (int q = 0; q < 4; q++)
                if (be[e].v[q] >= 0) elist[fill[be[e].v[q]]++] = (int)e;
    }
    std::vector<int4> ev(be.size());
    std::vector<int> et(be.size());
    for (size_t e = 0; e < be.size(); e++) {
        ev[e] = make_int4(be[e].v[0], be[e].v[1], be[e].v[2], be[e].v[3]);
        et[e] = be[e].type;
    }
    std::vector<double> NX(nn), NY(nn), NZ(nn);
    {
        cudaStream_t s;
        MGM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            DBuf<double> dx(nn), dy(nn), dz(nn), dnx(nn), dny(nn), dnz(nn);
            DBuf<int4> dev(std::max<size_t>(be.size(), 1));
            DBuf<int> det(std::max<size_t>(be.size(), 1)), drp(nn + 1), del(std::max<size_t>(elist.size(), 1));
            dx.upload(X.data(), nn, s); dy.upload(Y.data(), nn, s); dz.upload(Z.data(), nn, s);
            dev.upload(ev.data(), ev.size(), s); det.upload(et.data(), et.size(), s);
            drp.upload(rowptr.data(), nn + 1, s); del.upload(elist.data(), elist.size(), s);
            k_mesh_normals<<<blocks_for(nn, 256), 256, 0, s>>>((int)nn, dx.p, dy.p, dz.p, dev.p, det.p, drp.p, del.p,
                                                               dnx.p, dny.p, dnz.p);
            MGM_LAUNCHED();
            dnx.download(NX.data(), nn, s); dny.download(NY.data(), nn, s); dnz.download(NZ.data(), nn, s);
            MGM_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        MGM_CUDA(cudaStreamDestroy(s));
    }
    long nbnd = 0, ncorner = 0;
    for (long i = 0; i < nn; i++) { nbnd += BT[i] != 0; ncorner += CT[i] != 0; }
    MGM_REQUIRE(ncorner < nn, bad + "every node is a corner node");
    mgm_mesh *m = new mgm_mesh();
    m->n = (int)(nn - ncorner);
    m->nb = (int)(nbnd - ncorner);
    m->num_elem = (int)ne;
    const double L0 = hi[0] - lo[0], L1 = hi[1] - lo[1], L2 = hi[2] - lo[2];
    m->d_avg = dim == 2 ? std::sqrt(L0 * L1 / (double)ne) : std::cbrt(L0 * L1 * L2 / (double)ne);
    auto tail = [&](auto &dst, const auto &src) { dst.assign(src.begin() + ncorner, src.end()); };
    tail(m->x, X); tail(m->y, Y); tail(m->z, Z);
    tail(m->nx, NX); tail(m->ny, NY); tail(m->nz, NZ);
    tail(m->btag, BT); tail(m->corner, CT);
    return m;
}

template <class F>
int gguard(F &&f)
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

int mgm_mesh_read(const char *path, int dim, mgm_mesh **mesh)
{
    return gguard([&] {
        MGM_REQUIRE(mesh != nullptr, "mgm_mesh_read: null output");
        *mesh = nullptr;
        *mesh = read_mesh(path, dim);
    });
}

int mgm_mesh_info(const mgm_mesh *m, int *num_nodes, int *num_boundary_nodes, int *num_elem, double *d_avg)
{
    return gguard([&] {
        MGM_REQUIRE(m != nullptr, "mgm_mesh_info: null mesh");
        if (num_nodes) *num_nodes = m->n;
        if (num_boundary_nodes) *num_boundary_nodes = m->nb;
        if (num_elem) *num_elem = m->num_elem;
        if (d_avg) *d_avg = m->d_avg;
    });
}

int mgm_mesh_get(const mgm_mesh *m, double *x, double *y, double *z, double *nx, double *ny, double *nz,
                 unsigned char *boundary_tag, unsigned char *corner_tag)
{
    return gguard([&] {
        MGM_REQUIRE(m != nullptr, "mgm_mesh_get: null mesh");
        auto out = [&](auto *dst, const auto &src) {
            if (dst) std::copy(src.begin(), src.end(), dst);
        };
        out(x, m->x); out(y, m->y); out(z, m->z);
        out(nx, m->nx); out(ny, m->ny); out(nz, m->nz);
        out(boundary_tag, m->btag); out(corner_tag, m->corner);
    });
}

void mgm_mesh_free(mgm_mesh *m) { delete m; }

}  // extern "C"
