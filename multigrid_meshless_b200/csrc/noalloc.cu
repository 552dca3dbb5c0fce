// noalloc.cu -- average node spacing without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: applications whose device
// memory is entirely owned by another allocator (a framework's caching
// allocator or a fixed arena sized at start-up), and loops that cannot afford
// the device-wide synchronisation and pool fragmentation that cudaMalloc /
// cudaFree bring.  mgm_avg_dx_noalloc serves them: it computes what
// mgm_avg_dx computes, on device buffers the caller owns, and keeps its only
// scratch -- the per-node length array -- in a fixed file-scope device array.
//
// That array (MGM_NOALLOC_MAX_NODES doubles, 16 MiB) is reserved on every GPU
// that loads this library, for the life of the process.  All calls share it and
// it keeps the last call's contents, so calls that overlap on the GPU (from
// different streams or threads) race; serialise them.
#include <mutex>

#include "../../include/mgm.h"
#include "mgm_internal.cuh"

namespace mgm {

// kernels of calculate_avg_dx (setup.cu)
__global__ void k_spacing(int n, int k, int dim, const double *x, const double *y, const double *z, const uint8_t *btag,
                          const int *cloud, double *len);
__global__ void k_ordered_sum(int n, const double *len, double *out);

static __device__ __align__(256) double g_spacing_scratch[MGM_NOALLOC_MAX_NODES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
double *g_scratch_addr[kMaxDevices] = {nullptr};

// The device address of g_spacing_scratch on the current device, looked up
// once per device (the host-side name of the array is not a device address).
// The address is kept for the life of the process: a cudaDeviceReset after
// the first call would leave it stale, which the header states is not
// supported.  The caller's stream must belong to the current device.
double *scratch_for_current_device()
{
    int dev = 0;
    MGM_CUDA(cudaGetDevice(&dev));
    MGM_REQUIRE(dev >= 0 && dev < kMaxDevices, "mgm_avg_dx_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        MGM_CUDA(cudaGetSymbolAddress(&p, g_spacing_scratch));
        MGM_REQUIRE(p != nullptr, "mgm_avg_dx_noalloc: scratch array has no device address");
        g_scratch_addr[dev] = (double *)p;
    }
    return g_scratch_addr[dev];
}
}  // namespace

}  // namespace mgm

using namespace mgm;

extern "C" int mgm_avg_dx_noalloc(int n, int k, int dim, const double *d_x, const double *d_y, const double *d_z,
                                  const unsigned char *d_btag, const int *d_cloud, double *d_avg, void *stream)
{
    try {
        MGM_REQUIRE(n >= 1, "mgm_avg_dx_noalloc: n must be >= 1");
        MGM_REQUIRE(n <= MGM_NOALLOC_MAX_NODES,
                    "mgm_avg_dx_noalloc: n = " + std::to_string(n) + " exceeds the fixed scratch of " +
                        std::to_string(MGM_NOALLOC_MAX_NODES) + " nodes (use mgm_avg_dx)");
        MGM_REQUIRE(k >= 2, "mgm_avg_dx_noalloc: k must be >= 2");
        MGM_REQUIRE(dim == 2 || dim == 3, "mgm_avg_dx_noalloc: dim must be 2 or 3");
        MGM_REQUIRE(d_x && d_y && d_z && d_btag && d_cloud && d_avg, "mgm_avg_dx_noalloc: null pointer");
        double *len = scratch_for_current_device();
        cudaStream_t s = (cudaStream_t)stream;
        // every entry len[0..n) is written before it is read: nothing to clear
        k_spacing<<<blocks_for(n, 256), 256, 0, s>>>(n, k, dim, d_x, d_y, d_z, d_btag, d_cloud, len);
        MGM_LAUNCHED();
        k_ordered_sum<<<1, 1, 0, s>>>(n, len, d_avg);
        MGM_LAUNCHED();
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}
