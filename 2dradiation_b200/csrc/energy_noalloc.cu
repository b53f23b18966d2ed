// Global-energy reduction that allocates nothing: the partial sums live in a
// file-scope device array instead of memory obtained from cudaMalloc.
//
// It serves callers that cannot allocate device memory at the time they need
// the number but can pass device pointers to data they own: monitoring loops
// whose device-memory budget is fixed up front (an allocation there could fail
// or stall mid-run), and host applications that embed the library and route
// every device allocation through their own pool (a library-side cudaMalloc
// would bypass its accounting and synchronise the device).
//
// Limits and sharing (also stated in include/grlbm.h):
//   * at most kNoAllocPartials partial sums of kNoAllocCellsPerPartial interior
//     cells each, i.e. nx_ * ny_ <= 2,097,152 interior cells; larger grids are
//     rejected with GRLBM_ERR_ARGUMENT;
//   * every call on a device shares the one array, which keeps the previous
//     call's partial sums; each call rewrites every partial it reads, so
//     nothing needs clearing, but calls whose work overlaps on the GPU (two
//     streams, or two host threads) race on the array and must be ordered by
//     the caller;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before capturing a stream into a CUDA graph.  The cache
//     is never invalidated: after a cudaDeviceReset in the host process the
//     cached address is stale, so a process that resets a device must not
//     call this entry point on that device again.
#include <cuda_runtime.h>

#include <mutex>

#include <cstdio>

#include "../../include/grlbm.h"
#include "device_common.cuh"

namespace
{
constexpr int kNoAllocCellsPerPartial = 256;
constexpr int kNoAllocPartials = 8192;
constexpr int kMaxDevices = 64;

// the scratch: one FP64 partial sum per block of kNoAllocCellsPerPartial cells
static __device__ __align__(256) double g_energy_partials[kNoAllocPartials];

double *g_partials_addr[kMaxDevices] = {nullptr};
std::mutex g_partials_mutex;

// First pass: block b sums the interior E of cells [256 b, 256 b + 256) in a
// fixed order (interior cell c -> node (1 + c % nx_, 1 + c / nx_)).
__global__ void __launch_bounds__(kNoAllocCellsPerPartial)
    k_energy_blocks(const double *E, int64_t nx, int64_t nx_, int64_t ncell, double *partials)
{
    __shared__ double s[kNoAllocCellsPerPartial];
    const int t = threadIdx.x;
    const int64_t c = (int64_t)blockIdx.x * kNoAllocCellsPerPartial + t;
    s[t] = c < ncell ? E[(1 + c % nx_) + (1 + c / nx_) * nx] : 0.0;
    __syncthreads();
    for (int w = kNoAllocCellsPerPartial / 2; w > 0; w >>= 1)
    {
        if (t < w)
            s[t] += s[t + w];
        __syncthreads();
    }
    if (t == 0)
        partials[blockIdx.x] = s[0];
}

// Second pass: one block folds the partials in a fixed order.
__global__ void __launch_bounds__(256) k_energy_fold(const double *partials, int n, double *out)
{
    __shared__ double s[256];
    const int t = threadIdx.x;
    double acc = 0.0;
    for (int k = t; k < n; k += 256)
        acc += partials[k];
    s[t] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1)
    {
        if (t < w)
            s[t] += s[t + w];
        __syncthreads();
    }
    if (t == 0)
        *out = s[0];
}

// Device address of the scratch array on the current device (looked up once).
cudaError_t partials_address(double **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (dev < 0 || dev >= kMaxDevices)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_partials_mutex);
    if (!g_partials_addr[dev])
    {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_energy_partials);
        if (e != cudaSuccess)
            return e;
        g_partials_addr[dev] = static_cast<double *>(p);
    }
    *out = g_partials_addr[dev];
    return cudaSuccess;
}
} // namespace

extern "C" int grlbm_energy_noalloc(const double *E, int64_t nx_, int64_t ny_, double *total, void *stream)
{
    if (!E || !total || nx_ < 1 || ny_ < 1)
    {
        grlbm::set_global_error("grlbm_energy_noalloc: null pointer or empty grid");
        return GRLBM_ERR_ARGUMENT;
    }
    // each size checked on its own first, so that nx_ * ny_ cannot overflow
    constexpr int64_t kMaxCells = (int64_t)kNoAllocPartials * kNoAllocCellsPerPartial;
    if (nx_ > kMaxCells || ny_ > kMaxCells / nx_)
    {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "grlbm_energy_noalloc: %lld x %lld interior cells exceed its fixed scratch (at most %lld)",
                 (long long)nx_, (long long)ny_, (long long)kMaxCells);
        grlbm::set_global_error(msg);
        return GRLBM_ERR_ARGUMENT;
    }
    const int64_t ncell = nx_ * ny_;
    const int64_t blocks = (ncell + kNoAllocCellsPerPartial - 1) / kNoAllocCellsPerPartial;
    if (blocks > kNoAllocPartials)
    {
        char msg[160];
        snprintf(msg, sizeof msg,
                 "grlbm_energy_noalloc: %lld interior cells exceed its fixed scratch (at most %d)",
                 (long long)ncell, kNoAllocPartials * kNoAllocCellsPerPartial);
        grlbm::set_global_error(msg);
        return GRLBM_ERR_ARGUMENT;
    }
    double *partials = nullptr;
    if (partials_address(&partials) != cudaSuccess)
    {
        grlbm::set_global_error("grlbm_energy_noalloc: cannot look up the scratch array on this device");
        return GRLBM_ERR_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // an error left by earlier, unrelated asynchronous work is not this call's
    (void)cudaGetLastError();
    k_energy_blocks<<<(unsigned)blocks, kNoAllocCellsPerPartial, 0, s>>>(E, nx_ + 2, nx_, ncell, partials);
    k_energy_fold<<<1, 256, 0, s>>>(partials, (int)blocks, total);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
    {
        char msg[200];
        snprintf(msg, sizeof msg, "grlbm_energy_noalloc: kernel launch failed: %s", cudaGetErrorString(e));
        grlbm::set_global_error(msg);
        return GRLBM_ERR_CUDA;
    }
    return GRLBM_OK;
}
