// Pieces shared by the warp-per-tile step kernels of the fixed streaming
// types (kernels_step32.cu in FP32, kernels_step64.cu in FP64): the tile
// counter, the warps' buffers in shared memory, the staging waits and the
// lambda-iteration statistics.
#pragma once
#include "tma_util.cuh"

namespace grlbm
{
namespace step
{
// time limits of a staging wait (a copy lands within microseconds) and of the
// drain of a copy in flight after a wait has run out
constexpr unsigned long long kWaitNs = 200000000ull, kDrainNs = 2000000000ull;

__device__ __forceinline__ unsigned char *align128(unsigned char *p)
{
    const unsigned a = smem_addr(p);
    return p + ((128u - (a & 127u)) & 127u);
}

// the warp's buffers in the block's shared memory, from the first 128-byte
// boundary past `header` bytes
template <class T>
__device__ __forceinline__ T *warp_buffers(unsigned char *smem, int header, int warp_stride)
{
    const int warp = threadIdx.x >> 5;
    return reinterpret_cast<T *>(align128(smem + header) + (size_t)warp * (size_t)warp_stride);
}

// Per-warp running statistics of the lambda iteration.
struct IterStats
{
    unsigned long long sum;
    unsigned max;
};

// The warp's statistics (each lane counted its own cells), summed and
// maximised over the lanes, one atomic each.  Called by the whole warp.
__device__ __forceinline__ void flush_stats(const IterStats &st, unsigned long long *iter_sum, unsigned *iter_max)
{
    unsigned long long sum = st.sum;
    unsigned mx = st.max;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0 && sum)
    {
        atomicAdd(iter_sum, sum);
        atomicMax(iter_max, mx);
    }
}

__device__ __forceinline__ int take_tile(unsigned *counter)
{
    int t = 0;
    if ((threadIdx.x & 31) == 0)
        t = (int)atomicAdd(counter, 1u);
    return __shfl_sync(0xffffffffu, t, 0);
}

// The warp is done taking tiles from counter[0]; the launch's last warp
// (of gridDim.x * warps_per_block) clears both words for the next launch.
__device__ __forceinline__ void retire_warp(unsigned *counter, unsigned warps_per_block)
{
    if ((threadIdx.x & 31) == 0)
    {
        __threadfence(); // this warp's last take is ordered before its retirement
        if (atomicAdd(counter + 1, 1u) == gridDim.x * warps_per_block - 1u)
        {
            counter[0] = 0u;
            counter[1] = 0u;
        }
    }
}

// Waits for the warp's staged patch; on a timeout raises the fault word and
// lets the copy in flight land (bounded) before the warp stops.
__device__ __forceinline__ bool wait_tile(unsigned bar, unsigned &parity, unsigned *fault)
{
    const bool landed = mbar_wait(bar, parity, kWaitNs, fault);
    if (!__all_sync(0xffffffffu, landed))
    {
        if ((threadIdx.x & 31) == 0 && fault)
            *reinterpret_cast<volatile unsigned *>(fault) = 1u;
        mbar_wait(bar, parity, kDrainNs, nullptr);
        return false;
    }
    parity ^= 1u;
    return true;
}
} // namespace step
} // namespace grlbm
