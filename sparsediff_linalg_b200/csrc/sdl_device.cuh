// Device-side building blocks shared by the kernels: warp / block scans and
// reductions, the term-flattening search, and shared-memory bitonic sorts.
#pragma once

#include <cuda_runtime.h>
#include <climits>
#include <cstdint>

namespace sdl {

constexpr unsigned FULL_MASK = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        int t = __shfl_up_sync(FULL_MASK, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ long long warp_incl_scan_ll(long long v)
{
    const int lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        long long t = __shfl_up_sync(FULL_MASK, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Number of lanes whose inclusive prefix `incl` is <= u (incl non-decreasing over
// lanes). For 0 <= u < incl[31] this is the lane (entry) that term u belongs to.
__device__ __forceinline__ int warp_entry_of(int incl, int u)
{
    int lo = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1)
    {
        int v = __shfl_sync(FULL_MASK, incl, lo + step - 1);
        if (v <= u) lo += step;
    }
    return lo;
}

template <int THREADS>
__device__ __forceinline__ long long block_incl_scan_ll(long long v)
{
    __shared__ long long warp_tot[THREADS / 32];
    const int lane = lane_id(), w = threadIdx.x >> 5;
    long long incl = warp_incl_scan_ll(v);
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0)
    {
        long long t = lane < THREADS / 32 ? warp_tot[lane] : 0;
        t = warp_incl_scan_ll(t);
        if (lane < THREADS / 32) warp_tot[lane] = t;
    }
    __syncthreads();
    long long r = incl + (w > 0 ? warp_tot[w - 1] : 0);
    __syncthreads();
    return r;
}

template <int THREADS>
__device__ __forceinline__ long long block_reduce_sum_ll(long long v)
{
    __shared__ long long part[THREADS / 32];
    const int lane = lane_id(), w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    if (lane == 0) part[w] = v;
    __syncthreads();
    long long r = 0;
    if (threadIdx.x == 0)
        for (int k = 0; k < THREADS / 32; ++k) r += part[k];
    __syncthreads();
    return r; // valid in thread 0
}

// Inclusive scan over the block for a runtime block size (multiple of 32, <= 1024).
// `scratch` holds >= 32 ints of shared memory. Ends with a barrier.
__device__ __forceinline__ int block_incl_scan_int(int v, int *scratch)
{
    const int lane = lane_id(), w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int incl = warp_incl_scan(v);
    if (lane == 31) scratch[w] = incl;
    __syncthreads();
    if (w == 0)
    {
        int t = lane < nw ? scratch[lane] : 0;
        t = warp_incl_scan(t);
        if (lane < nw) scratch[lane] = t;
    }
    __syncthreads();
    int r = incl + (w > 0 ? scratch[w - 1] : 0);
    __syncthreads();
    return r;
}

__device__ __forceinline__ int next_pow2(int v)
{
    if (v <= 1) return 1;
    return 1 << (32 - __clz(v - 1));
}

// Ascending bitonic sort of P (power of two) keys in shared memory by one warp.
template <class K>
__device__ __forceinline__ void warp_bitonic_sort(K *buf, int P)
{
    const int lane = lane_id();
    for (int k = 2; k <= P; k <<= 1)
    {
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            for (int t = lane; t < (P >> 1); t += 32)
            {
                int i = 2 * t - (t & (j - 1));
                int l = i + j;
                bool asc = (i & k) == 0;
                K a = buf[i], b = buf[l];
                if ((a > b) == asc)
                {
                    buf[i] = b;
                    buf[l] = a;
                }
            }
            __syncwarp();
        }
    }
}

// Same by the whole block (blockDim threads).
template <class K>
__device__ __forceinline__ void block_bitonic_sort(K *buf, int P)
{
    for (int k = 2; k <= P; k <<= 1)
    {
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            for (int t = threadIdx.x; t < (P >> 1); t += blockDim.x)
            {
                int i = 2 * t - (t & (j - 1));
                int l = i + j;
                bool asc = (i & k) == 0;
                K a = buf[i], b = buf[l];
                if ((a > b) == asc)
                {
                    buf[i] = b;
                    buf[l] = a;
                }
            }
            __syncthreads();
        }
    }
}

// First position q in sorted a[0, n) with a[q] >= key.
template <class K>
__device__ __forceinline__ int lower_bound_dev(const K *a, int n, K key)
{
    int lo = 0, hi = n;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (a[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

} // namespace sdl
