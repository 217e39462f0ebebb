// Stable transpose of a compressed structure on the GPU.
//
// Upstream (src/sparse/CSC_matrix.c:62-104, CSR_matrix.c:144-187) transposes by a
// serial counting sort: count entries per column, scan, then scatter the entries in
// row-major order, which leaves the source rows ascending inside every column. Here
// the count and scatter run in parallel with atomics, which loses the order, so
// each entry carries its source position e and every output segment is then
// sorted by e; because source positions grow in row-major order, that restores
// exactly upstream's order (ties inside one source row included).
//
// Segments are sorted by size class: <= 32 keys in registers by one warp, <= 1024
// in shared memory by one warp, <= 8192 in shared memory by one CTA, larger ones by
// a CTA merge sort through a global scratch buffer.
#include <algorithm>
#include <vector>

#include "sdl_device.cuh"
#include "sdl_internal.h"

namespace sdl {
namespace {

constexpr int SCATTER_TILE = 2048;

__global__ void k_count_idx(const int *__restrict__ idx, int nnz, int *__restrict__ cnt)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz;
         e += (long long)gridDim.x * blockDim.x)
        atomicAdd(&cnt[idx[e]], 1);
}

// Last r in [lo, hi) with p[r] <= e (p non-decreasing, p[lo] <= e < p[hi]).
__device__ __forceinline__ int row_of(const int *p, int lo, int hi, int e)
{
    while (hi - lo > 1)
    {
        int mid = (lo + hi) >> 1;
        if (p[mid] <= e)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// keys[Tp[c] + slot] = (e << 32) | row for every source entry e = (row, c).
__global__ void k_scatter_keys(const int *__restrict__ p, const int *__restrict__ idx,
                               int rows, int nnz, const int *__restrict__ Tp,
                               int *__restrict__ fill, unsigned long long *__restrict__ keys)
{
    __shared__ int r_lo, r_hi;
    long long e0 = (long long)blockIdx.x * SCATTER_TILE;
    long long e1 = min((long long)nnz, e0 + SCATTER_TILE);
    if (e0 >= e1) return;
    if (p && threadIdx.x == 0)
    {
        r_lo = row_of(p, 0, rows, (int)e0);
        r_hi = row_of(p, r_lo, rows, (int)(e1 - 1)) + 1;
    }
    __syncthreads();
    for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x)
    {
        int r = p ? row_of(p, r_lo, r_hi, (int)e) : (int)e;
        int c = idx[e];
        int slot = atomicAdd(&fill[c], 1);
        keys[Tp[c] + slot] = ((unsigned long long)e << 32) | (unsigned)r;
    }
}

// size classes of segments
enum
{
    SEG_W32 = 0,
    SEG_W1K,
    SEG_C8K,
    SEG_BIG,
    SEG_NCLS
};

__global__ void k_seg_classify(const int *__restrict__ off, int nseg, int *__restrict__ counts,
                               int *__restrict__ list_pos, unsigned char *__restrict__ cls)
{
    __shared__ int sh[SEG_NCLS];
    if (threadIdx.x < SEG_NCLS) sh[threadIdx.x] = 0;
    __syncthreads();
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nseg;
         s += (long long)gridDim.x * blockDim.x)
    {
        int len = off[s + 1] - off[s];
        int c = len <= 1 ? 255 : len <= 32 ? SEG_W32 : len <= 1024 ? SEG_W1K : len <= 8192 ? SEG_C8K : SEG_BIG;
        cls[s] = (unsigned char)c;
        if (c != 255) atomicAdd(&sh[c], 1);
    }
    __syncthreads();
    if (threadIdx.x < SEG_NCLS && sh[threadIdx.x]) atomicAdd(&counts[threadIdx.x], sh[threadIdx.x]);
    (void)list_pos;
}

__global__ void k_seg_scatter(const unsigned char *__restrict__ cls, int nseg,
                              int *__restrict__ cursor, int *__restrict__ lists)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nseg;
         s += (long long)gridDim.x * blockDim.x)
    {
        int c = cls[s];
        if (c == 255) continue;
        int at = atomicAdd(&cursor[c], 1);
        lists[at] = (int)s;
    }
}

// <= 32 keys: one warp, keys in registers, shuffle bitonic network.
__global__ void k_segsort_w32(const int *__restrict__ list, int count, const int *__restrict__ off,
                              unsigned long long *__restrict__ keys)
{
    const int lane = lane_id();
    const int wpb = blockDim.x >> 5;
    for (long long w = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); w < count;
         w += (long long)gridDim.x * wpb)
    {
        int s = list[w];
        int b = off[s], len = off[s + 1] - b;
        unsigned long long v = lane < len ? keys[b + lane] : ~0ull;
#pragma unroll
        for (int k = 2; k <= 32; k <<= 1)
        {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1)
            {
                unsigned long long o = __shfl_xor_sync(FULL_MASK, v, j);
                bool lower = (lane & j) == 0;
                bool asc = (lane & k) == 0;
                // keep min if (lower == asc), else max
                bool take_min = (lower == asc);
                v = take_min ? (o < v ? o : v) : (o > v ? o : v);
            }
        }
        if (lane < len) keys[b + lane] = v;
    }
}

// <= 1024 keys: one warp per segment, shared-memory bitonic.
__global__ void k_segsort_w1k(const int *__restrict__ list, int count, const int *__restrict__ off,
                              unsigned long long *__restrict__ keys)
{
    extern __shared__ unsigned long long smk[];
    const int lane = lane_id();
    const int wpb = blockDim.x >> 5;
    unsigned long long *buf = smk + (threadIdx.x >> 5) * 1024;
    for (long long w = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); w < count;
         w += (long long)gridDim.x * wpb)
    {
        int s = list[w];
        int b = off[s], len = off[s + 1] - b;
        int P = next_pow2(len);
        for (int q = lane; q < P; q += 32) buf[q] = q < len ? keys[b + q] : ~0ull;
        __syncwarp();
        warp_bitonic_sort(buf, P);
        for (int q = lane; q < len; q += 32) keys[b + q] = buf[q];
        __syncwarp();
    }
}

// <= 8192 keys: one CTA per segment.
__global__ void k_segsort_c8k(const int *__restrict__ list, int count, const int *__restrict__ off,
                              unsigned long long *__restrict__ keys)
{
    extern __shared__ unsigned long long smk[];
    for (int w = blockIdx.x; w < count; w += gridDim.x)
    {
        int s = list[w];
        int b = off[s], len = off[s + 1] - b;
        int P = next_pow2(len);
        for (int q = threadIdx.x; q < P; q += blockDim.x) smk[q] = q < len ? keys[b + q] : ~0ull;
        __syncthreads();
        block_bitonic_sort(smk, P);
        for (int q = threadIdx.x; q < len; q += blockDim.x) keys[b + q] = smk[q];
        __syncthreads();
    }
}

constexpr int BIG_CHUNK = 8192;

// Big segments: sort BIG_CHUNK-sized chunks in shared memory, then merge runs
// pairwise (merge path per thread) between keys and scratch until one run is left.
__global__ void k_segsort_big(const int *__restrict__ list, int count, const int *__restrict__ off,
                              unsigned long long *__restrict__ keys,
                              unsigned long long *__restrict__ scratch)
{
    extern __shared__ unsigned long long smk[];
    for (int w = blockIdx.x; w < count; w += gridDim.x)
    {
        int s = list[w];
        int b = off[s], len = off[s + 1] - b;
        unsigned long long *src = keys + b, *dst = scratch + b;
        for (int c0 = 0; c0 < len; c0 += BIG_CHUNK)
        {
            int cl = min(BIG_CHUNK, len - c0);
            int P = next_pow2(cl);
            for (int q = threadIdx.x; q < P; q += blockDim.x) smk[q] = q < cl ? src[c0 + q] : ~0ull;
            __syncthreads();
            block_bitonic_sort(smk, P);
            for (int q = threadIdx.x; q < cl; q += blockDim.x) src[c0 + q] = smk[q];
            __syncthreads();
        }
        bool in_src = true;
        for (int width = BIG_CHUNK; width < len; width <<= 1)
        {
            const unsigned long long *in = in_src ? src : dst;
            unsigned long long *out = in_src ? dst : src;
            for (int ps = 0; ps < len; ps += 2 * width)
            {
                int na = min(width, len - ps);
                int nb = max(0, min(width, len - ps - width));
                const unsigned long long *A = in + ps, *B = in + ps + na;
                int tot = na + nb;
                int per = (tot + blockDim.x - 1) / blockDim.x;
                int d0 = min(tot, (int)threadIdx.x * per), d1 = min(tot, d0 + per);
                if (d0 < d1)
                {
                    int lo = max(0, d0 - nb), hi = min(d0, na);
                    while (lo < hi)
                    {
                        int mid = (lo + hi) >> 1;
                        if (A[mid] < B[d0 - 1 - mid])
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    int i = lo, j = d0 - lo;
                    for (int d = d0; d < d1; ++d)
                    {
                        bool takeA = j >= nb || (i < na && A[i] < B[j]);
                        out[ps + d] = takeA ? A[i++] : B[j++];
                    }
                }
            }
            __syncthreads();
            in_src = !in_src;
        }
        if (!in_src)
        {
            for (int q = threadIdx.x; q < len; q += blockDim.x) src[q] = dst[q];
            __syncthreads();
        }
    }
}

__global__ void k_unpack_keys(const unsigned long long *__restrict__ keys, int n,
                              int *__restrict__ Ti, int *__restrict__ src)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x)
    {
        unsigned long long k = keys[q];
        src[q] = (int)(k >> 32);
        Ti[q] = (int)(k & 0xffffffffu);
    }
}

} // namespace

// Sort every segment [off[s], off[s+1]) of keys ascending (keys unique per segment).
void segment_sort_u64(unsigned long long *d_keys, const int *d_off, int nseg, int nkeys,
                      cudaStream_t s)
{
    if (nseg <= 0 || nkeys <= 1) return;
    Runtime &rt = runtime();
    DevBuf<int> counts(2 * SEG_NCLS);
    DevBuf<unsigned char> cls(nseg);
    SDL_CUDA(cudaMemsetAsync(counts.get(), 0, counts.bytes(), s));
    int grid = (int)std::min<long long>((nseg + 255) / 256, (long long)rt.num_sms * 8);
    SDL_LAUNCH(k_seg_classify, grid, 256, 0, s, d_off, nseg, counts.get(), nullptr, cls.get());
    int h[SEG_NCLS];
    SDL_CUDA(cudaMemcpyAsync(h, counts.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    SDL_CUDA(cudaStreamSynchronize(s));
    int start[SEG_NCLS + 1];
    start[0] = 0;
    for (int c = 0; c < SEG_NCLS; ++c) start[c + 1] = start[c] + h[c];
    if (start[SEG_NCLS] == 0) return;
    DevBuf<int> lists(start[SEG_NCLS]);
    SDL_CUDA(cudaMemcpyAsync(counts.get() + SEG_NCLS, start, SEG_NCLS * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    SDL_LAUNCH(k_seg_scatter, grid, 256, 0, s, cls.get(), nseg, counts.get() + SEG_NCLS,
               lists.get());
    const int cap = rt.num_sms * 16;
    if (h[SEG_W32])
    {
        int g = std::min((h[SEG_W32] + 7) / 8, cap);
        SDL_LAUNCH(k_segsort_w32, g, 256, 0, s, lists.get() + start[SEG_W32], h[SEG_W32], d_off,
                   d_keys);
    }
    if (h[SEG_W1K])
    {
        int g = std::min((h[SEG_W1K] + 3) / 4, cap);
        size_t sm = 4 * 1024 * sizeof(unsigned long long);
        SDL_CUDA(cudaFuncSetAttribute(k_segsort_w1k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        SDL_LAUNCH(k_segsort_w1k, g, 128, sm, s, lists.get() + start[SEG_W1K], h[SEG_W1K], d_off,
                   d_keys);
    }
    if (h[SEG_C8K] || h[SEG_BIG])
    {
        size_t sm = 8192 * sizeof(unsigned long long);
        SDL_CUDA(cudaFuncSetAttribute(k_segsort_c8k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        SDL_CUDA(cudaFuncSetAttribute(k_segsort_big, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        if (h[SEG_C8K])
        {
            int g = std::min(h[SEG_C8K], cap);
            SDL_LAUNCH(k_segsort_c8k, g, 512, sm, s, lists.get() + start[SEG_C8K], h[SEG_C8K],
                       d_off, d_keys);
        }
        if (h[SEG_BIG])
        {
            DevBuf<unsigned long long> scratch(nkeys);
            int g = std::min(h[SEG_BIG], rt.num_sms);
            SDL_LAUNCH(k_segsort_big, g, 1024, sm, s, lists.get() + start[SEG_BIG], h[SEG_BIG],
                       d_off, d_keys, scratch.get());
            SDL_CUDA(cudaStreamSynchronize(s)); // scratch is freed on return
        }
    }
    SDL_CUDA(cudaStreamSynchronize(s)); // lists / cls are freed on return
}

void transpose_build(const int *d_p, const int *d_idx, int rows, int cols, int nnz,
                     TransposePlan &out, cudaStream_t s)
{
    Runtime &rt = runtime();
    out.rows = rows;
    out.cols = cols;
    out.nnz = nnz;
    out.Tp.reset((size_t)cols + 1);
    out.Ti.reset(nnz);
    out.src.reset(nnz);
    if (nnz == 0)
    {
        SDL_CUDA(cudaMemsetAsync(out.Tp.get(), 0, out.Tp.bytes(), s));
        SDL_CUDA(cudaStreamSynchronize(s));
        return;
    }
    DevBuf<int> cnt((size_t)cols + 1);
    SDL_CUDA(cudaMemsetAsync(cnt.get(), 0, cnt.bytes(), s));
    int grid = (int)std::min<long long>((nnz + 255) / 256, (long long)rt.num_sms * 8);
    SDL_LAUNCH(k_count_idx, grid, 256, 0, s, d_idx, nnz, cnt.get());
    exclusive_scan_i32_checked(cnt.get(), out.Tp.get(), cols, s);
    SDL_CUDA(cudaMemsetAsync(cnt.get(), 0, cnt.bytes(), s));
    DevBuf<unsigned long long> keys(nnz);
    int tiles = (int)((nnz + SCATTER_TILE - 1) / SCATTER_TILE);
    SDL_LAUNCH(k_scatter_keys, tiles, 256, 0, s, d_p, d_idx, rows, nnz, out.Tp.get(), cnt.get(),
               keys.get());
    segment_sort_u64(keys.get(), out.Tp.get(), cols, nnz, s);
    SDL_LAUNCH(k_unpack_keys, grid, 256, 0, s, keys.get(), nnz, out.Ti.get(), out.src.get());
    SDL_CUDA(cudaStreamSynchronize(s));
}

} // namespace sdl
