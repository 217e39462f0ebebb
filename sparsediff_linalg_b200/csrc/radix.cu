// Stable LSD radix sort of (32-bit key, 8-byte payload) pairs, 8 bits per pass.
// Used once per pattern to group the terms of the rows beyond the tile budget by
// output: stability keeps, inside every output, the input order -- upstream's
// visiting order.
//
// Per pass: a 256-bin digit histogram per tile of 4096 pairs, an exclusive scan of
// the histograms in (digit, tile) order, then a scatter in which each warp ranks its
// 512 pairs in order (match_any over the digit; per-warp running counts in shared
// memory), so equal digits keep their input order across warps, tiles and passes;
// the tile is reordered by digit in shared memory before it is written out.
#include <algorithm>

#include <mutex>
#include <unordered_set>

#include "sdl_device.cuh"
#include "sdl_internal.h"

namespace sdl {
namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_PER_WARP = 512;
constexpr int RS_TILE = RS_WARPS * RS_PER_WARP; // 4096 pairs per tile

__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const unsigned *__restrict__ keys, int n, int shift,
                                                        int ntiles, int *__restrict__ hist)
{
    __shared__ int cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * RS_TILE;
    for (int k = threadIdx.x; k < RS_TILE; k += RS_THREADS)
    {
        const long long i = base + k;
        if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[(long long)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// Scatter of one tile: every pair's rank among the tile's pairs of its digit (warps
// rank their 512 pairs in order with match_any; per-warp running counts in shared
// memory), the tile reordered by digit in shared memory, then written out in that
// order: the pairs of one digit go to consecutive positions, so the writes of
// neighbouring threads land next to each other.
constexpr size_t RS_SCATTER_SMEM = (size_t)RS_TILE * (sizeof(unsigned) + sizeof(uint2)) +
                                   (size_t)(RS_WARPS + 1) * 256 * sizeof(int);

__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const unsigned *__restrict__ keys,
                                                           const uint2 *__restrict__ vals, int n, int shift,
                                                           int ntiles, const int *__restrict__ offs,
                                                           unsigned *__restrict__ okeys, uint2 *__restrict__ ovals)
{
    extern __shared__ __align__(16) unsigned char rs_smem[];
    uint2 *sv = reinterpret_cast<uint2 *>(rs_smem);
    unsigned *sk = reinterpret_cast<unsigned *>(sv + RS_TILE);
    int(*wc)[256] = reinterpret_cast<int(*)[256]>(sk + RS_TILE);
    int *tstart = &wc[RS_WARPS][0];
    const int lane = lane_id(), w = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < RS_WARPS * 256; k += RS_THREADS) (&wc[0][0])[k] = 0;
    __syncthreads();
    const long long tbase = (long long)blockIdx.x * RS_TILE;
    const int tn = (int)min((long long)RS_TILE, (long long)n - tbase); // pairs of this tile
    const long long wbase = tbase + (long long)w * RS_PER_WARP;
    // counts per warp and digit
    for (int r = 0; r < RS_PER_WARP; r += 32)
    {
        const long long i = wbase + r + lane;
        if (i < n) atomicAdd(&wc[w][(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    // tile-local first position of every (warp, digit): digits in order, warps in
    // order inside a digit
    {
        const int d = threadIdx.x; // RS_THREADS == 256 digits
        int c = 0;
        for (int ww = 0; ww < RS_WARPS; ++ww) c += wc[ww][d];
        // exclusive scan of the digit totals over the block
        __shared__ int scr[32];
        const int incl = block_incl_scan_int(c, scr);
        int run = incl - c;
        tstart[d] = run;
        for (int ww = 0; ww < RS_WARPS; ++ww)
        {
            const int cw = wc[ww][d];
            wc[ww][d] = run;
            run += cw;
        }
    }
    __syncthreads();
    // ranks in input order, into shared memory in digit order
    for (int r = 0; r < RS_PER_WARP; r += 32)
    {
        const long long i = wbase + r + lane;
        const bool valid = i < n;
        const unsigned key = valid ? keys[i] : 0u;
        const int d = valid ? (int)((key >> shift) & 255u) : 256 + lane; // invalid lanes: unique groups
        const unsigned grp = __match_any_sync(FULL_MASK, d);
        int pos = 0;
        if (valid) pos = wc[w][d] + __popc(grp & lanemask_lt());
        __syncwarp();
        if (valid)
        {
            sk[pos] = key;
            sv[pos] = vals[i];
            if (lane == 31 - __clz(grp)) wc[w][d] += __popc(grp);
        }
        __syncwarp();
    }
    __syncthreads();
    // out in digit order: pair j of the reordered tile goes to its digit's global
    // start plus its place inside the digit's run
    for (int j = threadIdx.x; j < tn; j += RS_THREADS)
    {
        const unsigned key = sk[j];
        const int d = (int)((key >> shift) & 255u);
        const long long pos = (long long)offs[(long long)d * ntiles + blockIdx.x] + (j - tstart[d]);
        okeys[pos] = key;
        ovals[pos] = sv[j];
    }
}

} // namespace

void radix_sort_pairs(unsigned *keys, uint2 *vals, unsigned *keys_tmp, uint2 *vals_tmp, int n, int key_bits,
                      cudaStream_t s)
{
    if (n <= 1) return;
    {
        // the kernel attribute is per device: set it once for each device the
        // process sorts on (plans may be built from several host threads)
        static std::mutex mu;
        static std::unordered_set<int> done;
        int dev = 0;
        SDL_CUDA(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lk(mu);
        if (!done.count(dev))
        {
            SDL_CUDA(cudaFuncSetAttribute(k_rs_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)RS_SCATTER_SMEM));
            done.insert(dev);
        }
    }
    const int ntiles = (int)(((long long)n + RS_TILE - 1) / RS_TILE);
    if ((long long)ntiles * 256 > INT_MAX) fail(SDL_ERR_OVERFLOW, "radix sort: too many tiles");
    DevBuf<int> hist((size_t)ntiles * 256), offs((size_t)ntiles * 256 + 1);
    unsigned *ka = keys, *kb = keys_tmp;
    uint2 *va = vals, *vb = vals_tmp;
    const int passes = (key_bits + 7) / 8;
    for (int p = 0; p < passes; ++p)
    {
        const int shift = 8 * p;
        SDL_LAUNCH(k_rs_hist, ntiles, RS_THREADS, 0, s, ka, n, shift, ntiles, hist.get());
        exclusive_scan_i32_checked(hist.get(), offs.get(), ntiles * 256, s);
        SDL_LAUNCH(k_rs_scatter, ntiles, RS_THREADS, RS_SCATTER_SMEM, s, ka, va, n, shift, ntiles, offs.get(), kb,
                   vb);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (ka != keys)
    {
        SDL_CUDA(cudaMemcpyAsync(keys, ka, (size_t)n * sizeof(unsigned), cudaMemcpyDeviceToDevice, s));
        SDL_CUDA(cudaMemcpyAsync(vals, va, (size_t)n * sizeof(uint2), cudaMemcpyDeviceToDevice, s));
    }
    SDL_CUDA(cudaStreamSynchronize(s)); // hist / offs are freed on return
}

} // namespace sdl
