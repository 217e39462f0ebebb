// COO coalescing (and the matrix sums built on it): the plan sorts the triplets
// once, stably, by column and then by row, so they sit in (row, column, triplet)
// order; the first triplet of each distinct (row, column) opens an output, which
// gives the coalesced CSR structure and, in the same order, the triplet-to-output
// permutation. A value refill is then a gather in output order: one thread per
// output summing its triplets' values (times their factors, when given) from +0.0
// in ascending triplet order -- upstream's memset + accumulator order, bit for bit
// -- with the permutation read in order and the values gathered once each.
#include <algorithm>

#include "sdl_device.cuh"
#include "sdl_internal.h"

namespace sdl {

void radix_sort_pairs(unsigned *keys, uint2 *vals, unsigned *keys_tmp, uint2 *vals_tmp, int n, int key_bits,
                      cudaStream_t s);

namespace {

int grid_coal(long long n, int per_block)
{
    long long g = (n + per_block - 1) / per_block;
    return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 32));
}

// A thread per output, four outputs (one grid stride apart) at a time: the first
// triplet of each is fetched before any is summed, so four dependent chains (start
// -> position -> value) are in flight together; further triplets of an output (the
// duplicates) follow in ascending order. Each output is summed from +0.0 in
// ascending triplet order.
constexpr int COAL_ILP = 4;
__global__ void k_coal_fill(const int *__restrict__ ostart, const int *__restrict__ perm, const double *__restrict__ x,
                            const double *__restrict__ f, int nout, double *__restrict__ C)
{
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long base = blockIdx.x * (long long)blockDim.x + threadIdx.x; base < nout; base += step * COAL_ILP)
    {
        int q0[COAL_ILP], q1[COAL_ILP];
#pragma unroll
        for (int j = 0; j < COAL_ILP; ++j)
        {
            const long long o = base + j * step;
            q0[j] = q1[j] = 0;
            if (o < nout)
            {
                q0[j] = __ldcs(ostart + o);
                q1[j] = __ldcs(ostart + o + 1);
            }
        }
        int t[COAL_ILP];
#pragma unroll
        for (int j = 0; j < COAL_ILP; ++j) t[j] = q0[j] < q1[j] ? __ldcs(perm + q0[j]) : -1;
        double v[COAL_ILP];
#pragma unroll
        for (int j = 0; j < COAL_ILP; ++j)
            v[j] = t[j] < 0 ? 0.0 : (f ? __dmul_rn(f[t[j]], x[t[j]]) : x[t[j]]);
#pragma unroll
        for (int j = 0; j < COAL_ILP; ++j)
        {
            const long long o = base + j * step;
            if (o >= nout) continue;
            double acc = __dadd_rn(0.0, v[j]);
            for (int q = q0[j] + 1; q < q1[j]; ++q)
            {
                const int tq = __ldcs(perm + q);
                acc = __dadd_rn(acc, f ? __dmul_rn(f[tq], x[tq]) : x[tq]);
            }
            __stcs(C + o, acc);
        }
    }
}

// Structure and refill plan of a coalescing in one sort: the triplets are stably
// radix-sorted by column, then by row, so they end up in (row, column, triplet)
// order; the first triplet of every distinct (row, column) opens an output, in
// CSR order; k_coal_fill refills from it.
__global__ void k_cs_init(const int *__restrict__ rows, const int *__restrict__ cols, int n,
                          unsigned *__restrict__ keys, uint2 *__restrict__ vals)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    {
        keys[t] = (unsigned)cols[t];
        vals[t] = make_uint2((unsigned)t, (unsigned)rows[t]);
    }
}

// Column-sorted {column | triplet, row} -> row keys with {triplet, column}.
__global__ void k_cs_rekey(const unsigned *__restrict__ keys1, const uint2 *__restrict__ vals1, int n,
                           unsigned *__restrict__ keys2, uint2 *__restrict__ vals2)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    {
        const uint2 v = vals1[q];
        keys2[q] = v.y;
        vals2[q] = make_uint2(v.x, keys1[q]);
    }
}

__global__ void k_cs_flags(const unsigned *__restrict__ row, const uint2 *__restrict__ vals, int n, int *__restrict__ flag)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        flag[q] = (q == 0 || row[q] != row[q - 1] || vals[q].y != vals[q - 1].y) ? 1 : 0;
}

__global__ void k_cs_emit(const unsigned *__restrict__ row, const uint2 *__restrict__ vals, const int *__restrict__ flag,
                          const int *__restrict__ oid, int n, int *__restrict__ perm, int *__restrict__ ostart,
                          int *__restrict__ Ci, int *__restrict__ rowcnt)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    {
        perm[q] = (int)vals[q].x;
        if (flag[q])
        {
            const int o = oid[q];
            ostart[o] = (int)q;
            Ci[o] = (int)vals[q].y;
            atomicAdd(&rowcnt[row[q]], 1);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) ostart[oid[n]] = n;
}

} // namespace

int coalesce_sorted_build(const int *rows, const int *cols, int n, int m, int ncols, DevBuf<int> &Cp, DevBuf<int> &Ci,
                          DevBuf<int> &perm, DevBuf<int> &ostart, cudaStream_t s)
{
    Cp.reset((size_t)m + 1);
    perm.reset((size_t)std::max(1, n));
    if (n == 0)
    {
        SDL_CUDA(cudaMemsetAsync(Cp.get(), 0, Cp.bytes(), s));
        Ci.reset(1);
        ostart.reset(1);
        SDL_CUDA(cudaMemsetAsync(ostart.get(), 0, sizeof(int), s));
        SDL_CUDA(cudaStreamSynchronize(s));
        return 0;
    }
    auto bits_of = [](int v) {
        int b = 1;
        while (b < 31 && ((long long)1 << b) < (long long)v) ++b;
        return b;
    };
    DevBuf<unsigned> ka((size_t)n), kb((size_t)n);
    DevBuf<uint2> va((size_t)n), vb((size_t)n);
    const int g = grid_coal(n, 256);
    SDL_LAUNCH(k_cs_init, g, 256, 0, s, rows, cols, n, ka.get(), va.get());
    radix_sort_pairs(ka.get(), va.get(), kb.get(), vb.get(), n, bits_of(ncols), s);
    SDL_LAUNCH(k_cs_rekey, g, 256, 0, s, ka.get(), va.get(), n, kb.get(), vb.get());
    radix_sort_pairs(kb.get(), vb.get(), ka.get(), va.get(), n, bits_of(m), s);
    DevBuf<int> flag((size_t)n), oid((size_t)n + 1);
    SDL_LAUNCH(k_cs_flags, g, 256, 0, s, kb.get(), vb.get(), n, flag.get());
    const int nout = exclusive_scan_i32_checked(flag.get(), oid.get(), n, s);
    Ci.reset((size_t)std::max(1, nout));
    ostart.reset((size_t)nout + 1);
    DevBuf<int> rowcnt((size_t)m + 1);
    SDL_CUDA(cudaMemsetAsync(rowcnt.get(), 0, rowcnt.bytes(), s));
    SDL_LAUNCH(k_cs_emit, g, 256, 0, s, kb.get(), vb.get(), flag.get(), oid.get(), n, perm.get(), ostart.get(),
               Ci.get(), rowcnt.get());
    const int total = exclusive_scan_i32_checked(rowcnt.get(), Cp.get(), m, s);
    if (total != nout) fail(SDL_ERR_INTERNAL, "coalesce plan: row counts disagree with the outputs");
    SDL_CUDA(cudaStreamSynchronize(s));
    return nout;
}



void coalesce_order_fill(const int *ostart, const int *perm, const double *x, const double *f, int nout, double *C,
                         cudaStream_t s)
{
    if (nout <= 0) return;
    SDL_LAUNCH(k_coal_fill, grid_coal(nout, 256), 256, 0, s, ostart, perm, x, f, nout, C);
}

// ------------------------------------------------------------------ bucketed refill
// For large inputs the one-pass refill gathers every triplet value at random from
// an array far larger than L2, so DRAM moves whole sectors for 8 useful bytes. The
// bucketed refill splits it into two streaming-friendly passes:
//  1. the values are read in input order, a chunk of CO_CHUNK triplets per CTA,
//     and written into output-range buckets (bucket b holds the triplets of outputs
//     [b * span, (b + 1) * span)), each chunk's triplets of one bucket as one
//     contiguous run, after the chunk's runs of that bucket from earlier chunks --
//     so every bucket holds its triplets in input order;
//  2. the one-pass refill, reading from the buckets instead of the input: an
//     output's triplets now lie in one bucket of a few MB, which stays in L2 while
//     the outputs of that range are summed.
// The sums are the same sums in the same order (ascending triplet per output,
// from +0.0), so the result is bit-identical to the one-pass refill.
namespace {
// Outputs per bucket (a power of two; more when the buckets would exceed
// CO_MAX_BUCKETS): the buckets being summed in pass 2 stay in L2, and a chunk's
// run per bucket is chunk / buckets values long.
#ifndef SDL_COALESCE_SPAN_LOG2
#define SDL_COALESCE_SPAN_LOG2 20
#endif
constexpr int COALESCE_SPAN_LOG2 = SDL_COALESCE_SPAN_LOG2;
// CTAs per SM of the gather pass over the buckets
#ifndef SDL_COALESCE_FILL_CTAS
#define SDL_COALESCE_FILL_CTAS 8
#endif
constexpr int COALESCE_FILL_CTAS = SDL_COALESCE_FILL_CTAS;
constexpr int CO_CHUNK = 4096;
constexpr int CO_THREADS = 256;
constexpr int CO_MAX_BUCKETS = 512;

// Output index of every triplet (inverse of the output-order permutation).
__global__ void k_cb_owner(const int *__restrict__ ostart, const int *__restrict__ perm, int nout,
                           int *__restrict__ owner)
{
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < nout; o += (long long)gridDim.x * blockDim.x)
        for (int q = ostart[o]; q < ostart[o + 1]; ++q) owner[perm[q]] = (int)o;
}

// Per chunk: its triplets stably ordered by bucket (bitonic sort of bucket << 12 |
// index in shared memory), the order (lperm), each bucket's first position in it
// (cbound, nb + 1 per chunk), each bucket's count (count, bucket-major for the
// scan over chunks) and every triplet's rank inside its bucket's run (rank).
__global__ void __launch_bounds__(CO_THREADS) k_cb_chunks(const int *__restrict__ owner, int n, int span, int nb,
                                                         unsigned short *__restrict__ lperm, int *__restrict__ cbound,
                                                         int *__restrict__ count, int nchunks,
                                                         unsigned short *__restrict__ rank)
{
    __shared__ unsigned key[CO_CHUNK];
    __shared__ int bstart[CO_MAX_BUCKETS + 1];
    const int c = blockIdx.x;
    const long long t0 = (long long)c * CO_CHUNK;
    const int cnt = (int)(n - t0 < CO_CHUNK ? n - t0 : CO_CHUNK);
    for (int i = threadIdx.x; i < CO_CHUNK; i += CO_THREADS)
        key[i] = i < cnt ? ((unsigned)(owner[t0 + i] / span) << 12) | (unsigned)i : 0xffffffffu;
    for (int b = threadIdx.x; b <= nb; b += CO_THREADS) bstart[b] = cnt;
    __syncthreads();
    for (int k = 2; k <= CO_CHUNK; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            for (int i = threadIdx.x; i < CO_CHUNK; i += CO_THREADS)
            {
                const int l = i ^ j;
                if (l > i)
                {
                    const unsigned a = key[i], b = key[l];
                    if (((i & k) == 0) == (a > b))
                    {
                        key[i] = b;
                        key[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    // first position of every bucket present in the chunk; absent buckets take the
    // start of the next present one (filled backwards below)
    for (int i = threadIdx.x; i < cnt; i += CO_THREADS)
    {
        const int b = (int)(key[i] >> 12);
        if (i == 0 || (int)(key[i - 1] >> 12) != b) bstart[b] = i;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (int b = nb - 1; b >= 0; --b) bstart[b] = min(bstart[b], bstart[b + 1]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < cnt; i += CO_THREADS)
    {
        const int b = (int)(key[i] >> 12), li = (int)(key[i] & 0xfffu);
        lperm[t0 + i] = (unsigned short)li;
        rank[t0 + li] = (unsigned short)(i - bstart[b]);
    }
    for (int b = threadIdx.x; b <= nb; b += CO_THREADS)
    {
        cbound[(long long)c * (nb + 1) + b] = bstart[b];
        if (b < nb) count[(long long)b * nchunks + c] = bstart[b + 1] - bstart[b];
    }
}

// Bucket position of the triplet in every output-order slot.
__global__ void k_cb_perm2(const int *__restrict__ perm, const int *__restrict__ owner,
                           const unsigned short *__restrict__ rank, const long long *__restrict__ dst, int n, int span,
                           int nchunks, int *__restrict__ perm2)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    {
        const int t = perm[q];
        const int b = owner[t] / span, c = t / CO_CHUNK;
        perm2[q] = (int)(dst[(long long)b * nchunks + c] + rank[t]);
    }
}

// Pass 1: a CTA per chunk; the chunk's values (times their factors) are staged in
// shared memory, then every warp writes the runs of its share of the buckets.
__global__ void __launch_bounds__(CO_THREADS) k_cb_scatter(const double *__restrict__ x, const double *__restrict__ f,
                                                          int n, int nb, const unsigned short *__restrict__ lperm,
                                                          const int *__restrict__ cbound,
                                                          const long long *__restrict__ dstc,
                                                          double *__restrict__ buf)
{
    __shared__ double xs[CO_CHUNK];
    __shared__ int bs[CO_MAX_BUCKETS + 1];
    __shared__ long long ds[CO_MAX_BUCKETS];
    __shared__ unsigned short lp[CO_CHUNK];
    const int c = blockIdx.x;
    const long long t0 = (long long)c * CO_CHUNK;
    const int cnt = (int)(n - t0 < CO_CHUNK ? n - t0 : CO_CHUNK);
    for (int i = threadIdx.x; i < cnt; i += CO_THREADS)
    {
        xs[i] = f ? __dmul_rn(__ldcs(f + t0 + i), __ldcs(x + t0 + i)) : __ldcs(x + t0 + i);
        lp[i] = __ldcs(lperm + t0 + i);
    }
    for (int b = threadIdx.x; b <= nb; b += CO_THREADS) bs[b] = __ldcs(cbound + (long long)c * (nb + 1) + b);
    for (int b = threadIdx.x; b < nb; b += CO_THREADS) ds[b] = __ldcs(dstc + (long long)c * nb + b);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b = warp; b < nb; b += CO_THREADS / 32)
    {
        const int i0 = bs[b], i1 = bs[b + 1];
        if (i0 == i1) continue;
        double *out = buf + ds[b];
        for (int i = i0 + lane; i < i1; i += 32) out[i - i0] = xs[lp[i]];
    }
}

// Chunk-major copy of the bucket-major run offsets (what a chunk's CTA reads).
__global__ void k_cb_transpose_dst(const long long *__restrict__ dst, int nb, int nchunks, long long *__restrict__ dstc)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < (long long)nb * nchunks;
         k += (long long)gridDim.x * blockDim.x)
    {
        const long long b = k / nchunks, c = k - b * nchunks;
        dstc[c * nb + b] = dst[k];
    }
}
} // namespace

void coalesce_bucket_build(const int *ostart, const int *perm, int n, int nout, CoalesceBuckets &B, cudaStream_t s)
{
    B = CoalesceBuckets{};
    if (n < COALESCE_BUCKET_MIN || nout <= 0) return;
    Runtime &rt = runtime();
    int span = 1 << COALESCE_SPAN_LOG2;
    while ((long long)(nout + span - 1) / span > CO_MAX_BUCKETS) span <<= 1;
    const int nb = (nout + span - 1) / span;
    const int nchunks = (int)(((long long)n + CO_CHUNK - 1) / CO_CHUNK);
    DevBuf<int> owner((size_t)n);
    SDL_LAUNCH(k_cb_owner, grid_coal(nout, 256), 256, 0, s, ostart, perm, nout, owner.get());
    B.lperm.reset((size_t)n);
    B.cbound.reset((size_t)nchunks * (nb + 1));
    DevBuf<int> count((size_t)nb * nchunks);
    DevBuf<long long> count64((size_t)nb * nchunks);
    DevBuf<unsigned short> rank((size_t)n);
    SDL_LAUNCH(k_cb_chunks, nchunks, CO_THREADS, 0, s, owner.get(), n, span, nb, B.lperm.get(), B.cbound.get(),
               count.get(), nchunks, rank.get());
    // run offsets: bucket-major exclusive scan of the per-chunk counts
    widen_i32(count.get(), count64.get(), (long long)nb * nchunks, s);
    B.dst.reset((size_t)nb * nchunks + 1);
    const long long total = exclusive_scan_i64(count64.get(), B.dst.get(), (long long)nb * nchunks, s);
    if (total != n) fail(SDL_ERR_INTERNAL, "coalesce buckets: runs do not cover the triplets");
    B.perm2.reset((size_t)n);
    SDL_LAUNCH(k_cb_perm2, grid_coal(n, 256), 256, 0, s, perm, owner.get(), rank.get(), B.dst.get(), n, span,
               nchunks, B.perm2.get());
    // the scatter reads every chunk's run offsets in one piece
    DevBuf<long long> dstc((size_t)nb * nchunks);
    SDL_LAUNCH(k_cb_transpose_dst, grid_coal((long long)nb * nchunks, 256), 256, 0, s, B.dst.get(), nb, nchunks,
               dstc.get());
    B.dst = std::move(dstc);
    B.buf.reset((size_t)n);
    B.nb = nb;
    B.nchunks = nchunks;
    B.n = n;
    SDL_CUDA(cudaStreamSynchronize(s));
    (void)rt;
}

void coalesce_bucket_fill(const CoalesceBuckets &B, const int *ostart, const double *x, const double *f, int nout,
                          double *C, cudaStream_t s)
{
    SDL_LAUNCH(k_cb_scatter, B.nchunks, CO_THREADS, 0, s, x, f, B.n, B.nb, B.lperm.get(), B.cbound.get(), B.dst.get(),
               B.buf.get());
    // few outputs in flight (SMs x COALESCE_FILL_CTAS x 256 threads x 4 outputs: a
    // bucket or two), so the buckets being summed stay in L2
    const int grid = (int)std::max<long long>(
        1, std::min<long long>(((long long)nout + 255) / 256, (long long)runtime().num_sms * COALESCE_FILL_CTAS));
    SDL_LAUNCH(k_coal_fill, grid, 256, 0, s, ostart, B.perm2.get(), B.buf.get(), nullptr, nout, C);
}

} // namespace sdl
