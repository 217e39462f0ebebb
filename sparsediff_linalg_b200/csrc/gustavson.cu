// Row-wise sparse x sparse product on the GPU: C = kron(I_blocks, L) diag(d) A.
//
// Follows upstream's Gustavson core (src/sparse/gustavson.c):
//   symbolic  gustavson.c:26-105  exact column set of every row of C, ascending;
//   numeric   gustavson.c:107-143 acc[j] += (L.x[ii] * d[k]) * A.x[jj], visiting the
//             L entries of a row in order and, for each, A's row k in order.
// The numeric kernels reproduce that order for every output entry exactly: the
// terms of a row are flattened in upstream's visiting order, processed in chunks,
// and two terms of one chunk that hit the same entry are applied one after the
// other in term order (warp: __match_any_sync ranks; CTA: a claim table). Products
// and sums use __dmul_rn / __dadd_rn, so nothing is contracted into an FMA (the
// upstream build has none either), and the result is bit-identical.
//
// Rows are binned by their term count ("ub", an upper bound of their nnz):
//   symbolic: warp + shared-memory bitonic sort (<= 32 / 128 / 512 terms),
//             CTA + shared-memory sort (<= 2048 / 8192), CTA + shared-memory
//             bitmap over column windows (larger rows; the bitmap yields the
//             columns already sorted);
//   numeric:  row tiles (rows of <= TILE_T terms, grouped into CTA-sized tiles,
//             with an output-major schedule built once per pattern), CTA + shared
//             accumulator (<= 8192 output entries), CTA + accumulator in C.x itself
//             with a global column->position map (larger rows).
#include <algorithm>
#include <map>
#include <mutex>
#include <chrono>
#include <cstddef>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "sdl_device.cuh"
#include "sdl_internal.h"
#include "sdl_mlp.h"

namespace sdl {

void segment_sort_u64(unsigned long long *d_keys, const int *d_off, int nseg, int nkeys,
                      cudaStream_t s);
void radix_sort_pairs(unsigned *keys, uint2 *vals, unsigned *keys_tmp, uint2 *vals_tmp, int n, int key_bits,
                      cudaStream_t s);

namespace {

struct SymArgs
{
    const int *Lp, *Li;
    int L_m, n_L, n;
    const int *Ap, *Ai;
    const long long *ub_off; // offset of each row's column scratch
    int *tmp;
    int *row_nnz;
    const long long *cap;    // learned capacity of each row's scratch (null: its term count)
    unsigned char *overflow; // set to 1 for a row whose columns did not fit its capacity
};

__device__ __forceinline__ long long sym_cap(const SymArgs &a, int row)
{
    return a.cap ? a.cap[row] : 0x7fffffffffffffffLL;
}

struct NumArgs
{
    const int *Lp, *Li, *L_map;
    int L_m, n_L;
    const double *Lx, *d;
    const int *Ap, *Ai;
    const double *Ax;
    const int *Cp, *Ci;
    double *Cx;
    int *err;
    int L_nnz;       // entries of L (schedule build: entry index b * L_nnz + ii)
    int value_order; // entry values kept in L's value order (L_map a permutation)
};

// ------------------------------------------------------------ row statistics
__global__ void k_row_terms(const int *__restrict__ Lp, const int *__restrict__ Li, int L_m,
                            int n_L, int m_out, const int *__restrict__ Ap,
                            long long *__restrict__ ub)
{
    const int lane = lane_id(), wpb = blockDim.x >> 5;
    for (long long row = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); row < m_out;
         row += (long long)gridDim.x * wpb)
    {
        int b = (int)(row / L_m), r = (int)(row - (long long)b * L_m);
        long long sum = 0;
        for (int ii = Lp[r] + lane; ii < Lp[r + 1]; ii += 32)
        {
            int k = Li[ii] + b * n_L;
            sum += Ap[k + 1] - Ap[k];
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) sum += __shfl_xor_sync(FULL_MASK, sum, o);
        if (lane == 0) ub[row] = sum;
    }
}

// ------------------------------------------------------------ binning
__global__ void k_bin_count(const unsigned char *__restrict__ cls, int n, int nbins,
                            int *__restrict__ counts)
{
    __shared__ int sh[16];
    if (threadIdx.x < 16) sh[threadIdx.x] = 0;
    __syncthreads();
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
    {
        int c = cls[k];
        if (c < nbins) atomicAdd(&sh[c], 1);
    }
    __syncthreads();
    if (threadIdx.x < nbins && sh[threadIdx.x]) atomicAdd(&counts[threadIdx.x], sh[threadIdx.x]);
}

__global__ void k_bin_scatter(const unsigned char *__restrict__ cls, int n, int nbins,
                              int *__restrict__ cursor, int *__restrict__ lists)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
    {
        int c = cls[k];
        if (c < nbins) lists[atomicAdd(&cursor[c], 1)] = (int)k;
    }
}

__global__ void k_sym_classify(const long long *__restrict__ ub, int m_out, int warp_max,
                               unsigned char *__restrict__ cls)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
    {
        long long u = ub[r];
        int c = u == 0 ? 255 : u <= 32 ? SYM_W32 : u <= 128 ? SYM_W128 : u <= 512 ? SYM_W512
                         : u <= 2048 ? SYM_C2K : u <= 8192 ? SYM_C8K : SYM_BITMAP;
        if (u > warp_max && c <= SYM_W512) c = SYM_C2K; // rows above the warp threshold go to CTAs
        cls[r] = (unsigned char)c;
    }
}

// keep the class of the rows flagged in `mask`, drop the others
__global__ void k_mask_classes(const unsigned char *__restrict__ mask, int m_out, unsigned char *__restrict__ cls)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
        if (!mask[r]) cls[r] = 255;
}

// Numeric class and tile weight of every output row. A tile row costs its terms,
// one unit per 16 of its L entries and TILE_T / TILE_THREADS units; a larger row
// costs TILE_T, so it always ends its tile. Rows with more than TILE_MAX_LROW L
// entries never join a tile (the 18-bit entry index of a term word stays in range).
constexpr int TILE_MAX_LROW = 131072;
__global__ void k_num_classify(const long long *__restrict__ ub, const int *__restrict__ Cp,
                               const int *__restrict__ Lp, int L_m, int m_out, int tile_max,
                               unsigned char *__restrict__ cls, long long *__restrict__ weight)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
    {
        const long long u = ub[r];
        const int nr = Cp[r + 1] - Cp[r];
        const int rr = (int)(r % L_m);
        const int lenL = Lp[rr + 1] - Lp[rr];
        int c;
        if (u == 0)
            c = 255;
        else if (u <= tile_max && lenL <= TILE_MAX_LROW)
            c = NUM_TILE;
        else if (nr <= 2048)
            c = NUM_C2K;
        else if (nr <= 8192)
            c = NUM_C8K;
        else
            c = NUM_GMEM;
        cls[r] = (unsigned char)c;
        const long long lw = (lenL + 15) / 16 + TILE_T / TILE_THREADS;
        weight[r] = c == NUM_TILE ? u + lw : (c == 255 ? lw : TILE_T);
    }
}

// tile index of every row = floor(exclusive weight prefix / TILE_T); flag rows that
// start a tile
__global__ void k_tile_flags(const long long *__restrict__ wpref, int m_out, int budget, int *__restrict__ flag)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
        flag[r] = (r == 0 || wpref[r] / budget != wpref[r - 1] / budget) ? 1 : 0;
}

__global__ void k_tile_starts(const int *__restrict__ flag, const int *__restrict__ tile_of, int m_out,
                              int *__restrict__ tile_start)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
        if (flag[r]) tile_start[tile_of[r]] = (int)r;
}

// ------------------------------------------------------------ symbolic kernels
// Gather the column indices of all terms of `row` into buf (warp version).
__device__ __forceinline__ int warp_gather_terms(const SymArgs &a, int row, int *buf)
{
    const int lane = lane_id();
    int b = row / a.L_m, r = row - b * a.L_m;
    int ls = a.Lp[r], le = a.Lp[r + 1];
    int cnt = 0;
    for (int c = ls; c < le; c += 32)
    {
        int ii = c + lane, s = 0, len = 0;
        if (ii < le)
        {
            int k = a.Li[ii] + b * a.n_L;
            s = a.Ap[k];
            len = a.Ap[k + 1] - s;
        }
        int incl = warp_incl_scan(len);
        int total = __shfl_sync(FULL_MASK, incl, 31);
        for (int base = 0; base < total; base += 32)
        {
            int u = base + lane;
            int e = warp_entry_of(incl, u);
            int se = __shfl_sync(FULL_MASK, s, e);
            int ie = __shfl_sync(FULL_MASK, incl, e);
            int lne = __shfl_sync(FULL_MASK, len, e);
            if (u < total) buf[cnt + u] = a.Ai[se + u - (ie - lne)];
        }
        cnt += total;
    }
    return cnt;
}

template <int CAP>
__global__ void k_sym_warp(const int *__restrict__ rows, int count, SymArgs a)
{
    extern __shared__ int smi[];
    const int lane = lane_id(), wpb = blockDim.x >> 5;
    int *buf = smi + (threadIdx.x >> 5) * CAP;
    for (long long it = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); it < count;
         it += (long long)gridDim.x * wpb)
    {
        int row = rows[it];
        int cnt = warp_gather_terms(a, row, buf);
        int P = next_pow2(cnt);
        for (int q = cnt + lane; q < P; q += 32) buf[q] = INT_MAX;
        __syncwarp();
        warp_bitonic_sort(buf, P);
        long long off = a.ub_off[row], cap = sym_cap(a, row);
        int nn = 0;
        for (int base = 0; base < cnt; base += 32)
        {
            int q = base + lane;
            bool flag = q < cnt && (q == 0 || buf[q] != buf[q - 1]);
            unsigned bal = __ballot_sync(FULL_MASK, flag);
            long long at = nn + __popc(bal & lanemask_lt());
            if (flag && at < cap) a.tmp[off + at] = buf[q];
            nn += __popc(bal);
        }
        if (lane == 0)
        {
            a.row_nnz[row] = nn;
            if (nn > cap) a.overflow[row] = 1;
        }
        __syncwarp();
    }
}

// Chunked term enumeration for one CTA: loads up to blockDim L entries of row
// (b, r) starting at c into shared arrays and returns the number of terms.
struct CtaChunk
{
    int *incl, *s, *len;
    double *v;
    int *scr;
};

__device__ __forceinline__ int cta_load_chunk(const int *Li, const int *Ap, int b, int n_L,
                                              int c, int le, CtaChunk ch, const double *Lx,
                                              const int *L_map, const double *d, bool want_v)
{
    int ii = c + threadIdx.x, s = 0, len = 0;
    double v = 0.0;
    if (ii < le)
    {
        int k = Li[ii] + b * n_L;
        s = Ap[k];
        len = Ap[k + 1] - s;
        if (want_v)
        {
            double lx = Lx ? Lx[L_map ? L_map[ii] : ii] : 1.0;
            v = d ? __dmul_rn(lx, d[k]) : lx;
        }
    }
    int incl = block_incl_scan_int(len, ch.scr); // ends with a barrier
    ch.incl[threadIdx.x] = incl;
    ch.s[threadIdx.x] = s;
    ch.len[threadIdx.x] = len;
    if (want_v) ch.v[threadIdx.x] = v;
    __syncthreads();
    return ch.incl[blockDim.x - 1];
}

// entry of term u: first e in [0, nent) with incl[e] > u
__device__ __forceinline__ int cta_entry_of(const int *incl, int nent, int u)
{
    int lo = 0, hi = nent;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (incl[mid] <= u)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

template <int CAP>
__global__ void k_sym_cta(const int *__restrict__ rows, int count, SymArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    int *buf = (int *)smraw;
    CtaChunk ch;
    ch.incl = buf + CAP;
    ch.s = ch.incl + blockDim.x;
    ch.len = ch.s + blockDim.x;
    ch.scr = ch.len + blockDim.x;
    ch.v = nullptr;
    __shared__ int tot_sh;
    for (int it = blockIdx.x; it < count; it += gridDim.x)
    {
        int row = rows[it];
        int b = row / a.L_m, r = row - b * a.L_m;
        int ls = a.Lp[r], le = a.Lp[r + 1];
        int cnt = 0;
        for (int c = ls; c < le; c += blockDim.x)
        {
            int total = cta_load_chunk(a.Li, a.Ap, b, a.n_L, c, le, ch, nullptr, nullptr,
                                       nullptr, false);
            int nent = min((int)blockDim.x, le - c);
            for (int u = threadIdx.x; u < total; u += blockDim.x)
            {
                int e = cta_entry_of(ch.incl, nent, u);
                buf[cnt + u] = a.Ai[ch.s[e] + u - (ch.incl[e] - ch.len[e])];
            }
            cnt += total;
            __syncthreads();
        }
        int P = next_pow2(cnt);
        for (int q = cnt + threadIdx.x; q < P; q += blockDim.x) buf[q] = INT_MAX;
        __syncthreads();
        block_bitonic_sort(buf, P);
        long long off = a.ub_off[row], cap = sym_cap(a, row);
        int nn = 0;
        for (int base = 0; base < cnt; base += blockDim.x)
        {
            int q = base + threadIdx.x;
            int flag = (q < cnt && (q == 0 || buf[q] != buf[q - 1])) ? 1 : 0;
            int incl = block_incl_scan_int(flag, ch.scr);
            if (flag && nn + incl - 1 < cap) a.tmp[off + nn + incl - 1] = buf[q];
            if (threadIdx.x == blockDim.x - 1) tot_sh = incl;
            __syncthreads();
            nn += tot_sh;
            __syncthreads();
        }
        if (threadIdx.x == 0)
        {
            a.row_nnz[row] = nn;
            if (nn > cap) a.overflow[row] = 1;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ one-shot rows
// Symbolic and numeric in one pass, for a pattern met for the first time: every
// term of the row is gathered as a key (column << 32 | term index) with its value
// (L.x * d[k]) * A.x, the keys are sorted, and each run of equal columns -- its
// terms in visiting order, since the term index breaks ties -- is summed from +0.0
// in that order: the column and the value of one output of C, exactly the sum the
// numeric pass computes. Outputs go to the row's slot range [off, off + cap);
// a row with more outputs than its capacity is flagged and redone.
struct OneShotArgs
{
    const int *Lp, *Li, *L_map;
    int L_m, n_L;
    const double *Lx, *d;
    const int *Ap, *Ai;
    const double *Ax;
    const long long *off; // first slot of each row
    const long long *cap; // slots of each row (null: unbounded)
    int *col;
    double *val;
    int *row_nnz;
    unsigned char *overflow;
};

__device__ __forceinline__ double oneshot_entry_value(const OneShotArgs &a, int ii, int k)
{
    const double lx = a.Lx ? a.Lx[a.L_map ? a.L_map[ii] : ii] : 1.0;
    return a.d ? __dmul_rn(lx, a.d[k]) : lx;
}

// Sorted keys -> outputs: run q (first key of its column) sums its terms in order.
__device__ __forceinline__ double oneshot_run_sum(const unsigned long long *key, const double *val, int cnt, int q)
{
    const unsigned c = (unsigned)(key[q] >> 32);
    double acc = 0.0;
    for (int r = q; r < cnt && (unsigned)(key[r] >> 32) == c; ++r) acc = __dadd_rn(acc, val[(unsigned)key[r]]);
    return acc;
}

template <int CAP>
__global__ void k_oneshot_warp(const int *__restrict__ rows, int count, OneShotArgs a)
{
    extern __shared__ __align__(16) unsigned char osm[];
    const int lane = lane_id(), wpb = blockDim.x >> 5, w = threadIdx.x >> 5;
    unsigned long long *key = reinterpret_cast<unsigned long long *>(osm) + (size_t)w * 2 * CAP;
    double *val = reinterpret_cast<double *>(key + CAP);
    for (long long it = blockIdx.x * (long long)wpb + w; it < count; it += (long long)gridDim.x * wpb)
    {
        const int row = rows[it];
        const int b = row / a.L_m, r = row - b * a.L_m;
        const int ls = a.Lp[r], le = a.Lp[r + 1];
        int cnt = 0;
        for (int c = ls; c < le; c += 32)
        {
            const int ii = c + lane;
            int s = 0, len = 0;
            double v = 0.0;
            if (ii < le)
            {
                const int k = a.Li[ii] + b * a.n_L;
                s = a.Ap[k];
                len = a.Ap[k + 1] - s;
                v = oneshot_entry_value(a, ii, k);
            }
            const int incl = warp_incl_scan(len);
            const int total = __shfl_sync(FULL_MASK, incl, 31);
            for (int base = 0; base < total; base += 32)
            {
                const int u = base + lane;
                const int e = warp_entry_of(incl, u);
                const int se = __shfl_sync(FULL_MASK, s, e), ie = __shfl_sync(FULL_MASK, incl, e),
                          lne = __shfl_sync(FULL_MASK, len, e);
                const double ve = __shfl_sync(FULL_MASK, v, e);
                if (u < total)
                {
                    const int jj = se + u - (ie - lne);
                    key[cnt + u] = ((unsigned long long)(unsigned)a.Ai[jj] << 32) | (unsigned)(cnt + u);
                    val[cnt + u] = __dmul_rn(ve, a.Ax[jj]);
                }
            }
            cnt += total;
        }
        const int P = next_pow2(cnt);
        for (int q = cnt + lane; q < P; q += 32) key[q] = ~0ULL;
        __syncwarp();
        warp_bitonic_sort(key, P);
        const long long off = a.off[row], cap = a.cap ? a.cap[row] : 0x7fffffffffffffffLL;
        int nn = 0;
        for (int base = 0; base < cnt; base += 32)
        {
            const int q = base + lane;
            const bool flag = q < cnt && (q == 0 || (unsigned)(key[q] >> 32) != (unsigned)(key[q - 1] >> 32));
            const unsigned bal = __ballot_sync(FULL_MASK, flag);
            const long long at = nn + __popc(bal & lanemask_lt());
            if (flag && at < cap)
            {
                a.col[off + at] = (int)(key[q] >> 32);
                a.val[off + at] = oneshot_run_sum(key, val, cnt, q);
            }
            nn += __popc(bal);
        }
        if (lane == 0)
        {
            a.row_nnz[row] = nn;
            if (nn > cap) a.overflow[row] = 1;
        }
        __syncwarp();
    }
}

template <int CAP>
__global__ void k_oneshot_cta(const int *__restrict__ rows, int count, OneShotArgs a)
{
    extern __shared__ __align__(16) unsigned char osm[];
    unsigned long long *key = reinterpret_cast<unsigned long long *>(osm);
    double *val = reinterpret_cast<double *>(key + CAP);
    CtaChunk ch;
    ch.v = val + CAP;
    ch.incl = reinterpret_cast<int *>(ch.v + blockDim.x);
    ch.s = ch.incl + blockDim.x;
    ch.len = ch.s + blockDim.x;
    ch.scr = ch.len + blockDim.x;
    __shared__ int tot_sh;
    for (int it = blockIdx.x; it < count; it += gridDim.x)
    {
        const int row = rows[it];
        const int b = row / a.L_m, r = row - b * a.L_m;
        const int ls = a.Lp[r], le = a.Lp[r + 1];
        int cnt = 0;
        for (int c = ls; c < le; c += blockDim.x)
        {
            const int total = cta_load_chunk(a.Li, a.Ap, b, a.n_L, c, le, ch, a.Lx, a.L_map, a.d, true);
            const int nent = min((int)blockDim.x, le - c);
            for (int u = threadIdx.x; u < total; u += blockDim.x)
            {
                const int e = cta_entry_of(ch.incl, nent, u);
                const int jj = ch.s[e] + u - (ch.incl[e] - ch.len[e]);
                key[cnt + u] = ((unsigned long long)(unsigned)a.Ai[jj] << 32) | (unsigned)(cnt + u);
                val[cnt + u] = __dmul_rn(ch.v[e], a.Ax[jj]);
            }
            cnt += total;
            __syncthreads();
        }
        const int P = next_pow2(cnt);
        for (int q = cnt + threadIdx.x; q < P; q += blockDim.x) key[q] = ~0ULL;
        __syncthreads();
        block_bitonic_sort(key, P);
        const long long off = a.off[row], cap = a.cap ? a.cap[row] : 0x7fffffffffffffffLL;
        int nn = 0;
        for (int base = 0; base < cnt; base += blockDim.x)
        {
            const int q = base + threadIdx.x;
            const int flag =
                (q < cnt && (q == 0 || (unsigned)(key[q] >> 32) != (unsigned)(key[q - 1] >> 32))) ? 1 : 0;
            const int incl = block_incl_scan_int(flag, ch.scr);
            const long long at = nn + incl - 1;
            if (flag && at < cap)
            {
                a.col[off + at] = (int)(key[q] >> 32);
                a.val[off + at] = oneshot_run_sum(key, val, cnt, q);
            }
            if (threadIdx.x == blockDim.x - 1) tot_sh = incl;
            __syncthreads();
            nn += tot_sh;
            __syncthreads();
        }
        if (threadIdx.x == 0)
        {
            a.row_nnz[row] = nn;
            if (nn > cap) a.overflow[row] = 1;
        }
        __syncthreads();
    }
}

__global__ void k_mark_class(const unsigned char *__restrict__ cls, int m_out, int which,
                             unsigned char *__restrict__ out)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out; r += (long long)gridDim.x * blockDim.x)
        out[r] = cls[r] == which ? 1 : 0;
}

// Large rows: mark columns in a shared-memory bitmap, one column window at a time;
// reading the bitmap word by word yields the columns in ascending order.
// Rows taken in list order: from a shared counter when given (the list is then
// ordered by work, largest first), else every gridDim-th.
__global__ void k_sym_bitmap(const int *__restrict__ rows, int count, SymArgs a, int words, int *__restrict__ next_row)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned *bm = (unsigned *)smraw;
    CtaChunk ch;
    ch.incl = (int *)(bm + words);
    ch.s = ch.incl + blockDim.x;
    ch.len = ch.s + blockDim.x;
    ch.scr = ch.len + blockDim.x;
    ch.v = nullptr;
    __shared__ int tot_sh;
    __shared__ int it_sh;
    const int wbits = words * 32;
    for (int it = blockIdx.x;;)
    {
        if (next_row)
        {
            __syncthreads();
            if (threadIdx.x == 0) it_sh = atomicAdd(next_row, 1);
            __syncthreads();
            it = it_sh;
        }
        if (it >= count) break;
        int row = rows[it];
        int b = row / a.L_m, r = row - b * a.L_m;
        int ls = a.Lp[r], le = a.Lp[r + 1];
        long long off = a.ub_off[row], cap = sym_cap(a, row);
        int running = 0;
        for (long long ws = 0; ws < a.n; ws += wbits)
        {
            for (int q = threadIdx.x; q < words; q += blockDim.x) bm[q] = 0u;
            __syncthreads();
            for (int c = ls; c < le; c += blockDim.x)
            {
                int total = cta_load_chunk(a.Li, a.Ap, b, a.n_L, c, le, ch, nullptr, nullptr,
                                           nullptr, false);
                int nent = min((int)blockDim.x, le - c);
                for (int u = threadIdx.x; u < total; u += blockDim.x)
                {
                    int e = cta_entry_of(ch.incl, nent, u);
                    long long j = a.Ai[ch.s[e] + u - (ch.incl[e] - ch.len[e])] - ws;
                    if (j >= 0 && j < wbits) atomicOr(&bm[j >> 5], 1u << (j & 31));
                }
                __syncthreads();
            }
            int wpt = (words + blockDim.x - 1) / blockDim.x;
            int w0 = min(words, (int)threadIdx.x * wpt), w1 = min(words, w0 + wpt);
            int mine = 0;
            for (int q = w0; q < w1; ++q) mine += __popc(bm[q]);
            int incl = block_incl_scan_int(mine, ch.scr);
            long long pos = off + running + incl - mine;
            for (int q = w0; q < w1; ++q)
            {
                unsigned word = bm[q];
                while (word)
                {
                    int bit = __ffs(word) - 1;
                    if (pos - off < cap) a.tmp[pos] = (int)(ws + q * 32 + bit);
                    ++pos;
                    word &= word - 1;
                }
            }
            if (threadIdx.x == blockDim.x - 1) tot_sh = incl;
            __syncthreads();
            running += tot_sh;
            __syncthreads();
        }
        if (threadIdx.x == 0)
        {
            a.row_nnz[row] = running;
            if (running > cap) a.overflow[row] = 1;
        }
        __syncthreads();
        if (!next_row) it += gridDim.x;
    }
}

// Scratch span (work) of each listed row: off[row + 1] - off[row].
__global__ void k_row_spans(const int *__restrict__ rows, int n, const long long *__restrict__ off,
                            long long *__restrict__ out)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        out[q] = off[rows[q] + 1] - off[rows[q]];
}

// Compaction of per-row slot ranges into C: row r's Cp[r + 1] - Cp[r] outputs are
// copied from its slots (off0[r] in src0, or off1[r] in src1 for rows flagged in
// sel) to C.i (and C.x when value sources are given, except for rows flagged in
// late). The work is cut by outputs, not rows: CTA chunks of COMPACT_Q consecutive
// outputs (a skewed product's longest rows are shared out instead of landing on
// one CTA), each chunk's first row found beforehand (k_compact_chunks). A chunk's
// rows are staged COMPACT_R at a time (row offsets, slot offsets, flags) and its
// threads stride over the outputs, each finding its row by a search over the
// staged offsets, so rows of one or two outputs do not leave a warp idle.
constexpr int COMPACT_Q = 2048;
constexpr int COMPACT_R = 1024;

// first_row[c] = the row holding output c * COMPACT_Q: each non-empty row marks the
// chunk starts inside its range.
__global__ void k_compact_chunks(const int *__restrict__ Cp, int m_out, int *__restrict__ first_row)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
    {
        const int q0 = Cp[r], q1 = Cp[r + 1];
        for (long long c = ((long long)q0 + COMPACT_Q - 1) / COMPACT_Q; c * COMPACT_Q < q1; ++c)
            first_row[c] = (int)r;
    }
}

__global__ void __launch_bounds__(256) k_compact_rows(const int *__restrict__ Cp, int m_out,
                                                      const int *__restrict__ first_row,
                                                      const long long *__restrict__ off0,
                                                      const long long *__restrict__ off1,
                                                      const unsigned char *__restrict__ sel,
                                                      const unsigned char *__restrict__ late,
                                                      const int *__restrict__ src0c, const int *__restrict__ src1c,
                                                      const double *__restrict__ src0v,
                                                      const double *__restrict__ src1v, int *__restrict__ Ci,
                                                      double *__restrict__ Cx)
{
    __shared__ int cp[COMPACT_R + 1];
    __shared__ long long so[COMPACT_R];
    __shared__ unsigned char fl[COMPACT_R];
    const int total = Cp[m_out];
    for (long long c = blockIdx.x; c * COMPACT_Q < total; c += gridDim.x)
    {
        const int q0 = (int)(c * COMPACT_Q);
        const int q1 = (int)min((long long)total, c * COMPACT_Q + COMPACT_Q);
        for (int r0 = first_row[c];;)
        {
            const int nr = min(COMPACT_R, m_out - r0);
            __syncthreads(); // the previous rows' offsets are no longer read
            for (int i = threadIdx.x; i <= nr; i += blockDim.x) cp[i] = Cp[r0 + i];
            for (int i = threadIdx.x; i < nr; i += blockDim.x)
            {
                const bool alt = sel && sel[r0 + i];
                so[i] = alt ? off1[r0 + i] : off0[r0 + i];
                fl[i] = (unsigned char)((alt ? 1 : 0) | (late && late[r0 + i] ? 2 : 0));
            }
            __syncthreads();
            const int qa = max(q0, cp[0]), qb = min(q1, cp[nr]);
            constexpr int ILP = 4; // outputs per thread whose loads are in flight together
            for (int qq = qa + threadIdx.x; qq < qb; qq += ILP * blockDim.x)
            {
                int col[ILP], lo[ILP];
                double val[ILP];
#pragma unroll
                for (int k = 0; k < ILP; ++k)
                {
                    const int q = qq + k * blockDim.x;
                    lo[k] = -1;
                    if (q >= qb) continue;
                    int l = 0, hi = nr; // last row i with cp[i] <= q
                    while (hi - l > 1)
                    {
                        const int mid = (l + hi) >> 1;
                        if (cp[mid] <= q)
                            l = mid;
                        else
                            hi = mid;
                    }
                    lo[k] = l;
                    const long long at = so[l] + (q - cp[l]);
                    const bool alt = fl[l] & 1;
                    col[k] = alt ? src1c[at] : src0c[at];
                    if (Cx && !(fl[l] & 2)) val[k] = alt ? src1v[at] : src0v[at];
                }
#pragma unroll
                for (int k = 0; k < ILP; ++k)
                {
                    if (lo[k] < 0) continue;
                    const int q = qq + k * blockDim.x;
                    Ci[q] = col[k];
                    if (Cx && !(fl[lo[k]] & 2)) Cx[q] = val[k];
                }
            }
            if (cp[nr] >= q1 || r0 + nr >= m_out) break; // the chunk's last output is done
            r0 += nr;
        }
    }
}

// C.i (and C.x) of every row from its slot range (see k_compact_rows).
void compact_rows(const int *Cp, int m_out, int nnz, const long long *off0, const long long *off1,
                  const unsigned char *sel, const unsigned char *late, const int *src0c, const int *src1c,
                  const double *src0v, const double *src1v, int *Ci, double *Cx, cudaStream_t s)
{
    if (nnz <= 0 || m_out <= 0) return;
    Runtime &rt = runtime();
    const long long nchunks = ((long long)nnz + COMPACT_Q - 1) / COMPACT_Q;
    DevBuf<int> first_row((size_t)nchunks);
    const int cgrid = (int)std::max<long long>(1, std::min<long long>(((long long)m_out + 255) / 256,
                                                                      (long long)rt.num_sms * 8));
    SDL_LAUNCH(k_compact_chunks, cgrid, 256, 0, s, Cp, m_out, first_row.get());
    const int grid = (int)std::max<long long>(1, std::min<long long>(nchunks, (long long)rt.num_sms * 8));
    SDL_LAUNCH(k_compact_rows, grid, 256, 0, s, Cp, m_out, first_row.get(), off0, off1, sel, late, src0c, src1c,
               src0v, src1v, Ci, Cx);
    SDL_CUDA(cudaStreamSynchronize(s)); // first_row is released on return
}

// ------------------------------------------------------------ numeric kernels
// ------------------------------------------------------------ row tiles
// Outputs and terms of a tile are each below 2 * TILE_T.
constexpr int TILE_ACC = 2 * TILE_T;

// last index q in [0, n) with a[q] <= key (a non-decreasing, a[0] <= key)
__device__ __forceinline__ int last_le(const int *a, int n, int key)
{
    int lo = 0, hi = n;
    while (hi - lo > 1)
    {
        int mid = (lo + hi) >> 1;
        if (a[mid] <= key)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

struct BuildSmem
{
    int *cnt; // TILE_ACC: terms per output
    int *cur; // TILE_ACC: list cursor of an output with three or more terms, -1 otherwise
    int *row_cs, *row_nr, *row_ls, *row_b, *row_outoff, *row_eoff;
    int *e_incl, *e_s, *e_len, *e_row;
    int *scr;
    int *misc; // [1]: list outputs of a chunk, [2]: their terms
};
constexpr size_t build_smem_bytes()
{
    return ((size_t)2 * TILE_ACC + 4 * TILE_THREADS + 2 * (TILE_THREADS + 1) + 4 * TILE_THREADS + 32 + 4) * 4;
}

// Term enumeration of one tile, shared by both passes of the schedule build. The
// tile's L entries (every entry of its rows, in order: entry e is schedule entry
// vbase + e) are taken 256 at a time; fe(e, s, toff, len, slot) is called for each
// by its thread (s = A.p[k], toff = offset of its first term in the tile, len = its
// terms, slot = index of its value in V),
// then ft(valid, e, u, o) for every term in upstream's visiting order, 256
// consecutive terms per step (valid false for the idle threads of the last step,
// so every thread takes every barrier): u is the term's index in the tile, o its
// output inside the tile window.
template <class FE, class FT>
__device__ __forceinline__ int tile_terms(const NumArgs &a, const BuildSmem &t, int nrows, int total_raw, FE fe,
                                           FT ft)
{
    const int tid = threadIdx.x;
    int cursor = 0;
    for (int ec = 0; ec < total_raw; ec += TILE_THREADS)
    {
        const int e = ec + tid;
        int s = 0, len = 0, lrow = 0, slot = 0;
        if (e < total_raw)
        {
            lrow = last_le(t.row_eoff, nrows, e);
            const int ii = t.row_ls[lrow] + (e - t.row_eoff[lrow]);
            const int k = a.Li[ii] + t.row_b[lrow] * a.n_L;
            s = a.Ap[k];
            len = a.Ap[k + 1] - s;
            slot = t.row_b[lrow] * a.L_nnz + (a.value_order ? a.L_map[ii] : ii);
        }
        const int inc = block_incl_scan_int(len, t.scr);
        if (e < total_raw) fe(e, s, cursor + inc - len, len, slot);
        t.e_incl[tid] = inc;
        t.e_s[tid] = s;
        t.e_len[tid] = len;
        t.e_row[tid] = lrow;
        __syncthreads();
        const int total = t.e_incl[TILE_THREADS - 1];
        const int nent = min(TILE_THREADS, total_raw - ec);
        for (int base = 0; base < total; base += TILE_THREADS)
        {
            const int uu = base + tid;
            bool valid = uu < total;
            int el = 0, o = 0;
            if (valid)
            {
                el = cta_entry_of(t.e_incl, nent, uu);
                const int jj = t.e_s[el] + uu - (t.e_incl[el] - t.e_len[el]);
                const int j = a.Ai[jj];
                const int lr = t.e_row[el];
                const int w = t.row_nr[lr];
                const int *crow = a.Ci + t.row_cs[lr];
                const int pos = lower_bound_dev(crow, w, j);
                if (pos >= w || crow[pos] != j)
                {
                    atomicOr(a.err, 1);
                    valid = false;
                }
                o = t.row_outoff[lr] + pos;
            }
            ft(valid, ec + el, cursor + uu, o);
        }
        cursor += total;
        __syncthreads();
    }
    return cursor;
}

// kv[L_map[ii]] = Li[ii]; flags a map that is not a permutation of [0, n).
__global__ void k_value_rows(const int *__restrict__ L_map, const int *__restrict__ Li, int n,
                             int *__restrict__ kv, int *__restrict__ cnt, int *__restrict__ bad)
{
    for (long long ii = blockIdx.x * (long long)blockDim.x + threadIdx.x; ii < n;
         ii += (long long)gridDim.x * blockDim.x)
    {
        const int m = L_map[ii];
        if ((unsigned)m >= (unsigned)n || atomicAdd(&cnt[m], 1) != 0)
            atomicOr(bad, 1);
        else
            kv[m] = Li[ii];
    }
}

// Compiles the entry-major refill schedule of one tile (one CTA per tile, once per
// pattern): the ES records of the tile's entries, one word per term (see TileDesc), and the
// list section of the outputs with three or more terms: nlist + 1 headers
// (output | first list item << 12) and the term indices of each such output in
// upstream's visiting order.
// COUNT pass: the numbers of term words and list-section words of every tile.
// BUILD pass: writes everything at the offsets the scans of those numbers gave.
template <bool BUILD>
__global__ void __launch_bounds__(TILE_THREADS) k_tile_schedule(
    NumArgs a, const unsigned char *__restrict__ rcls, const int *__restrict__ tile_start,
    long long *__restrict__ tile_nterms, long long *__restrict__ tile_nx,
    const long long *__restrict__ word_begin, const long long *__restrict__ x_begin,
    TileDesc *__restrict__ tiles, unsigned *__restrict__ W, unsigned *__restrict__ X, int2 *__restrict__ ES)
{
    extern __shared__ __align__(16) int bsm[];
    BuildSmem t;
    t.cnt = bsm;
    t.cur = t.cnt + TILE_ACC;
    t.row_cs = t.cur + TILE_ACC;
    t.row_nr = t.row_cs + TILE_THREADS;
    t.row_ls = t.row_nr + TILE_THREADS;
    t.row_b = t.row_ls + TILE_THREADS;
    t.row_outoff = t.row_b + TILE_THREADS;
    t.row_eoff = t.row_outoff + TILE_THREADS + 1;
    t.e_incl = t.row_eoff + TILE_THREADS + 1;
    t.e_s = t.e_incl + TILE_THREADS;
    t.e_len = t.e_s + TILE_THREADS;
    t.e_row = t.e_len + TILE_THREADS;
    t.scr = t.e_row + TILE_THREADS;
    t.misc = t.scr + 32;
    const int tid = threadIdx.x;
    const int tile = blockIdx.x;
    const int r0 = tile_start[tile], nrows = tile_start[tile + 1] - r0;
    for (int q = tid; q < TILE_ACC; q += TILE_THREADS) t.cnt[q] = 0;
    int nr = 0, ne = 0;
    if (tid < nrows)
    {
        const int r = r0 + tid;
        const int b = r / a.L_m, rr = r - b * a.L_m;
        const int cs = a.Cp[r], ls = a.Lp[rr];
        const int c = rcls[r];
        if (c == NUM_TILE) nr = a.Cp[r + 1] - cs;
        // every L entry of the tile's rows up to a larger row (always the last row),
        // so that entry e of the tile is entry vbase + e
        if (c == NUM_TILE || c == 255) ne = a.Lp[rr + 1] - ls;
        t.row_cs[tid] = cs;
        t.row_nr[tid] = nr;
        t.row_ls[tid] = ls;
        t.row_b[tid] = b;
    }
    const int inr = block_incl_scan_int(nr, t.scr);
    const int ine = block_incl_scan_int(ne, t.scr);
    if (tid < nrows)
    {
        t.row_outoff[tid] = inr - nr;
        t.row_eoff[tid] = ine - ne;
    }
    if (tid == TILE_THREADS - 1)
    {
        t.row_outoff[nrows] = inr;
        t.row_eoff[nrows] = ine;
    }
    __syncthreads();
    const int total_out = t.row_outoff[nrows], total_raw = t.row_eoff[nrows];
    if (total_out > TILE_ACC)
    {
        if (tid == 0) atomicOr(a.err, 2);
        return; // cannot happen with the tile weights; the host reports it
    }
    const int b0 = r0 / a.L_m;
    const int vb = b0 * a.L_nnz + a.Lp[r0 - b0 * a.L_m];
    const long long wb = BUILD ? word_begin[tile] : 0, xb = BUILD ? x_begin[tile] : 0;

    // pass A: terms per output; the ES records of the entries
    const int nterms = tile_terms(
        a, t, nrows, total_raw,
        [&](int e, int s, int toff, int len, int slot) {
            if (BUILD && len > 0) ES[vb + e] = make_int2(s - toff, slot);
            if (e >= (1 << 18) && len > 0) atomicOr(a.err, 2);
        },
        [&](bool valid, int, int, int o) {
            if (valid) atomicAdd(&t.cnt[o], 1);
        });
    __syncthreads();
    // outputs with three or more terms: list index and first item
    int nlist = 0, nitems = 0;
    for (int oc = 0; oc < total_out; oc += TILE_THREADS)
    {
        const int o = oc + tid;
        const int c = o < total_out ? t.cnt[o] : 0;
        if (o < total_out && c == 0) atomicOr(a.err, 1); // every output has a term
        const int m = c >= 3 ? 1 : 0;
        const int im = block_incl_scan_int(m, t.scr);
        const int it = block_incl_scan_int(m ? c : 0, t.scr);
        if (o < total_out)
        {
            t.cur[o] = m ? nitems + it - c : -1;
            if (BUILD && m) X[xb + nlist + im - 1] = (unsigned)o | ((unsigned)(nitems + it - c) << 12);
        }
        if (tid == TILE_THREADS - 1)
        {
            t.misc[1] = im;
            t.misc[2] = it;
        }
        __syncthreads();
        nlist += t.misc[1];
        nitems += t.misc[2];
        __syncthreads();
    }
    if (!BUILD)
    {
        if (tid == 0)
        {
            tile_nterms[tile] = nterms;
            tile_nx[tile] = nlist ? nlist + 1 + nitems : 0;
        }
        return;
    }
    if (nlist && tid == 0) X[xb + nlist] = (unsigned)nitems << 12;
    // pass B: the term words; the term indices of list outputs into their lists in
    // visiting order (warps take turns, equal outputs inside a warp ranked by lane)
    unsigned *xl = X + xb + nlist + 1;
    const int warp = tid >> 5, lane = lane_id();
    tile_terms(
        a, t, nrows, total_raw, [&](int, int, int, int, int) {},
        [&](bool valid, int e, int u, int o) {
            bool listed = false;
            if (valid)
            {
                const int c = t.cnt[o];
                const unsigned kind = c == 1 ? TERM_ONE : (c == 2 ? TERM_PAIR : TERM_LIST);
                W[wb + u] = ((unsigned)e << 14) | (kind << 12) | (unsigned)o;
                listed = kind == TERM_LIST;
            }
            if (!nlist) return; // uniform over the block
            for (int w = 0; w < TILE_THREADS / 32; ++w)
            {
                if (warp == w)
                {
                    const int key = listed ? o : -(lane + 1);
                    const unsigned grp = __match_any_sync(FULL_MASK, key);
                    int slot = 0;
                    if (listed) slot = t.cur[o] + __popc(grp & lanemask_lt());
                    __syncwarp();
                    if (listed)
                    {
                        xl[slot] = (unsigned)u;
                        if (lane == 31 - __clz(grp)) t.cur[o] += __popc(grp);
                    }
                }
                __syncthreads();
            }
        });
    if (tid == 0)
    {
        TileDesc dsc;
        dsc.vbase = vb;
        dsc.word_begin = (int)wb;
        dsc.nterms = nterms;
        dsc.out_begin = t.row_cs[0];
        dsc.nout = total_out;
        dsc.x_begin = nlist ? (int)xb : -1;
        dsc.nlist = nlist;
        dsc.prod = 0;
        tiles[tile] = dsc;
    }
}

// Entry values of one refill: V[i] = L.x * d[k] (upstream's order of the two
// factors; L.x alone without d, 1.0 for a unit L) for every entry of
// kron(I_blocks, L). With S.kv (L_map a permutation) V is in L's value order,
// i = b * L_nnz + (index of the value), so L.x is read in order and kv gives the
// entry's row of A; otherwise i = b * L_nnz + ii. Each thread takes EV_ILP entries,
// spaced one grid apart, and issues all their loads before the first store.
#ifndef SDL_EV_ILP
#define SDL_EV_ILP 4
#endif
constexpr int EV_ILP = SDL_EV_ILP;
__device__ __forceinline__ void entry_values_run(const ProdSched &S, const ProdPtrs &P, long long first,
                                                 long long end, long long step)
{
    for (long long base = first; base < end; base += step * EV_ILP)
    {
        int xi[EV_ILP], k[EV_ILP];
#pragma unroll
        for (int j = 0; j < EV_ILP; ++j)
        {
            const long long i = base + j * step;
            xi[j] = -1;
            k[j] = 0;
            if (i < end)
            {
                const int b = S.blocks > 1 ? (int)(i / S.L_nnz) : 0;
                const int sl = (int)(i - (long long)b * S.L_nnz);
                if (P.d) k[j] = (S.kv ? S.kv[sl] : S.Li[sl]) + b * S.n_L;
                xi[j] = (!S.kv && S.L_map) ? S.L_map[sl] : sl; // index of the L value
            }
        }
        double lx[EV_ILP], dk[EV_ILP];
#pragma unroll
        for (int j = 0; j < EV_ILP; ++j)
        {
            lx[j] = 1.0;
            dk[j] = 1.0;
            if (xi[j] >= 0)
            {
                if (P.Lx) lx[j] = P.Lx[xi[j]];
                if (P.d) dk[j] = P.d[k[j]];
            }
        }
#pragma unroll
        for (int j = 0; j < EV_ILP; ++j)
        {
            const long long i = base + j * step;
            if (i < end) S.V[i] = P.d ? __dmul_rn(lx[j], dk[j]) : lx[j];
        }
    }
}

__global__ void __launch_bounds__(256) k_entry_values(ProdSched S, ProdPtrs P)
{
    // the refill launched after this grid may start its prologue now; it waits for
    // this grid's completion before it reads V
    asm volatile("griddepcontrol.launch_dependents;");
    const long long step = (long long)gridDim.x * blockDim.x;
    entry_values_run(S, P, blockIdx.x * (long long)blockDim.x + threadIdx.x, S.nV, step);
}

// Batched: one CTA per chunk of one product's entries.
__global__ void __launch_bounds__(256) k_entry_values_batched(const EntChunk *__restrict__ chunks,
                                                              const ProdPtrs *__restrict__ ptrs,
                                                              const ProdSched *__restrict__ scheds)
{
    const EntChunk c = chunks[blockIdx.x];
    const ProdSched S = scheds[c.prod];
    const ProdPtrs P = ptrs[c.prod];
    if (!P.Lx && !P.d) return; // unit product: the refill reads no V
    entry_values_run(S, P, c.begin + threadIdx.x, c.begin + c.count, blockDim.x);
}

#ifndef SDL_REFILL_MINB
#define SDL_REFILL_MINB 5
#endif
#ifndef SDL_REFILL_UNROLL
#define SDL_REFILL_UNROLL 4
#endif
constexpr int RUNROLL = SDL_REFILL_UNROLL; // terms per thread whose loads are in flight together
// Refill CTAs: 256 threads with windows of TILE_ACC outputs (every plan; the batched
// refill), or 128 threads with windows of TILE_ACC / 2 for plans whose tiles have at
// most that many outputs (tile budget and tile rows of at most TILE_T / 2 terms: a
// tile then holds fewer than TILE_T terms), twice as many CTAs per SM and a barrier
// among 4 warps instead of 8.
constexpr int REFILL_THREADS = 256;
constexpr int REFILL_THREADS_SMALL = 128;
template <int NT>
__host__ __device__ constexpr int win_of()
{
    return NT == REFILL_THREADS ? TILE_ACC : TILE_ACC / 2;
}
template <int NT>
__host__ __device__ constexpr int refill_minb()
{
    return NT == REFILL_THREADS ? SDL_REFILL_MINB : 2 * SDL_REFILL_MINB;
}


// Base pointers of the product a tile belongs to: kernel parameters for a single
// product, the batch's tables otherwise.
struct ProdBase
{
    const unsigned *W, *X;
    const double *Ax, *V;
    const int2 *ES;
    double *C;
    unsigned nV, nA; // both < 2^31
};
template <bool BATCHED>
__device__ __forceinline__ ProdBase prod_base(int prod, const ProdPtrs *__restrict__ ptrs,
                                              const ProdSched *__restrict__ scheds, const ProdPtrs &P1,
                                              const ProdSched &S1)
{
    ProdBase r;
    if (BATCHED)
    {
        r.Ax = ptrs[prod].Ax;
        r.C = ptrs[prod].Cx;
        r.W = scheds[prod].W;
        r.X = scheds[prod].X;
        // a unit product (no L values, no d) has every entry value 1.0: V is not read
        r.V = (ptrs[prod].Lx || ptrs[prod].d) ? scheds[prod].V : nullptr;
        r.ES = scheds[prod].ES;
        r.nV = (unsigned)scheds[prod].nV;
        r.nA = (unsigned)scheds[prod].nA;
    }
    else
    {
        r.Ax = P1.Ax;
        r.C = P1.Cx;
        r.W = S1.W;
        r.X = S1.X;
        r.V = (P1.Lx || P1.d) ? S1.V : nullptr;
        r.ES = S1.ES;
        r.nV = (unsigned)S1.nV;
        r.nA = (unsigned)S1.nA;
    }
    return r;
}

// Shared memory of a refill CTA: two windows, a ring of four tile descriptors and,
// for batched refills, the resolved base pointers of each descriptor's product.
template <int NT>
__host__ __device__ constexpr size_t refill_smem_bytes()
{
    return 2 * (size_t)win_of<NT>() * 8 + 4 * sizeof(TileDesc) + 4 * sizeof(ProdBase);
}

// Staged refill (single products): each tile's term words and entry records, two
// contiguous runs of the schedule, are copied into one of two shared-memory slots by
// two 1-D bulk copies (cp.async.bulk, this GPU's own memory, no multicast) issued by
// one thread while the tile before it runs, completing on the slot's mbarrier. A
// slot holds wcap words then ecap records; the copies start at the 16-byte boundary
// at or below the run (the schedule's arrays carry 16 bytes of padding past their
// ends for the rounded-up tails).
constexpr int STAGE_HDR = 4 * (int)sizeof(int) + 2 * (int)sizeof(unsigned long long); // entry counts, mbarriers
constexpr size_t STAGED_SMEM_MAX = 64 * 1024; // shared memory of a staged refill CTA at most
inline size_t staged_smem_bytes(int nt, int wcap, int ecap)
{
    const size_t base = nt == 256 ? refill_smem_bytes<256>() : refill_smem_bytes<128>();
    return base + STAGE_HDR + 2 * ((size_t)wcap * 4 + (size_t)ecap * 8);
}

__device__ __forceinline__ unsigned rf_smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void rf_mbar_init(unsigned long long *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(rf_smem_u32(bar)) : "memory");
}

// One thread: the tile's words and records into `slot`, completing on `bar`. The
// records end at nV at the latest (the validated term words never index past it;
// list words, whose entries the copy does not need, may count beyond).
__device__ __forceinline__ void rf_stage_tile(unsigned *slot, int wcap, const TileDesc &D, int nent,
                                              const unsigned *W, const int2 *ES, unsigned nV,
                                              unsigned long long *bar)
{
    const int wb = D.word_begin & ~3;
    const int wn = ((D.word_begin + D.nterms + 3) & ~3) - wb; // words, a multiple of 4
    const int eb = D.vbase & ~1;
    const long long eend = min((long long)D.vbase + nent, (long long)nV);
    const int en = eend > eb ? (int)(((eend + 1) & ~1LL) - eb) : 0; // records, a multiple of 2
    const unsigned bytes = (unsigned)wn * 4u + (unsigned)en * 8u;
    unsigned long long state;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
                 : "=l"(state)
                 : "r"(rf_smem_u32(bar)), "r"(bytes)
                 : "memory");
    (void)state;
    if (wn > 0)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(rf_smem_u32(slot)), "l"(W + wb), "r"((unsigned)wn * 4u), "r"(rf_smem_u32(bar))
                     : "memory");
    if (en > 0)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(rf_smem_u32(slot + wcap)), "l"(ES + eb), "r"((unsigned)en * 8u), "r"(rf_smem_u32(bar))
                     : "memory");
}

// Waits for phase `parity` of `bar` to complete, at most ~2^20 polls (with a short
// sleep between them); false if it did not.
__device__ __forceinline__ bool rf_mbar_wait(unsigned long long *bar, unsigned parity)
{
    const unsigned a = rf_smem_u32(bar);
    for (int it = 0; it < (1 << 20); ++it)
    {
        unsigned ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
        if (it > 8) __nanosleep(64);
    }
    return false;
}

template <int NT>
__device__ __forceinline__ void load_terms(const unsigned *__restrict__ W, int nterms, int base,
                                           unsigned (&w)[RUNROLL])
{
#pragma unroll
    for (int j = 0; j < RUNROLL; ++j)
    {
        const int u = base + threadIdx.x + j * NT;
        w[j] = u < nterms ? W[u] : (TERM_LIST << 12); // a list word is skipped by the term pass
    }
}

// One term u of entry e of a tile: V[slot] * A.x[bq + u]; false if the schedule
// does not hold a valid entry / position (reported through err by the caller).
__device__ __forceinline__ bool term_value(const ProdBase &pb, int vbase, unsigned w, int u, double &prod)
{
    const unsigned vi = (unsigned)(vbase + (int)(w >> 14));
    if (vi >= pb.nV) return false;
    const int2 es = pb.ES[vi];
    const unsigned a = (unsigned)(es.x + u);
    if (a >= pb.nA || (unsigned)es.y >= pb.nV) return false;
    prod = pb.V ? __dmul_rn(pb.V[es.y], pb.Ax[a]) : __dmul_rn(1.0, pb.Ax[a]);
    return true;
}

// Sum of a list output's terms from +0.0 in upstream's visiting order; the loads of
// four terms are in flight together.
__device__ __forceinline__ double list_sum(const ProdBase &pb, const TileDesc &D, const unsigned *__restrict__ items,
                                           int first, int end, int *err)
{
    const unsigned *Wt = pb.W + D.word_begin;
    double acc = 0.0;
    for (int i = first; i < end; i += 4)
    {
        double pr[4];
        bool ok[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            ok[j] = false;
            pr[j] = 0.0;
            if (i + j < end)
            {
                const int u = (int)items[i + j];
                ok[j] = (unsigned)u < (unsigned)D.nterms && term_value(pb, D.vbase, Wt[u], u, pr[j]);
                if (!ok[j]) atomicOr(err, 1);
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (ok[j]) acc = __dadd_rn(acc, pr[j]);
    }
    return acc;
}

// Copies a tile descriptor into the ring; in a batched refill the thread that holds
// the product index also resolves the product's base pointers into the ring (two
// tiles ahead of their use, so the refill never waits on them).
template <bool BATCHED>
__device__ __forceinline__ void copy_desc(TileDesc *dst, ProdBase *bdst, const TileDesc *__restrict__ src,
                                          const ProdPtrs *__restrict__ ptrs, const ProdSched *__restrict__ scheds,
                                          const ProdPtrs &P1, const ProdSched &S1)
{
    if (threadIdx.x < (int)(sizeof(TileDesc) / 4))
    {
        const int v = reinterpret_cast<const int *>(src)[threadIdx.x];
        reinterpret_cast<int *>(dst)[threadIdx.x] = v;
        if (BATCHED && threadIdx.x == (int)(offsetof(TileDesc, prod) / 4))
            *bdst = prod_base<true>(v, ptrs, scheds, P1, S1);
    }
}

// Base pointers of the tile in ring slot `slot`.
template <bool BATCHED>
__device__ __forceinline__ ProdBase base_of(const ProdBase *bse, int slot, const ProdPtrs &P1, const ProdSched &S1)
{
    if (BATCHED) return bse[slot];
    return prod_base<false>(0, nullptr, nullptr, P1, S1);
}

// Refill of the tile rows from the entry-major schedule. Persistent CTAs walk their
// tiles (blockIdx.x, + gridDim.x, ...). Per step every thread takes RUNROLL terms:
// word -> the entry's ES record (consecutive terms share entries: a few lines per
// warp) -> V[slot] and A.x[bq + u] (consecutive terms of an entry read one A row)
// -> the product into the tile's window in shared memory: stored for an output's
// only term (0.0 + v * A.x: upstream's accumulator starts at +0.0), atomically
// added for the two terms of a two-term output ((0 + a) + b == (0 + b) + a, signed
// zeros included). Outputs with three or more terms are summed afterwards by one
// thread each, in upstream's visiting order. The window is written back to C once,
// coalesced, and cleared; two windows alternate, so a tile needs one barrier. The
// words of the next step -- or of the next tile, whose descriptor is read two
// tiles ahead -- are loaded while a step's gathers are in flight.
// ESS (staged, single products): the tile's term words and entry records come from
// shared memory, bulk-copied there while the tile before it runs (the entry counts
// tile_nent travel with the descriptors, two tiles ahead), so a step issues only the
// V and A.x gathers to global memory. Same products, same sums: same bits.
template <bool BATCHED, int NT, bool ESS = false>
__global__ void __launch_bounds__(NT, refill_minb<NT>()) k_tile_refill(
    const TileDesc *__restrict__ tiles, int ntiles, const ProdPtrs *__restrict__ ptrs,
    const ProdSched *__restrict__ scheds, ProdPtrs P1, ProdSched S1, int *__restrict__ err,
    const int *__restrict__ tile_nent, int wcap, int ecap)
{
    constexpr int WIN = win_of<NT>();
    constexpr int RSTEP = RUNROLL * NT;
    extern __shared__ __align__(16) double rsm[];
    TileDesc *dsc = reinterpret_cast<TileDesc *>(rsm + 2 * WIN);
    ProdBase *bse = reinterpret_cast<ProdBase *>(dsc + 4);
    // ESS: the ring's entry counts, the two slots' mbarriers, the two slots
    int *nent_r = reinterpret_cast<int *>(bse + 4);
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(nent_r + 4);
    unsigned *slots = reinterpret_cast<unsigned *>(bars + 2);
    const int sstride = wcap + 2 * ecap; // 4-byte units per slot
    const int tid = threadIdx.x;
    const int G = gridDim.x;
    int t = blockIdx.x;
    if (t >= ntiles) return;
    for (int i = tid; i < 2 * WIN; i += NT) rsm[i] = 0.0;
    copy_desc<BATCHED>(dsc, bse, tiles + t, ptrs, scheds, P1, S1);
    if (t + G < ntiles) copy_desc<BATCHED>(dsc + 1, bse + 1, tiles + t + G, ptrs, scheds, P1, S1);
    if (ESS && tid == NT - 1)
    {
        nent_r[0] = tile_nent[t];
        if (t + G < ntiles) nent_r[1] = tile_nent[t + G];
        rf_mbar_init(&bars[0]);
        rf_mbar_init(&bars[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned w[RUNROLL];
    {
        const ProdBase pb = base_of<BATCHED>(bse, 0, P1, S1);
        if (ESS)
        {
            if (tid == 0) rf_stage_tile(slots, wcap, dsc[0], nent_r[0], pb.W, pb.ES, pb.nV, &bars[0]);
        }
        else
            load_terms<NT>(pb.W + dsc[0].word_begin, dsc[0].nterms, 0, w);
    }
    // launched as a programmatic dependent of the entry-value kernel: everything
    // above overlaps its tail; V is read only after it has completed (a no-op for
    // an ordinary launch)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    bool bad = false; // ESS: a slot that never arrived (its terms are skipped, err set)
    for (int k = 0;; ++k)
    {
        const TileDesc &D = dsc[k & 3];
        const bool has1 = t + G < ntiles;
        if (t + 2 * G < ntiles)
        {
            copy_desc<BATCHED>(dsc + ((k + 2) & 3), bse + ((k + 2) & 3), tiles + t + 2 * G, ptrs, scheds, P1, S1);
            if (ESS && tid == NT - 1) nent_r[(k + 2) & 3] = tile_nent[t + 2 * G];
        }
        double *win = rsm + (k & 1) * WIN;
        const ProdBase pb = base_of<BATCHED>(bse, k & 3, P1, S1);
        const unsigned *ws = nullptr;
        const int2 *esl = nullptr;
        if (ESS)
        {
            // the next tile's runs into the other slot (last read by the tile before
            // this one, whose term pass ended at a barrier)
            if (has1 && tid == 0)
                rf_stage_tile(slots + ((k + 1) & 1) * sstride, wcap, dsc[(k + 1) & 3], nent_r[(k + 1) & 3], pb.W,
                              pb.ES, pb.nV, &bars[(k + 1) & 1]);
            if (!bad && !rf_mbar_wait(&bars[k & 1], (unsigned)(k >> 1) & 1u))
            {
                atomicOr(err, 1);
                bad = true;
            }
            ws = slots + (k & 1) * sstride + (D.word_begin & 3);
            esl = reinterpret_cast<const int2 *>(slots + (k & 1) * sstride + wcap) + (D.vbase & 1);
        }
        const int nterms = D.nterms, nout = D.nout, vbase = D.vbase;
        if (ESS)
        {
            for (int base = 0; base < nterms; base += RSTEP)
            {
                unsigned ww[RUNROLL];
                int2 es[RUNROLL];
                bool term[RUNROLL];
#pragma unroll
                for (int j = 0; j < RUNROLL; ++j)
                {
                    const int u = base + tid + j * NT;
                    ww[j] = (!bad && u < nterms) ? ws[u] : (TERM_LIST << 12);
                    term[j] = !(ww[j] & (TERM_LIST << 12));
                    es[j] = term[j] ? esl[(int)(ww[j] >> 14)] : make_int2(0, 0);
                }
                double v[RUNROLL], x[RUNROLL];
#pragma unroll
                for (int j = 0; j < RUNROLL; ++j)
                {
                    v[j] = term[j] ? (pb.V ? pb.V[es[j].y] : 1.0) : 0.0;
                    x[j] = term[j] ? pb.Ax[es[j].x + base + tid + j * NT] : 0.0;
                }
#pragma unroll
                for (int j = 0; j < RUNROLL; ++j)
                {
                    if (!term[j]) continue;
                    const int p = (int)(ww[j] & 0xfffu);
                    const double prod = __dmul_rn(v[j], x[j]);
                    if (ww[j] & (TERM_PAIR << 12))
                        atomicAdd(&win[p], prod);
                    else
                        win[p] = __dadd_rn(0.0, prod);
                }
            }
        }
        else
        for (int base = 0;; base += RSTEP)
        {
            const bool last = base + RSTEP >= nterms;
            // every index below was checked once for the whole schedule when it was
            // built (k_validate_schedule); the padding words past nterms are list words
            int2 es[RUNROLL];
            bool term[RUNROLL];
#pragma unroll
            for (int j = 0; j < RUNROLL; ++j)
            {
                term[j] = !(w[j] & (TERM_LIST << 12));
                es[j] = term[j] ? pb.ES[vbase + (int)(w[j] >> 14)] : make_int2(0, 0);
            }
            double v[RUNROLL], x[RUNROLL];
#pragma unroll
            for (int j = 0; j < RUNROLL; ++j)
            {
                v[j] = term[j] ? (pb.V ? pb.V[es[j].y] : 1.0) : 0.0;
                x[j] = term[j] ? pb.Ax[es[j].x + base + tid + j * NT] : 0.0;
            }
            unsigned wn[RUNROLL];
            if (!last)
                load_terms<NT>(pb.W + D.word_begin, nterms, base + RSTEP, wn);
            else if (has1)
            {
                const TileDesc &Dn = dsc[(k + 1) & 3];
                const ProdBase pn = base_of<BATCHED>(bse, (k + 1) & 3, P1, S1);
                load_terms<NT>(pn.W + Dn.word_begin, Dn.nterms, 0, wn);
            }
            else
                load_terms<NT>(nullptr, 0, 0, wn); // nothing: list words
#pragma unroll
            for (int j = 0; j < RUNROLL; ++j)
            {
                if (!term[j]) continue;
                const int p = (int)(w[j] & 0xfffu);
                const double prod = __dmul_rn(v[j], x[j]);
                if (w[j] & (TERM_PAIR << 12))
                    atomicAdd(&win[p], prod);
                else
                    win[p] = __dadd_rn(0.0, prod);
            }
#pragma unroll
            for (int j = 0; j < RUNROLL; ++j) w[j] = wn[j];
            if (last) break;
        }
        __syncthreads(); // the window is complete
        if (D.nlist > 0)
        {
            const unsigned *hdr = pb.X + D.x_begin;
            const unsigned *items = hdr + D.nlist + 1;
            for (int l = tid; l < D.nlist; l += NT)
            {
                const unsigned h = hdr[l];
                const int p = (int)(h & 0xfffu);
                const double acc = list_sum(pb, D, items, (int)(h >> 12), (int)(hdr[l + 1] >> 12), err);
                if (p < nout)
                    win[p] = acc;
                else
                    atomicOr(err, 1);
            }
            __syncthreads();
        }
        // write-back (and clear) two outputs per 16-byte access where the tile's
        // first output is 16-byte aligned in C
        double *C = pb.C + D.out_begin;
        if ((reinterpret_cast<uintptr_t>(C) & 15) == 0)
        {
            double2 *C2 = reinterpret_cast<double2 *>(C);
            double2 *w2 = reinterpret_cast<double2 *>(win);
            for (int o = tid; o < (nout >> 1); o += NT)
            {
                C2[o] = w2[o];
                w2[o] = make_double2(0.0, 0.0);
            }
            if ((nout & 1) && tid == 0)
            {
                C[nout - 1] = win[nout - 1];
                win[nout - 1] = 0.0;
            }
        }
        else
            for (int o = tid; o < nout; o += NT)
            {
                C[o] = win[o];
                win[o] = 0.0;
            }
        if (!has1) break;
        t += G; // the words of the next tile were loaded by the last step
    }
}

// ------------------------------------------------------------ pipelined refill
// The same refill as k_tile_refill for a single product whose tiles hold at most
// PIPE_T terms, PIPE_E entries and PIPE_WIN outputs, with every load of a tile
// moved off the critical path by asynchronous copies into shared memory: the
// tile's term words and entry records are copied two tiles ahead (cp.async), its
// A.x value of every term and V value of every entry one tile ahead (cp.async
// gathers addressed by the staged records), so computing a tile reads shared
// memory only. Three stages rotate; one wait and one barrier per tile open each
// step. Products, order of the sums and roundings are those of k_tile_refill
// (bit-identical): a single term stored as 0.0 + v * A.x, a pair added atomically,
// outputs of three or more terms summed in visiting order by one thread each.
constexpr int PIPE_NT = 256;
constexpr int PIPE_T = 1024;
constexpr int PIPE_E = 512;
constexpr int PIPE_WIN = 1024;
constexpr int PIPE_RU = PIPE_T / PIPE_NT;
// descriptor ring: a descriptor is copied three tiles ahead, into a slot last used
// five tiles earlier (barriers in between), never one a slower thread still reads
constexpr int PIPE_RING = 8;

struct PipeStage
{
    unsigned w[PIPE_T];
    int2 es[PIPE_E];
    double ax[PIPE_T];
    double v[PIPE_E];
};

__host__ __device__ constexpr size_t pipe_smem_bytes()
{
    return 3 * sizeof(PipeStage) + 2 * PIPE_WIN * sizeof(double) + PIPE_RING * (sizeof(TileDesc) + sizeof(int));
}

__device__ __forceinline__ unsigned pipe_smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void pipe_cp4(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(pipe_smem_u32(dst)), "l"(src));
}
__device__ __forceinline__ void pipe_cp8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(pipe_smem_u32(dst)), "l"(src));
}
__device__ __forceinline__ void pipe_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void pipe_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// stage a: the tile's term words and entry records
__device__ __forceinline__ void pipe_stage_a(PipeStage &st, const TileDesc &D, int nent, const ProdSched &S)
{
    for (int u = threadIdx.x; u < D.nterms; u += PIPE_NT) pipe_cp4(&st.w[u], S.W + D.word_begin + u);
    for (int e = threadIdx.x; e < nent; e += PIPE_NT) pipe_cp8(&st.es[e], S.ES + D.vbase + e);
}

// stage b: A.x of every term and V of every entry, addressed by the staged records;
// the thread's words are kept for the compute step
__device__ __forceinline__ void pipe_stage_b(PipeStage &st, const TileDesc &D, int nent, const double *Ax,
                                             const double *V, unsigned (&w)[PIPE_RU])
{
#pragma unroll
    for (int j = 0; j < PIPE_RU; ++j)
    {
        const int u = threadIdx.x + j * PIPE_NT;
        w[j] = u < D.nterms ? st.w[u] : (TERM_LIST << 12); // a list word is skipped by the term step
        if (u < D.nterms) pipe_cp8(&st.ax[u], Ax + st.es[w[j] >> 14].x + u);
    }
    for (int e = threadIdx.x; e < nent; e += PIPE_NT)
    {
        if (V)
            pipe_cp8(&st.v[e], V + st.es[e].y);
        else
            st.v[e] = 1.0;
    }
}

__global__ void __launch_bounds__(PIPE_NT, 2) k_tile_refill_pipe(const TileDesc *__restrict__ tiles, int ntiles,
                                                                 const int *__restrict__ nent_of, ProdPtrs P1,
                                                                 ProdSched S1, int *__restrict__ err)
{
    extern __shared__ __align__(16) unsigned char psm[];
    PipeStage *st = reinterpret_cast<PipeStage *>(psm);
    double *wins = reinterpret_cast<double *>(psm + 3 * sizeof(PipeStage));
    TileDesc *dsc = reinterpret_cast<TileDesc *>(wins + 2 * PIPE_WIN);
    int *nent_r = reinterpret_cast<int *>(dsc + PIPE_RING);
    const int tid = threadIdx.x, G = gridDim.x;
    int t = blockIdx.x;
    if (t >= ntiles) return;
    const double *V = (P1.Lx || P1.d) ? S1.V : nullptr;
    auto load_desc = [&](int slot, int tile) {
        if (tid < (int)(sizeof(TileDesc) / 4))
            reinterpret_cast<int *>(dsc + slot)[tid] = reinterpret_cast<const int *>(tiles + tile)[tid];
        else if (tid == (int)(sizeof(TileDesc) / 4))
            nent_r[slot] = nent_of[tile];
    };
    for (int i = tid; i < 2 * PIPE_WIN; i += PIPE_NT) wins[i] = 0.0;
    load_desc(0, t);
    if (t + G < ntiles) load_desc(1, t + G);
    if (t + 2 * G < ntiles) load_desc(2, t + 2 * G);
    __syncthreads();
    pipe_stage_a(st[0], dsc[0], nent_r[0], S1);
    pipe_commit();
    if (t + G < ntiles) pipe_stage_a(st[1], dsc[1], nent_r[1], S1);
    pipe_commit();
    // launched as a programmatic dependent of the entry-value kernel: V is read only
    // after that grid completed (a no-op for an ordinary launch)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    pipe_wait_all();
    __syncthreads();
    unsigned w[PIPE_RU];
    pipe_stage_b(st[0], dsc[0], nent_r[0], P1.Ax, V, w);
    pipe_commit();
    for (int k = 0;; ++k)
    {
        const bool has1 = t + G < ntiles, has2 = t + 2 * G < ntiles;
        if (t + 3 * G < ntiles) load_desc((k + 3) & (PIPE_RING - 1), t + 3 * G);
        // stage b of this tile and stage a of the next have landed; the descriptor
        // copied last step is visible
        pipe_wait_all();
        __syncthreads();
        if (has2) pipe_stage_a(st[(k + 2) % 3], dsc[(k + 2) & (PIPE_RING - 1)], nent_r[(k + 2) & (PIPE_RING - 1)], S1);
        pipe_commit();
        unsigned wn[PIPE_RU];
#pragma unroll
        for (int j = 0; j < PIPE_RU; ++j) wn[j] = TERM_LIST << 12;
        if (has1)
            pipe_stage_b(st[(k + 1) % 3], dsc[(k + 1) & (PIPE_RING - 1)], nent_r[(k + 1) & (PIPE_RING - 1)], P1.Ax,
                         V, wn);
        pipe_commit();
        const TileDesc &D = dsc[k & (PIPE_RING - 1)];
        const PipeStage &cs = st[k % 3];
        double *win = wins + (k & 1) * PIPE_WIN;
#pragma unroll
        for (int j = 0; j < PIPE_RU; ++j)
        {
            if (w[j] & (TERM_LIST << 12)) continue;
            const int u = tid + j * PIPE_NT;
            const int p = (int)(w[j] & 0xfffu);
            const double prod = __dmul_rn(cs.v[w[j] >> 14], cs.ax[u]);
            if (w[j] & (TERM_PAIR << 12))
                atomicAdd(&win[p], prod);
            else
                win[p] = __dadd_rn(0.0, prod);
        }
        __syncthreads(); // the window is complete
        if (D.nlist > 0)
        {
            const unsigned *hdr = S1.X + D.x_begin;
            const unsigned *items = hdr + D.nlist + 1;
            for (int l = tid; l < D.nlist; l += PIPE_NT)
            {
                const unsigned h = hdr[l];
                const int p = (int)(h & 0xfffu);
                double acc = 0.0;
                for (int i = (int)(h >> 12); i < (int)(hdr[l + 1] >> 12); ++i)
                {
                    const int u = (int)items[i];
                    if ((unsigned)u >= (unsigned)D.nterms)
                    {
                        atomicOr(err, 1);
                        continue;
                    }
                    acc = __dadd_rn(acc, __dmul_rn(cs.v[cs.w[u] >> 14], cs.ax[u]));
                }
                if (p < D.nout)
                    win[p] = acc;
                else
                    atomicOr(err, 1);
            }
            __syncthreads();
        }
        double *C = P1.Cx + D.out_begin;
        const int nout = D.nout;
        if ((reinterpret_cast<uintptr_t>(C) & 15) == 0)
        {
            double2 *C2 = reinterpret_cast<double2 *>(C);
            double2 *w2 = reinterpret_cast<double2 *>(win);
            for (int o = tid; o < (nout >> 1); o += PIPE_NT)
            {
                C2[o] = w2[o];
                w2[o] = make_double2(0.0, 0.0);
            }
            if ((nout & 1) && tid == 0)
            {
                C[nout - 1] = win[nout - 1];
                win[nout - 1] = 0.0;
            }
        }
        else
            for (int o = tid; o < nout; o += PIPE_NT)
            {
                C[o] = win[o];
                win[o] = 0.0;
            }
        if (!has1) break;
        t += G;
#pragma unroll
        for (int j = 0; j < PIPE_RU; ++j) w[j] = wn[j];
    }
    pipe_wait_all();
}

// Value pointers from a device binding table (batched refills replayed from a CUDA
// graph read the pointers bound at replay time), when given.
__device__ __forceinline__ void bind_values(NumArgs &a, const ProdPtrs *__restrict__ vals)
{
    if (vals)
    {
        a.Lx = vals->Lx;
        a.d = vals->d;
        a.Ax = vals->Ax;
        a.Cx = vals->Cx;
    }
}

// Medium rows: one CTA per row, shared accumulator indexed by output position;
// a claim table orders same-position terms of a chunk by term index.
template <int CAP>
__global__ void k_num_cta(const int *__restrict__ rows, int count, NumArgs a,
                          const ProdPtrs *__restrict__ vals)
{
    bind_values(a, vals);
    extern __shared__ __align__(16) unsigned char smraw[];
    double *acc = (double *)smraw;
    CtaChunk ch;
    ch.v = acc + CAP;
    int *ci = (int *)(ch.v + blockDim.x);
    int *claim = ci + CAP;
    ch.incl = claim + CAP;
    ch.s = ch.incl + blockDim.x;
    ch.len = ch.s + blockDim.x;
    ch.scr = ch.len + blockDim.x;
    for (int it = blockIdx.x; it < count; it += gridDim.x)
    {
        int row = rows[it];
        int b = row / a.L_m, r = row - b * a.L_m;
        int cs = a.Cp[row], nr = a.Cp[row + 1] - cs;
        for (int q = threadIdx.x; q < nr; q += blockDim.x)
        {
            ci[q] = a.Ci[cs + q];
            acc[q] = 0.0;
            claim[q] = INT_MAX;
        }
        __syncthreads();
        int ls = a.Lp[r], le = a.Lp[r + 1];
        for (int c = ls; c < le; c += blockDim.x)
        {
            int total = cta_load_chunk(a.Li, a.Ap, b, a.n_L, c, le, ch, a.Lx, a.L_map, a.d, true);
            int nent = min((int)blockDim.x, le - c);
            for (int base = 0; base < total; base += blockDim.x)
            {
                int u = base + threadIdx.x;
                bool pending = u < total;
                int pos = 0;
                double prod = 0.0;
                if (pending)
                {
                    int e = cta_entry_of(ch.incl, nent, u);
                    int jj = ch.s[e] + u - (ch.incl[e] - ch.len[e]);
                    int j = a.Ai[jj];
                    prod = __dmul_rn(ch.v[e], a.Ax[jj]);
                    pos = lower_bound_dev(ci, nr, j);
                    if (pos >= nr || ci[pos] != j)
                    {
                        atomicOr(a.err, 1);
                        pending = false;
                    }
                }
                while (true)
                {
                    if (pending) atomicMin(&claim[pos], u);
                    __syncthreads();
                    bool won = pending && claim[pos] == u;
                    if (won) acc[pos] = __dadd_rn(acc[pos], prod);
                    __syncthreads();
                    if (won)
                    {
                        claim[pos] = INT_MAX;
                        pending = false;
                    }
                    if (!__syncthreads_or(pending)) break;
                }
            }
            __syncthreads();
        }
        for (int q = threadIdx.x; q < nr; q += blockDim.x) a.Cx[cs + q] = acc[q];
        __syncthreads();
    }
}

constexpr int GMEM_CLAIM = 8192; // claim slots (a power of two)
constexpr int GMEM_TPT = 4;       // terms per thread in one claim round
constexpr int GMEM_EPT = 2;       // L entries per thread in one chunk
constexpr int GMEM_CTAS_PER_SM = 2;
constexpr int GMEM_THREADS = 512;
constexpr int GMEM_CHUNK = GMEM_THREADS * GMEM_EPT;

__host__ __device__ constexpr size_t gmem_smem_bytes()
{
    // per chunk entry: value (8 B), inclusive term count, A row start and length
    // (4 B each); the claim table; the scan scratch
    return (size_t)GMEM_CHUNK * 20 + GMEM_CLAIM * 4 + 64 * 4;
}

// Large rows: accumulate straight into C.x; a per-CTA global map column -> position
// (only this row's columns are ever read, so it never needs clearing) and a hashed
// claim table keep same-position terms in order. The row's L entries are taken
// GMEM_CHUNK at a time (GMEM_EPT consecutive entries per thread), and their terms
// in claim rounds of GMEM_TPT terms per thread: every pending term claims its slot
// with its term index, the smallest index of a slot adds its product, and the round
// repeats until no term is pending -- so the terms of one output are added in
// ascending term order (upstream's visiting order), whichever threads hold them.
// RANK: the map is a rank structure instead -- per 64 columns one 16-byte entry
// {column bitmap of the row's columns in the word, position of the word's first
// column}, position = prefix + popcount of the lower bits -- 1/16 of the plain map's
// bytes, so the CTAs' maps (n / 4 bytes each) stay in L2; the row writes one entry
// per word it touches and reads only those, so it needs no clearing either.
__device__ __forceinline__ int rank_pos(const uint4 *__restrict__ rmap, int j)
{
    const uint4 e = rmap[j >> 6];
    const unsigned long long bits = ((unsigned long long)e.y << 32) | e.x;
    const unsigned long long below = bits & ((1ull << (j & 63)) - 1ull);
    return (int)e.z + __popcll(below);
}

template <bool RANK>
__global__ void __launch_bounds__(GMEM_THREADS, GMEM_CTAS_PER_SM) k_num_gmem(const int *__restrict__ rows, int count, NumArgs a,
                                                          int *__restrict__ posmap_all, int n,
                                                          const ProdPtrs *__restrict__ vals,
                                                          int *__restrict__ next_row)
{
    bind_values(a, vals);
    extern __shared__ __align__(16) unsigned char smraw[];
    double *ev = (double *)smraw;                 // entry values
    int *incl = (int *)(ev + GMEM_CHUNK);         // inclusive term counts
    int *es = incl + GMEM_CHUNK;                  // A row starts
    int *elen = es + GMEM_CHUNK;                  // A row lengths
    int *claim = elen + GMEM_CHUNK;
    int *scr = claim + GMEM_CLAIM;
    int *posmap = posmap_all + (long long)blockIdx.x * n;
    uint4 *rmap = reinterpret_cast<uint4 *>(posmap_all) + (long long)blockIdx.x * ((n + 63) / 64);
    __shared__ int it_sh;
    // rows taken in list order: from a shared counter when given (the list is then
    // ordered by work, largest first), else every gridDim-th
    for (int it = blockIdx.x;;)
    {
        if (next_row)
        {
            __syncthreads();
            if (threadIdx.x == 0) it_sh = atomicAdd(next_row, 1);
            __syncthreads();
            it = it_sh;
        }
        if (it >= count) break;
        int row = rows[it];
        int b = row / a.L_m, r = row - b * a.L_m;
        int cs = a.Cp[row], nr = a.Cp[row + 1] - cs;
        double *acc = a.Cx + cs;
        for (int q = threadIdx.x; q < nr; q += blockDim.x)
        {
            const int j = a.Ci[cs + q];
            if (RANK)
            {
                // the thread holding a word's first column writes the word's entry
                const int w = j >> 6;
                if (q == 0 || (a.Ci[cs + q - 1] >> 6) != w)
                {
                    unsigned long long bits = 0;
                    for (int r = q; r < nr; ++r)
                    {
                        const int jr = a.Ci[cs + r];
                        if ((jr >> 6) != w) break;
                        bits |= 1ull << (jr & 63);
                    }
                    rmap[w] = make_uint4((unsigned)bits, (unsigned)(bits >> 32), (unsigned)q, 0u);
                }
            }
            else
                posmap[j] = q;
            acc[q] = 0.0;
        }
        for (int q = threadIdx.x; q < GMEM_CLAIM; q += blockDim.x) claim[q] = INT_MAX;
        __syncthreads();
        int ls = a.Lp[r], le = a.Lp[r + 1];
        for (int c = ls; c < le; c += GMEM_CHUNK)
        {
            // this thread's GMEM_EPT consecutive entries, their term counts scanned
            const int e0 = threadIdx.x * GMEM_EPT;
            int mine = 0;
            int lens[GMEM_EPT];
#pragma unroll
            for (int k = 0; k < GMEM_EPT; ++k)
            {
                const int ii = c + e0 + k;
                int st = 0, ln = 0;
                double v = 0.0;
                if (ii < le)
                {
                    const int kk = a.Li[ii] + b * a.n_L;
                    st = a.Ap[kk];
                    ln = a.Ap[kk + 1] - st;
                    const double lx = a.Lx ? a.Lx[a.L_map ? a.L_map[ii] : ii] : 1.0;
                    v = a.d ? __dmul_rn(lx, a.d[kk]) : lx;
                }
                es[e0 + k] = st;
                elen[e0 + k] = ln;
                ev[e0 + k] = v;
                lens[k] = ln;
                mine += ln;
            }
            const int before = block_incl_scan_int(mine, scr) - mine; // ends with a barrier
            int run = before;
#pragma unroll
            for (int k = 0; k < GMEM_EPT; ++k)
            {
                run += lens[k];
                incl[e0 + k] = run;
            }
            __syncthreads();
            const int total = incl[GMEM_CHUNK - 1];
            const int nent = min(GMEM_CHUNK, le - c);
            for (int base = 0; base < total; base += blockDim.x * GMEM_TPT)
            {
                int pos[GMEM_TPT];
                double prod[GMEM_TPT];
                unsigned pend = 0; // bit k: term k of this thread still to be added
#pragma unroll
                for (int k = 0; k < GMEM_TPT; ++k)
                {
                    const int u = base + k * blockDim.x + threadIdx.x;
                    pos[k] = 0;
                    prod[k] = 0.0;
                    if (u < total)
                    {
                        int e = cta_entry_of(incl, nent, u);
                        int jj = es[e] + u - (incl[e] - elen[e]);
                        int j = a.Ai[jj];
                        prod[k] = __dmul_rn(ev[e], a.Ax[jj]);
                        pos[k] = RANK ? rank_pos(rmap, j) : posmap[j];
                        if (pos[k] < 0 || pos[k] >= nr)
                            atomicOr(a.err, 1);
                        else
                            pend |= 1u << k;
                    }
                }
                while (true)
                {
#pragma unroll
                    for (int k = 0; k < GMEM_TPT; ++k)
                        if (pend & (1u << k))
                            atomicMin(&claim[pos[k] & (GMEM_CLAIM - 1)], base + k * (int)blockDim.x + (int)threadIdx.x);
                    __syncthreads();
                    unsigned won = 0;
#pragma unroll
                    for (int k = 0; k < GMEM_TPT; ++k)
                        if ((pend & (1u << k)) &&
                            claim[pos[k] & (GMEM_CLAIM - 1)] == base + k * (int)blockDim.x + (int)threadIdx.x)
                        {
                            won |= 1u << k;
                            acc[pos[k]] = __dadd_rn(acc[pos[k]], prod[k]);
                        }
                    __syncthreads();
#pragma unroll
                    for (int k = 0; k < GMEM_TPT; ++k)
                        if (won & (1u << k)) claim[pos[k] & (GMEM_CLAIM - 1)] = INT_MAX;
                    pend &= ~won;
                    if (!__syncthreads_or(pend != 0)) break;
                }
            }
            __syncthreads();
        }
        __syncthreads();
        if (!next_row) it += gridDim.x;
    }
}

// ------------------------------------------------------------ host helpers
int grid_for(long long work_items, int per_block, int cap)
{
    long long g = (work_items + per_block - 1) / per_block;
    return (int)std::max<long long>(1, std::min<long long>(g, cap));
}

// Groups item ids by class (classes >= nbins are dropped). counts/offsets on host.
void bin_items(const unsigned char *d_cls, int n, int nbins, DevBuf<int> &lists, int *count,
               int *offset, cudaStream_t s)
{
    Runtime &rt = runtime();
    DevBuf<int> cnt(2 * nbins);
    SDL_CUDA(cudaMemsetAsync(cnt.get(), 0, cnt.bytes(), s));
    int grid = grid_for(n, 256, rt.num_sms * 8);
    SDL_LAUNCH(k_bin_count, grid, 256, 0, s, d_cls, n, nbins, cnt.get());
    SDL_CUDA(cudaMemcpyAsync(count, cnt.get(), nbins * sizeof(int), cudaMemcpyDeviceToHost, s));
    SDL_CUDA(cudaStreamSynchronize(s));
    offset[0] = 0;
    for (int c = 0; c < nbins; ++c) offset[c + 1] = offset[c] + count[c];
    lists.reset(std::max(1, offset[nbins]));
    if (offset[nbins] == 0) return;
    SDL_CUDA(cudaMemcpyAsync(cnt.get() + nbins, offset, nbins * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    SDL_LAUNCH(k_bin_scatter, grid, 256, 0, s, d_cls, n, nbins, cnt.get() + nbins, lists.get());
    SDL_CUDA(cudaStreamSynchronize(s));
}

template <class K>
void set_smem(K kernel, size_t bytes)
{
    if (bytes > 48 * 1024)
        SDL_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

} // namespace

namespace {

// Launches the symbolic kernel of every row class over the binned row lists.
void sym_launch(const SymArgs &sa, const int *lists, const int *cnt, const int *off,
                const ProductDesc &d, const TuneConfig &cfg, cudaStream_t s)
{
    Runtime &rt = runtime();
    const int cap = rt.num_sms * 16;
    const int wpb = std::max(1, std::min(16, cfg.rows_per_cta_warp));
    if (cnt[SYM_W32])
        SDL_LAUNCH(k_sym_warp<32>, grid_for(cnt[SYM_W32], wpb, cap), wpb * 32, wpb * 32 * 4, s,
                   lists + off[SYM_W32], cnt[SYM_W32], sa);
    if (cnt[SYM_W128])
        SDL_LAUNCH(k_sym_warp<128>, grid_for(cnt[SYM_W128], wpb, cap), wpb * 32, wpb * 128 * 4, s,
                   lists + off[SYM_W128], cnt[SYM_W128], sa);
    if (cnt[SYM_W512])
        SDL_LAUNCH(k_sym_warp<512>, grid_for(cnt[SYM_W512], wpb, cap), wpb * 32, wpb * 512 * 4, s,
                   lists + off[SYM_W512], cnt[SYM_W512], sa);
    if (cnt[SYM_C2K])
    {
        const int th = cfg.cta_threads_2k == 128 || cfg.cta_threads_2k == 512 ? cfg.cta_threads_2k : 256;
        size_t sm = 2048 * 4 + (3 * th + 32) * 4;
        SDL_LAUNCH(k_sym_cta<2048>, grid_for(cnt[SYM_C2K], 1, cap), th, sm, s, lists + off[SYM_C2K],
                   cnt[SYM_C2K], sa);
    }
    if (cnt[SYM_C8K])
    {
        int th = 512;
        size_t sm = 8192 * 4 + (3 * th + 32) * 4;
        set_smem(k_sym_cta<8192>, sm);
        SDL_LAUNCH(k_sym_cta<8192>, grid_for(cnt[SYM_C8K], 1, cap), th, sm, s, lists + off[SYM_C8K],
                   cnt[SYM_C8K], sa);
    }
    if (cnt[SYM_BITMAP])
    {
        int th = 1024;
        size_t fixed = (3 * th + 32) * 4;
        long long want_words = ((long long)d.A_n + 31) / 32;
        long long max_words = (rt.smem_optin - (long long)fixed - 1024) / 4;
        long long w = std::min((want_words + 31) / 32 * 32, max_words / 32 * 32);
        int words = (int)std::max<long long>(32, w);
        size_t sm = (size_t)words * 4 + fixed;
        set_smem(k_sym_bitmap, sm);
        const int nbr = cnt[SYM_BITMAP];
        const int grid = grid_for(nbr, 1, rt.num_sms * 2);
        if (nbr <= grid)
            SDL_LAUNCH(k_sym_bitmap, grid, th, sm, s, lists + off[SYM_BITMAP], nbr, sa, words, nullptr);
        else
        {
            // more rows than CTAs: handed out largest first (by their scratch span) from
            // a counter, so no CTA is left with several of the largest rows
            DevBuf<long long> span((size_t)nbr);
            SDL_LAUNCH(k_row_spans, grid_for(nbr, 256, rt.num_sms * 4), 256, 0, s, lists + off[SYM_BITMAP], nbr,
                       sa.ub_off, span.get());
            std::vector<int> hrows(nbr);
            std::vector<long long> hspan(nbr);
            SDL_CUDA(cudaMemcpyAsync(hrows.data(), lists + off[SYM_BITMAP], (size_t)nbr * sizeof(int),
                                     cudaMemcpyDeviceToHost, s));
            SDL_CUDA(cudaMemcpyAsync(hspan.data(), span.get(), (size_t)nbr * sizeof(long long),
                                     cudaMemcpyDeviceToHost, s));
            SDL_CUDA(cudaStreamSynchronize(s));
            std::vector<int> idx(nbr);
            for (int q = 0; q < nbr; ++q) idx[q] = q;
            std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return hspan[x] > hspan[y]; });
            for (int q = 0; q < nbr; ++q) idx[q] = hrows[idx[q]];
            DevBuf<int> order((size_t)nbr), counter(1);
            SDL_CUDA(cudaMemcpyAsync(order.get(), idx.data(), (size_t)nbr * sizeof(int), cudaMemcpyHostToDevice, s));
            SDL_CUDA(cudaMemsetAsync(counter.get(), 0, sizeof(int), s));
            SDL_LAUNCH(k_sym_bitmap, grid, th, sm, s, order.get(), nbr, sa, words, counter.get());
            SDL_CUDA(cudaStreamSynchronize(s)); // idx and the queue are released on return
        }
    }
}

void validate_product(const ProductDesc &d, const TuneConfig &cfg, Product &P, cudaStream_t s)
{
    if (d.blocks < 1) fail(SDL_ERR_INVALID, "product: blocks must be >= 1");
    if (d.L_m < 0 || d.A_m < 0 || d.A_n < 0) fail(SDL_ERR_INVALID, "product: negative size");
    if (d.A_m % d.blocks != 0)
        fail(SDL_ERR_INVALID, "product: rows of A must be a multiple of blocks");
    long long m_out_ll = (long long)d.L_m * d.blocks;
    if (m_out_ll > INT_MAX) fail(SDL_ERR_OVERFLOW, "product: blocks * rows of L exceeds INT_MAX");
    P.desc = d;
    P.cfg = cfg;
    P.m_out = (int)m_out_ll;
    P.n = d.A_n;
    P.n_L = d.A_m / d.blocks;
    validate_compressed(d.Lp, d.Li, d.L_m, P.n_L, d.L_nnz, "product operand L", s);
    validate_compressed(d.Ap, d.Ai, d.A_m, d.A_n, d.A_nnz, "product operand A", s);
    if (d.L_map) validate_compressed(nullptr, d.L_map, 0, INT_MAX, d.L_nnz, "product L_map", s);
}

// ------------------------------------------------------------ rows beyond the tile budget
// Term counts and output counts of the big rows.
__global__ void k_big_sizes(const int *__restrict__ rows, int nbig, const long long *__restrict__ ub,
                            const int *__restrict__ Cp, long long *__restrict__ terms, long long *__restrict__ outs)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nbig;
         i += (long long)gridDim.x * blockDim.x)
    {
        const int r = rows[i];
        terms[i] = ub[r];
        outs[i] = Cp[r + 1] - Cp[r];
    }
}

// One CTA per big row at a time (grid-stride over the rows): every term of the row,
// in upstream's visiting order t (stored at the row's term offset + t), gets the key
// = its output's index among all big-row outputs and its {A position, entry-value
// slot}. Output positions come from a per-CTA global map column -> position; only
// the row's own columns are ever read, so it needs no clearing.
__global__ void __launch_bounds__(512, 2) k_big_terms(const int *__restrict__ rows, int nbig,
                                                      const int *__restrict__ tterm_off,
                                                      const int *__restrict__ bout_off, NumArgs a,
                                                      int *__restrict__ posmap_all, int n,
                                                      unsigned *__restrict__ keys, uint2 *__restrict__ data,
                                                      const int *__restrict__ order, int *__restrict__ next_row)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    CtaChunk ch;
    ch.v = nullptr;
    ch.incl = reinterpret_cast<int *>(smraw);
    ch.s = ch.incl + blockDim.x;
    ch.len = ch.s + blockDim.x;
    ch.scr = ch.len + blockDim.x;
    int *posmap = posmap_all + (long long)blockIdx.x * n;
    uint4 *rmap = reinterpret_cast<uint4 *>(posmap_all) + (long long)blockIdx.x * ((n + 63) / 64);
    __shared__ int q_sh;
    // the rows in the order `order` gives (largest first), handed out by a counter
    for (;;)
    {
        __syncthreads();
        if (threadIdx.x == 0) q_sh = atomicAdd(next_row, 1);
        __syncthreads();
        if (q_sh >= nbig) break;
        const int it = order[q_sh];
        const int row = rows[it];
        const int b = row / a.L_m, r = row - b * a.L_m;
        const int cs = a.Cp[row], nr = a.Cp[row + 1] - cs;
        for (int q = threadIdx.x; q < nr; q += blockDim.x) posmap[a.Ci[cs + q]] = q;
        __syncthreads();
        const long long base = tterm_off[it];
        long long cursor = 0;
        const int ls = a.Lp[r], le = a.Lp[r + 1];
        for (int c = ls; c < le; c += blockDim.x)
        {
            const int total = cta_load_chunk(a.Li, a.Ap, b, a.n_L, c, le, ch, nullptr, nullptr, nullptr, false);
            const int nent = min((int)blockDim.x, le - c);
            for (int u = threadIdx.x; u < total; u += blockDim.x)
            {
                const int e = cta_entry_of(ch.incl, nent, u);
                const int jj = ch.s[e] + u - (ch.incl[e] - ch.len[e]);
                const int ii = c + e;
                const int pos = posmap[a.Ai[jj]];
                const long long t = cursor + u;
                const unsigned slot = (unsigned)(b * a.L_nnz + (a.value_order ? a.L_map[ii] : ii));
                if (pos < 0 || pos >= nr)
                {
                    atomicOr(a.err, 1);
                    continue;
                }
                keys[base + t] = (unsigned)(bout_off[it] + pos);
                data[base + t] = make_uint2((unsigned)jj, slot);
            }
            cursor += total;
            __syncthreads();
        }
        __syncthreads();
    }
}

// After the stable sort by output: the first pair of every output (every output
// has a term, so each output index starts exactly one run).
__global__ void k_big_starts(const unsigned *__restrict__ keys, int T, int O, int *__restrict__ ostart,
                             int *__restrict__ err)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < T;
         i += (long long)gridDim.x * blockDim.x)
    {
        const unsigned k = keys[i];
        if (k >= (unsigned)O)
        {
            atomicOr(err, 1);
            continue;
        }
        if (i == 0 || keys[i - 1] != k) ostart[k] = (int)i;
    }
}

// Output-major refill of the big rows: a thread per output sums its pairs from +0.0
// in upstream's visiting order (loads of four pairs in flight together). A CTA takes
// 256 consecutive big outputs; its first row is found by a search, then each thread
// steps forward over the rows its output is past.
template <bool BATCHED>
__global__ void __launch_bounds__(256) k_big_refill(const int *__restrict__ brows, int nbig,
                                                    const int *__restrict__ bout_off, int nout,
                                                    const int *__restrict__ bostart, const uint2 *__restrict__ pairs,
                                                    const int *__restrict__ Cp, const ProdPtrs *__restrict__ vals_dev,
                                                    ProdPtrs vals, const double *__restrict__ V, long long nV,
                                                    long long nA, int *__restrict__ err)
{
    __shared__ int r_first;
    ProdPtrs P = vals;
    if (BATCHED) P = *vals_dev;
    const double *Vp = (P.Lx || P.d) ? V : nullptr;
    const int o_first = blockIdx.x * blockDim.x;
    if (o_first >= nout) return;
    if (threadIdx.x == 0)
    {
        int lo = 0, hi = nbig; // last row with bout_off <= o_first
        while (hi - lo > 1)
        {
            const int mid = (lo + hi) >> 1;
            if (bout_off[mid] <= o_first)
                lo = mid;
            else
                hi = mid;
        }
        r_first = lo;
    }
    __syncthreads();
    const int o = o_first + threadIdx.x;
    if (o >= nout) return;
    int r = r_first;
    while (r + 1 < nbig && bout_off[r + 1] <= o) ++r;
    const int cpos = Cp[brows[r]] + (o - bout_off[r]);
    const int i0 = bostart[o], i1 = bostart[o + 1];
    double acc = 0.0;
    for (int i = i0; i < i1; i += 4)
    {
        double pr[4];
        bool ok[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            ok[j] = false;
            pr[j] = 0.0;
            if (i + j < i1)
            {
                const uint2 q = pairs[i + j];
                if ((long long)q.x < nA && (long long)q.y < nV)
                {
                    ok[j] = true;
                    pr[j] = __dmul_rn(Vp ? Vp[q.y] : 1.0, P.Ax[q.x]);
                }
                else
                    atomicOr(err, 1);
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (ok[j]) acc = __dadd_rn(acc, pr[j]);
    }
    P.Cx[cpos] = acc;
}

// Output-major term lists of the rows beyond the tile budget (k_big_terms, a stable
// radix sort by output, k_big_starts). Kept within 31-bit offsets; larger products
// keep the CTA kernels.
void build_big_lists(const ProductDesc &d, Product &P, const long long *ub, const NumArgs &na, cudaStream_t s)
{
    Runtime &rt = runtime();
    P.big_lists = false;
    const int nbig = P.num_count[NUM_C2K] + P.num_count[NUM_C8K] + P.num_count[NUM_GMEM];
    if (nbig == 0) return;
    const int *rows = P.num_rows.get() + P.num_offset[NUM_C2K]; // classes C2K, C8K, GMEM are adjacent
    DevBuf<long long> terms(nbig), outs(nbig), toff((size_t)nbig + 1), ooff((size_t)nbig + 1);
    SDL_LAUNCH(k_big_sizes, grid_for(nbig, 256, rt.num_sms * 8), 256, 0, s, rows, nbig, ub, P.Cp.get(),
               terms.get(), outs.get());
    const long long T = exclusive_scan_i64(terms.get(), toff.get(), nbig, s);
    const long long O = exclusive_scan_i64(outs.get(), ooff.get(), nbig, s);
    if (T >= INT_MAX || O >= INT_MAX || T < O) return; // the CTA kernels handle them
    // 32-bit copies of the offsets (the sort and the refill take int offsets)
    std::vector<long long> ht((size_t)nbig + 1), ho((size_t)nbig + 1);
    SDL_CUDA(cudaMemcpyAsync(ht.data(), toff.get(), ht.size() * sizeof(long long), cudaMemcpyDeviceToHost, s));
    SDL_CUDA(cudaMemcpyAsync(ho.data(), ooff.get(), ho.size() * sizeof(long long), cudaMemcpyDeviceToHost, s));
    SDL_CUDA(cudaStreamSynchronize(s));
    std::vector<int> hti(ht.begin(), ht.end()), hoi(ho.begin(), ho.end());
    DevBuf<int> toff32 = DevBuf<int>((size_t)nbig + 1);
    P.bout_off.reset((size_t)nbig + 1);
    SDL_CUDA(cudaMemcpyAsync(toff32.get(), hti.data(), hti.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    SDL_CUDA(cudaMemcpyAsync(P.bout_off.get(), hoi.data(), hoi.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    // terms -> (output, pair), then a stable sort by output
    const long long per_slot = std::max(1, P.n);
    const int slots = (int)std::min<long long>(
        {(long long)rt.num_sms * 2, std::max<long long>(1, (2LL << 30) / (per_slot * 4)), (long long)nbig});
    // the rows by term count, largest first (a counter hands them out)
    std::vector<int> ord(nbig);
    {
        std::vector<long long> tc(nbig);
        for (int i = 0; i < nbig; ++i) tc[i] = ht[i + 1] - ht[i];
        for (int i = 0; i < nbig; ++i) ord[i] = i;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return tc[x] > tc[y]; });
    }
    DevBuf<int> order((size_t)nbig), counter(1);
    SDL_CUDA(cudaMemcpyAsync(order.get(), ord.data(), (size_t)nbig * sizeof(int), cudaMemcpyHostToDevice, s));
    SDL_CUDA(cudaMemsetAsync(counter.get(), 0, sizeof(int), s));
    {
        DevBuf<int> posmap((size_t)slots * per_slot);
        DevBuf<unsigned> keys(std::max<long long>(1, T)), keys2(std::max<long long>(1, T));
        DevBuf<uint2> tmp(std::max<long long>(1, T));
        P.bpairs.reset(std::max<long long>(1, T));
        const int th = 512;
        const size_t sm = (3 * (size_t)th + 32) * 4;
        SDL_LAUNCH(k_big_terms, slots, th, sm, s, rows, nbig, toff32.get(), P.bout_off.get(), na, posmap.get(), P.n,
                   keys.get(), P.bpairs.get(), order.get(), counter.get());
        if (take_device_error(s)) fail(SDL_ERR_INTERNAL, "product plan: a term column is missing from its row");
        int bits = 1;
        while (bits < 32 && (1LL << bits) < O) ++bits;
        radix_sort_pairs(keys.get(), P.bpairs.get(), keys2.get(), tmp.get(), (int)T, bits, s);
        P.bostart.reset((size_t)O + 1);
        SDL_CUDA(cudaMemcpyAsync(P.bostart.get() + O, &hti[nbig], sizeof(int), cudaMemcpyHostToDevice, s));
        SDL_LAUNCH(k_big_starts, grid_for(T, 256, rt.num_sms * 8), 256, 0, s, keys.get(), (int)T, (int)O,
                   P.bostart.get(), rt.d_error);
        if (take_device_error(s)) fail(SDL_ERR_INTERNAL, "product plan: heavy-row term lists are inconsistent");
    }
    P.brows.reset(nbig);
    SDL_CUDA(cudaMemcpyAsync(P.brows.get(), rows, (size_t)nbig * sizeof(int), cudaMemcpyDeviceToDevice, s));
    SDL_CUDA(cudaStreamSynchronize(s));
    P.nbig = nbig;
    P.big_outputs = (int)O;
    P.big_lists = true;
}

// Checks every index the tile refill will use, once per schedule: per tile, its
// window and output range, its words inside the word array, and for every term
// word that is not a list word its entry, the entry's A position for that term and
// its value slot, and its output inside the window; per list, its output and items.
// The refill's term loop then reads without per-term checks.
__global__ void k_validate_schedule(const TileDesc *__restrict__ tiles, int ntiles, const unsigned *__restrict__ W,
                                    long long word_total, const unsigned *__restrict__ X, long long x_total,
                                    const int2 *__restrict__ ES, long long nV, long long nA, long long nnzC,
                                    int *__restrict__ err)
{
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    {
        const TileDesc D = tiles[t];
        if (D.nterms < 0 || D.nout < 0 || D.nout > TILE_ACC || D.out_begin < 0 ||
            (long long)D.out_begin + D.nout > nnzC || D.word_begin < 0 ||
            (long long)D.word_begin + D.nterms > word_total || D.vbase < 0 || D.prod != 0)
        {
            if (threadIdx.x == 0) atomicOr(err, 4);
            continue;
        }
        for (int u = threadIdx.x; u < D.nterms; u += blockDim.x)
        {
            const unsigned w = W[D.word_begin + u];
            if (w & (TERM_LIST << 12)) continue;
            const long long vi = (long long)D.vbase + (w >> 14);
            if (vi >= nV)
            {
                atomicOr(err, 4);
                continue;
            }
            const int2 es = ES[vi];
            const long long a = (long long)es.x + u;
            if (a < 0 || a >= nA || es.y < 0 || es.y >= nV || (int)(w & 0xfffu) >= D.nout) atomicOr(err, 4);
        }
        if (D.nlist > 0)
        {
            if (D.x_begin < 0 || (long long)D.x_begin + D.nlist + 1 > x_total)
            {
                if (threadIdx.x == 0) atomicOr(err, 4);
                continue;
            }
            const unsigned *hdr = X + D.x_begin;
            const long long items_end = (long long)(hdr[D.nlist] >> 12);
            if ((long long)D.x_begin + D.nlist + 1 + items_end > x_total)
            {
                if (threadIdx.x == 0) atomicOr(err, 4);
                continue;
            }
            for (int l = threadIdx.x; l < D.nlist; l += blockDim.x)
                if ((int)(hdr[l] & 0xfffu) >= D.nout || (hdr[l] >> 12) > (hdr[l + 1] >> 12)) atomicOr(err, 4);
            const unsigned *items = hdr + D.nlist + 1;
            for (long long i = threadIdx.x; i < items_end; i += blockDim.x)
                if (items[i] >= (unsigned)D.nterms) atomicOr(err, 4);
        }
    }
}

// Largest window (outputs) of the plan's tiles.
__global__ void k_tile_max_out(const TileDesc *__restrict__ tiles, int ntiles, int *__restrict__ out)
{
    int m = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ntiles;
         t += (long long)gridDim.x * blockDim.x)
        m = max(m, tiles[t].nout);
    atomicMax(out, m);
}

// Entries of every tile (its largest entry index + 1, from its term words; entry
// indices grow along a tile's words) and the largest term and entry counts of a tile.
__global__ void k_tile_nent(const TileDesc *__restrict__ tiles, int ntiles, const unsigned *__restrict__ W,
                            int *__restrict__ nent, int *__restrict__ mx)
{
    const int lane = lane_id(), wpb = blockDim.x >> 5;
    int mt = 0, me = 0;
    for (long long t = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); t < ntiles; t += (long long)gridDim.x * wpb)
    {
        const TileDesc D = tiles[t];
        int e = -1;
        for (int u = lane; u < D.nterms; u += 32) e = max(e, (int)(W[D.word_begin + u] >> 14));
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) e = max(e, __shfl_xor_sync(FULL_MASK, e, o));
        if (lane == 0) nent[t] = e + 1;
        mt = max(mt, D.nterms);
        me = max(me, e + 1);
    }
    if (lane == 0)
    {
        atomicMax(&mx[0], mt);
        atomicMax(&mx[1], me);
    }
}

// Everything the refill needs once C's structure is known: row classes, the
// compiled tile schedule and the larger rows' scratch.
void build_schedule(const ProductDesc &d, Product &P, const long long *ub, cudaStream_t s)
{
    NvtxRange nvtx_range_("sdl: refill plan");
    Runtime &rt = runtime();
    const int m_out = P.m_out;
    DevBuf<long long> weight(m_out), wpref((size_t)m_out + 1);
    DevBuf<unsigned char> rcls(m_out);
    // rows with more terms than tile_max leave the tiles for the larger-row kernels
    const int tile_max = P.cfg.tile_max_terms > 0 ? std::min(TILE_T, P.cfg.tile_max_terms) : TILE_T;
    SDL_LAUNCH(k_num_classify, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, ub, P.Cp.get(), d.Lp, d.L_m,
               m_out, tile_max, rcls.get(), weight.get());
    bin_items(rcls.get(), m_out, NUM_NBINS, P.num_rows, P.num_count, P.num_offset, s);
    exclusive_scan_i64(weight.get(), wpref.get(), m_out, s);
    DevBuf<int> flag(m_out), tile_of((size_t)m_out + 1);
    const int budget = P.cfg.tile_budget > 0 ? std::max(TILE_T / 8, std::min(TILE_T, P.cfg.tile_budget)) : TILE_T;
    SDL_LAUNCH(k_tile_flags, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, wpref.get(), m_out, budget,
               flag.get());
    P.ntiles = exclusive_scan_i32_checked(flag.get(), tile_of.get(), m_out, s);
    DevBuf<int> tile_start((size_t)P.ntiles + 1);
    SDL_LAUNCH(k_tile_starts, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, flag.get(),
               tile_of.get(), m_out, tile_start.get());
    SDL_CUDA(cudaMemcpyAsync(tile_start.get() + P.ntiles, &P.m_out, sizeof(int), cudaMemcpyHostToDevice, s));
    const int nt = std::max(1, P.ntiles);
    const long long nV = (long long)d.L_nnz * d.blocks;
    if (nV > INT_MAX || d.A_nnz < 0)
        fail(SDL_ERR_OVERFLOW, "product: blocks * entries of L exceeds the schedule's 31-bit entry index");
    // entry values in L's value order when L_map is a permutation of [0, L_nnz)
    // (the refill then reads L.x in order); kv gives each value's row of A
    int value_order = 0;
    P.kv.release();
    if (d.L_map && d.L_nnz > 0)
    {
        DevBuf<int> cnt(d.L_nnz), bad(1);
        P.kv.reset(d.L_nnz);
        SDL_CUDA(cudaMemsetAsync(cnt.get(), 0, cnt.bytes(), s));
        SDL_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(int), s));
        SDL_LAUNCH(k_value_rows, grid_for(d.L_nnz, 256, rt.num_sms * 8), 256, 0, s, d.L_map, d.Li, d.L_nnz,
                   P.kv.get(), cnt.get(), bad.get());
        int hbad = 1;
        SDL_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        SDL_CUDA(cudaStreamSynchronize(s));
        if (hbad)
            P.kv.release();
        else
            value_order = 1;
    }
    DevBuf<long long> tile_nterms(nt), tile_nx(nt), word_begin((size_t)nt + 1), x_begin((size_t)nt + 1);
    NumArgs na{d.Lp, d.Li, d.L_map, d.L_m, P.n_L, nullptr, nullptr, d.Ap, d.Ai, nullptr,
               P.Cp.get(), P.Ci.get(), nullptr, rt.d_error, d.L_nnz, value_order};
    set_smem(k_tile_schedule<false>, build_smem_bytes());
    set_smem(k_tile_schedule<true>, build_smem_bytes());
    SDL_LAUNCH(k_tile_schedule<false>, P.ntiles, TILE_THREADS, build_smem_bytes(), s, na, rcls.get(),
               tile_start.get(), tile_nterms.get(), tile_nx.get(), nullptr, nullptr, nullptr, nullptr,
               nullptr, nullptr);
    const long long word_total = exclusive_scan_i64(tile_nterms.get(), word_begin.get(), P.ntiles, s);
    const long long x_total = exclusive_scan_i64(tile_nx.get(), x_begin.get(), P.ntiles, s);
    if (word_total > INT_MAX || x_total > INT_MAX)
        fail(SDL_ERR_OVERFLOW, "product: the tile rows' terms exceed the schedule's 31-bit offsets");
    P.tiles.reset(nt);
    // W and ES carry 16 bytes past their ends: the staged refill's bulk copies round
    // a tile's runs out to 16-byte boundaries
    P.W.reset(std::max<long long>(1, word_total) + 4);
    P.X.reset(std::max<long long>(1, x_total));
    P.V.reset(std::max<long long>(1, nV));
    P.ES.reset(std::max<long long>(1, nV) + 2);
    SDL_LAUNCH(k_tile_schedule<true>, P.ntiles, TILE_THREADS, build_smem_bytes(), s, na, rcls.get(),
               tile_start.get(), nullptr, nullptr, word_begin.get(), x_begin.get(), P.tiles.get(),
               P.W.get(), P.X.get(), P.ES.get());
    if (take_device_error(s)) fail(SDL_ERR_INTERNAL, "product plan: a term column is missing from its row");
    if (P.ntiles > 0)
    {
        SDL_LAUNCH(k_validate_schedule, grid_for(P.ntiles, 1, rt.num_sms * 8), 256, 0, s, P.tiles.get(), P.ntiles,
                   P.W.get(), word_total, P.X.get(), x_total, P.ES.get(), nV, (long long)d.A_nnz,
                   (long long)P.nnz, rt.d_error);
        if (take_device_error(s)) fail(SDL_ERR_INTERNAL, "product plan: the refill schedule failed its bounds check");
        DevBuf<int> mo(1);
        SDL_CUDA(cudaMemsetAsync(mo.get(), 0, sizeof(int), s));
        SDL_LAUNCH(k_tile_max_out, grid_for(P.ntiles, 256, rt.num_sms * 4), 256, 0, s, P.tiles.get(), P.ntiles,
                   mo.get());
        SDL_CUDA(cudaMemcpyAsync(&P.max_tile_out, mo.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        P.tile_nent.reset((size_t)P.ntiles);
        DevBuf<int> mx(2);
        SDL_CUDA(cudaMemsetAsync(mx.get(), 0, mx.bytes(), s));
        SDL_LAUNCH(k_tile_nent, grid_for(P.ntiles, 8, rt.num_sms * 8), 256, 0, s, P.tiles.get(), P.ntiles, P.W.get(),
                   P.tile_nent.get(), mx.get());
        int hmx[2] = {0, 0};
        SDL_CUDA(cudaMemcpyAsync(hmx, mx.get(), sizeof(hmx), cudaMemcpyDeviceToHost, s));
        SDL_CUDA(cudaStreamSynchronize(s));
        P.max_tile_terms = hmx[0];
        P.max_tile_ent = hmx[1];
    }
    build_big_lists(d, P, ub, na, s);
    if (P.num_count[NUM_GMEM] && !P.big_lists)
    {
        long long per_slot = std::max(1, P.n);
        long long max_slots = std::max<long long>(1, (2LL << 30) / (per_slot * 4));
        P.gmem_slots = (int)std::min<long long>({(long long)rt.num_sms * GMEM_CTAS_PER_SM, max_slots,
                                                 (long long)P.num_count[NUM_GMEM]});
        P.gmem_scratch.reset((size_t)P.gmem_slots * per_slot);
    }
}

// Learned row statistics: term count, and from the network the row's capacity
// (predicted nnz with a margin, never above the term count) and predicted class.
__global__ void k_row_terms_learned(const int *__restrict__ Lp, const int *__restrict__ Li, int L_m,
                                    int n_L, int m_out, const int *__restrict__ Ap, int n,
                                    const float *__restrict__ P, float margin, long long *__restrict__ ub,
                                    long long *__restrict__ cap, unsigned char *__restrict__ pcls)
{
    __shared__ float sp[MLP_NPARAMS];
    for (int q = threadIdx.x; q < MLP_NPARAMS; q += blockDim.x) sp[q] = P[q];
    __syncthreads();
    const int lane = lane_id(), wpb = blockDim.x >> 5;
    for (long long row = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); row < m_out;
         row += (long long)gridDim.x * wpb)
    {
        int b = (int)(row / L_m), r = (int)(row - (long long)b * L_m);
        long long sum = 0;
        int mx = 0;
        for (int ii = Lp[r] + lane; ii < Lp[r + 1]; ii += 32)
        {
            int k = Li[ii] + b * n_L;
            int len = Ap[k + 1] - Ap[k];
            sum += len;
            mx = max(mx, len);
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1)
        {
            sum += __shfl_xor_sync(FULL_MASK, sum, o);
            mx = max(mx, __shfl_xor_sync(FULL_MASK, mx, o));
        }
        float f[MLP_IN];
        {
            float lu = log1pf((float)sum), lm = log1pf((float)mx), ln = log1pf((float)n);
            f[0] = log1pf((float)(Lp[r + 1] - Lp[r]));
            f[1] = lu;
            f[2] = lm;
            f[3] = ln;
            f[4] = fminf(4.f, (float)sum / (float)max(1, n));
            f[5] = lu - lm;
            f[6] = lu - ln;
            f[7] = 1.f;
        }
        float mine = 0.f;
#pragma unroll
        for (int q = 0; q < MLP_IN; ++q)
            if (lane == q) mine = f[q];
        float y = mlp_row_forward(sp, mine);
        float y1 = __shfl_sync(FULL_MASK, y, 1), y2 = __shfl_sync(FULL_MASK, y, 2),
              y3 = __shfl_sync(FULL_MASK, y, 3);
        if (lane == 0)
        {
            ub[row] = sum;
            double pred = expm1((double)fminf(y, 40.f));
            long long c = (long long)ceil(fmax(0.0, pred) * (1.0 + margin)) + 8;
            cap[row] = c < sum ? c : sum;
            pcls[row] = (unsigned char)(y1 >= y2 && y1 >= y3 ? 0 : (y2 >= y3 ? 1 : 2));
        }
    }
}

__global__ void k_overflow_terms(const unsigned char *__restrict__ overflow, const long long *__restrict__ ub,
                                 int m_out, long long *__restrict__ fb_len)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
        fb_len[r] = overflow[r] ? ub[r] : 0;
}

__global__ void k_class_hits(const unsigned char *__restrict__ pcls, const int *__restrict__ Cp, int m_out,
                             unsigned long long *__restrict__ hits)
{
    unsigned long long h = 0;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
        h += pcls[r] == mlp_class_of(Cp[r + 1] - Cp[r]) ? 1 : 0;
    atomicAdd(hits, h);
}

} // namespace

void product_symbolic(const ProductDesc &d, const TuneConfig &cfg, Product &P, cudaStream_t s,
                      bool keep_row_terms)
{
    NvtxRange nvtx_range_("sdl: symbolic pass");
    Runtime &rt = runtime();
    validate_product(d, cfg, P, s);
    const int m_out = P.m_out;
    P.Cp.reset((size_t)m_out + 1);
    DevBuf<long long> ub(std::max(1, m_out)), ub_off((size_t)m_out + 1);
    if (m_out == 0)
    {
        SDL_CUDA(cudaMemsetAsync(P.Cp.get(), 0, sizeof(int), s));
        P.nnz = 0;
        P.terms = 0;
        SDL_CUDA(cudaStreamSynchronize(s));
        return;
    }
    SDL_LAUNCH(k_row_terms, grid_for(m_out, 8, rt.num_sms * 16), 256, 0, s, d.Lp, d.Li, d.L_m,
               P.n_L, m_out, d.Ap, ub.get());
    P.terms = exclusive_scan_i64(ub.get(), ub_off.get(), m_out, s);

    DevBuf<int> row_nnz(m_out);
    SDL_CUDA(cudaMemsetAsync(row_nnz.get(), 0, row_nnz.bytes(), s));
    DevBuf<int> tmp(std::max<long long>(1, P.terms));
    DevBuf<unsigned char> cls(m_out);
    SDL_LAUNCH(k_sym_classify, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, ub.get(), m_out,
               cfg.warp_max_terms, cls.get());
    DevBuf<int> lists;
    int cnt[SYM_NBINS], off[SYM_NBINS + 1];
    bin_items(cls.get(), m_out, SYM_NBINS, lists, cnt, off, s);
    SymArgs sa{d.Lp, d.Li, d.L_m, P.n_L, d.A_n, d.Ap, d.Ai, ub_off.get(), tmp.get(), row_nnz.get(),
               nullptr, nullptr};
    sym_launch(sa, lists.get(), cnt, off, d, cfg, s);

    P.nnz = exclusive_scan_i32_checked(row_nnz.get(), P.Cp.get(), m_out, s);
    P.Ci.reset(std::max(1, P.nnz));
    if (P.nnz > 0)
        compact_rows(P.Cp.get(), m_out, P.nnz, ub_off.get(), nullptr, nullptr, nullptr, tmp.get(), nullptr, nullptr,
                     nullptr, P.Ci.get(), nullptr, s);
    P.scratch_bytes = (long long)tmp.bytes();
    build_schedule(d, P, ub.get(), s);
    if (keep_row_terms) P.row_terms = std::move(ub);
    SDL_CUDA(cudaStreamSynchronize(s));
}

void product_symbolic_learned(const ProductDesc &d, const TuneConfig &cfg, const Mlp &net, float margin,
                              Product &P, LearnedStats &st, cudaStream_t s)
{
    NvtxRange nvtx_range_("sdl: learned symbolic pass");
    Runtime &rt = runtime();
    validate_product(d, cfg, P, s);
    const int m_out = P.m_out;
    st = LearnedStats{};
    P.Cp.reset((size_t)m_out + 1);
    if (m_out == 0)
    {
        SDL_CUDA(cudaMemsetAsync(P.Cp.get(), 0, sizeof(int), s));
        P.nnz = 0;
        P.terms = 0;
        SDL_CUDA(cudaStreamSynchronize(s));
        return;
    }
    DevBuf<long long> ub(m_out), cap(m_out), cap_off((size_t)m_out + 1), ub_off((size_t)m_out + 1);
    DevBuf<unsigned char> pcls(m_out), overflow(m_out);
    SDL_LAUNCH(k_row_terms_learned, grid_for(m_out, 8, rt.num_sms * 16), 256, 0, s, d.Lp, d.Li, d.L_m,
               P.n_L, m_out, d.Ap, d.A_n, net.params.get(), margin, ub.get(), cap.get(), pcls.get());
    P.terms = exclusive_scan_i64(ub.get(), ub_off.get(), m_out, s);
    st.cap_total = exclusive_scan_i64(cap.get(), cap_off.get(), m_out, s);
    st.ub_total = P.terms;

    DevBuf<int> row_nnz(m_out);
    SDL_CUDA(cudaMemsetAsync(row_nnz.get(), 0, row_nnz.bytes(), s));
    SDL_CUDA(cudaMemsetAsync(overflow.get(), 0, overflow.bytes(), s));
    DevBuf<int> tmp(std::max<long long>(1, st.cap_total));
    DevBuf<unsigned char> cls(m_out);
    SDL_LAUNCH(k_sym_classify, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, ub.get(), m_out,
               cfg.warp_max_terms, cls.get());
    DevBuf<int> lists;
    int cnt[SYM_NBINS], off[SYM_NBINS + 1];
    bin_items(cls.get(), m_out, SYM_NBINS, lists, cnt, off, s);
    SymArgs sa{d.Lp, d.Li, d.L_m, P.n_L, d.A_n, d.Ap, d.Ai, cap_off.get(), tmp.get(), row_nnz.get(),
               cap.get(), overflow.get()};
    sym_launch(sa, lists.get(), cnt, off, d, cfg, s);

    // rows whose columns did not fit: the exact pass again, into term-count space
    DevBuf<long long> fb_len(m_out), fb_off((size_t)m_out + 1);
    SDL_LAUNCH(k_overflow_terms, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, overflow.get(), ub.get(),
               m_out, fb_len.get());
    st.fallback_terms = exclusive_scan_i64(fb_len.get(), fb_off.get(), m_out, s);
    DevBuf<int> fb(std::max<long long>(1, st.fallback_terms));
    if (st.fallback_terms > 0)
    {
        // classes of the overflowing rows only
        DevBuf<unsigned char> fcls(m_out);
        SDL_CUDA(cudaMemcpyAsync(fcls.get(), cls.get(), m_out, cudaMemcpyDeviceToDevice, s));
        SDL_LAUNCH(k_mask_classes, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, overflow.get(), m_out,
                   fcls.get());
        DevBuf<int> flists;
        int fcnt[SYM_NBINS], foff[SYM_NBINS + 1];
        bin_items(fcls.get(), m_out, SYM_NBINS, flists, fcnt, foff, s);
        for (int c = 0; c < SYM_NBINS; ++c) st.fallback_rows += fcnt[c];
        SymArgs fa{d.Lp, d.Li, d.L_m, P.n_L, d.A_n, d.Ap, d.Ai, fb_off.get(), fb.get(), row_nnz.get(),
                   nullptr, nullptr};
        sym_launch(fa, flists.get(), fcnt, foff, d, cfg, s);
    }
    P.nnz = exclusive_scan_i32_checked(row_nnz.get(), P.Cp.get(), m_out, s);
    P.Ci.reset(std::max(1, P.nnz));
    if (P.nnz > 0)
        compact_rows(P.Cp.get(), m_out, P.nnz, cap_off.get(), fb_off.get(), overflow.get(), nullptr, tmp.get(),
                     fb.get(), nullptr, nullptr, P.Ci.get(), nullptr, s);
    {
        DevBuf<unsigned long long> hits(1);
        SDL_CUDA(cudaMemsetAsync(hits.get(), 0, 8, s));
        SDL_LAUNCH(k_class_hits, grid_for(m_out, 256, rt.num_sms * 4), 256, 0, s, pcls.get(), P.Cp.get(),
                   m_out, hits.get());
        unsigned long long h = 0;
        SDL_CUDA(cudaMemcpyAsync(&h, hits.get(), 8, cudaMemcpyDeviceToHost, s));
        SDL_CUDA(cudaStreamSynchronize(s));
        st.class_hits = (long long)h;
        st.rows = m_out;
    }
    P.scratch_bytes = (long long)tmp.bytes() + (long long)fb.bytes();
    build_schedule(d, P, ub.get(), s);
    SDL_CUDA(cudaStreamSynchronize(s));
}

namespace {
// Launches the one-shot kernel of every row class up to 8192 terms.
void oneshot_launch(const OneShotArgs &oa, const int *lists, const int *cnt, const int *off, const TuneConfig &cfg,
                    cudaStream_t s)
{
    Runtime &rt = runtime();
    const int gcap = rt.num_sms * 16;
    const int wpb = std::max(1, std::min(8, cfg.rows_per_cta_warp));
    if (cnt[SYM_W32])
    {
        const size_t sm = (size_t)wpb * 2 * 32 * 8;
        SDL_LAUNCH(k_oneshot_warp<32>, grid_for(cnt[SYM_W32], wpb, gcap), wpb * 32, sm, s, lists + off[SYM_W32],
                   cnt[SYM_W32], oa);
    }
    if (cnt[SYM_W128])
    {
        const size_t sm = (size_t)wpb * 2 * 128 * 8;
        SDL_LAUNCH(k_oneshot_warp<128>, grid_for(cnt[SYM_W128], wpb, gcap), wpb * 32, sm, s, lists + off[SYM_W128],
                   cnt[SYM_W128], oa);
    }
    if (cnt[SYM_W512])
    {
        const size_t sm = (size_t)wpb * 2 * 512 * 8;
        set_smem(k_oneshot_warp<512>, sm);
        SDL_LAUNCH(k_oneshot_warp<512>, grid_for(cnt[SYM_W512], wpb, gcap), wpb * 32, sm, s, lists + off[SYM_W512],
                   cnt[SYM_W512], oa);
    }
    if (cnt[SYM_C2K])
    {
        const int th = 256;
        const size_t sm = 2048 * 16 + (size_t)th * 8 + (3 * th + 32) * 4;
        set_smem(k_oneshot_cta<2048>, sm);
        SDL_LAUNCH(k_oneshot_cta<2048>, grid_for(cnt[SYM_C2K], 1, gcap), th, sm, s, lists + off[SYM_C2K],
                   cnt[SYM_C2K], oa);
    }
    if (cnt[SYM_C8K])
    {
        const int th = 512;
        const size_t sm = 8192 * 16 + (size_t)th * 8 + (3 * th + 32) * 4;
        set_smem(k_oneshot_cta<8192>, sm);
        SDL_LAUNCH(k_oneshot_cta<8192>, grid_for(cnt[SYM_C8K], 1, gcap), th, sm, s, lists + off[SYM_C8K],
                   cnt[SYM_C8K], oa);
    }
}
} // namespace

namespace {
// Term counts of the listed rows.
__global__ void k_gather_row_terms(const int *__restrict__ rows, int n, const long long *__restrict__ terms,
                                   long long *__restrict__ out)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) out[q] = terms[rows[q]];
}
} // namespace

void product_oneshot_learned(const ProductDesc &d, const TuneConfig &cfg, const Mlp &net, float margin,
                             const double *Lx, const double *dvec, const double *Ax, Product &P,
                             DevBuf<double> &Cx, LearnedStats &st, cudaStream_t s)
{
    NvtxRange nvtx_range_("sdl: learned one-shot pass");
    Runtime &rt = runtime();
    validate_product(d, cfg, P, s);
    const int m_out = P.m_out;
    st = LearnedStats{};
    P.Cp.reset((size_t)m_out + 1);
    P.plan_ready = false;
    if (m_out == 0)
    {
        SDL_CUDA(cudaMemsetAsync(P.Cp.get(), 0, sizeof(int), s));
        P.nnz = 0;
        P.terms = 0;
        P.Ci.reset(1);
        Cx.reset(1);
        P.row_terms.reset(1);
        SDL_CUDA(cudaStreamSynchronize(s));
        return;
    }
    if (d.A_nnz > 0 && !Ax) fail(SDL_ERR_INVALID, "one-shot product: NULL A values");
    DevBuf<long long> ub(m_out), cap(m_out), cap_off((size_t)m_out + 1), ub_off((size_t)m_out + 1);
    DevBuf<unsigned char> pcls(m_out), overflow(m_out), cls(m_out);
    SDL_LAUNCH(k_row_terms_learned, grid_for(m_out, 8, rt.num_sms * 16), 256, 0, s, d.Lp, d.Li, d.L_m,
               P.n_L, m_out, d.Ap, d.A_n, net.params.get(), margin, ub.get(), cap.get(), pcls.get());
    P.terms = exclusive_scan_i64(ub.get(), ub_off.get(), m_out, s);
    st.cap_total = exclusive_scan_i64(cap.get(), cap_off.get(), m_out, s);
    st.ub_total = P.terms;
    DevBuf<int> row_nnz(m_out);
    SDL_CUDA(cudaMemsetAsync(row_nnz.get(), 0, row_nnz.bytes(), s));
    SDL_CUDA(cudaMemsetAsync(overflow.get(), 0, overflow.bytes(), s));
    DevBuf<int> tcol(std::max<long long>(1, st.cap_total));
    DevBuf<double> tval(std::max<long long>(1, st.cap_total));
    SDL_LAUNCH(k_sym_classify, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, ub.get(), m_out, cfg.warp_max_terms,
               cls.get());
    DevBuf<int> lists;
    int cnt[SYM_NBINS], off[SYM_NBINS + 1];
    bin_items(cls.get(), m_out, SYM_NBINS, lists, cnt, off, s);
    // rows up to 8192 terms: structure and values in one pass
    OneShotArgs oa{d.Lp, d.Li, d.L_map, d.L_m, P.n_L, Lx, dvec, d.Ap, d.Ai, Ax, cap_off.get(), cap.get(),
                   tcol.get(), tval.get(), row_nnz.get(), overflow.get()};
    oneshot_launch(oa, lists.get(), cnt, off, cfg, s);
    // larger rows: their columns by the bitmap pass (values once C is laid out)
    int bcnt[SYM_NBINS] = {0};
    bcnt[SYM_BITMAP] = cnt[SYM_BITMAP];
    if (bcnt[SYM_BITMAP])
    {
        SymArgs sa{d.Lp, d.Li, d.L_m, P.n_L, d.A_n, d.Ap, d.Ai, cap_off.get(), tcol.get(), row_nnz.get(),
                   cap.get(), overflow.get()};
        sym_launch(sa, lists.get(), bcnt, off, d, cfg, s);
    }
    // rows whose outputs did not fit their capacity: the same passes again,
    // unbounded, into term-count space
    DevBuf<long long> fb_len(m_out), fb_off((size_t)m_out + 1);
    SDL_LAUNCH(k_overflow_terms, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, overflow.get(), ub.get(), m_out,
               fb_len.get());
    st.fallback_terms = exclusive_scan_i64(fb_len.get(), fb_off.get(), m_out, s);
    DevBuf<int> fcol(std::max<long long>(1, st.fallback_terms));
    DevBuf<double> fval(std::max<long long>(1, st.fallback_terms));
    if (st.fallback_terms > 0)
    {
        DevBuf<unsigned char> fcls(m_out);
        SDL_CUDA(cudaMemcpyAsync(fcls.get(), cls.get(), m_out, cudaMemcpyDeviceToDevice, s));
        SDL_LAUNCH(k_mask_classes, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, overflow.get(), m_out,
                   fcls.get());
        DevBuf<int> flists;
        int fcnt[SYM_NBINS], foff[SYM_NBINS + 1];
        bin_items(fcls.get(), m_out, SYM_NBINS, flists, fcnt, foff, s);
        for (int c = 0; c < SYM_NBINS; ++c) st.fallback_rows += fcnt[c];
        OneShotArgs fa{d.Lp, d.Li, d.L_map, d.L_m, P.n_L, Lx, dvec, d.Ap, d.Ai, Ax, fb_off.get(), nullptr,
                       fcol.get(), fval.get(), row_nnz.get(), nullptr};
        oneshot_launch(fa, flists.get(), fcnt, foff, cfg, s);
        int fb_bits[SYM_NBINS] = {0};
        fb_bits[SYM_BITMAP] = fcnt[SYM_BITMAP];
        if (fb_bits[SYM_BITMAP])
        {
            SymArgs sb{d.Lp, d.Li, d.L_m, P.n_L, d.A_n, d.Ap, d.Ai, fb_off.get(), fcol.get(), row_nnz.get(),
                       nullptr, nullptr};
            sym_launch(sb, flists.get(), fb_bits, foff, d, cfg, s);
        }
    }
    P.nnz = exclusive_scan_i32_checked(row_nnz.get(), P.Cp.get(), m_out, s);
    P.Ci.reset(std::max(1, P.nnz));
    Cx.reset(std::max(1, P.nnz));
    // rows whose values come after the compaction (the large rows)
    DevBuf<unsigned char> late(m_out);
    SDL_LAUNCH(k_mark_class, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, cls.get(), m_out, (int)SYM_BITMAP,
               late.get());
    if (P.nnz > 0)
        compact_rows(P.Cp.get(), m_out, P.nnz, cap_off.get(), fb_off.get(), overflow.get(), late.get(), tcol.get(),
                     fcol.get(), tval.get(), fval.get(), P.Ci.get(), Cx.get(), s);
    // values of the larger rows: accumulated in C.x through a per-CTA column ->
    // position map, same-position terms applied in visiting order
    if (cnt[SYM_BITMAP] && P.nnz > 0)
    {
        // rank maps: per CTA one 16-byte entry (4 ints) per 64 columns
        const long long per_slot = 4LL * ((std::max(1, P.n) + 63) / 64);
        const long long max_slots = std::max<long long>(1, (2LL << 30) / (per_slot * 4));
        const int slots = (int)std::min<long long>(
            {(long long)rt.num_sms * GMEM_CTAS_PER_SM, max_slots, (long long)cnt[SYM_BITMAP]});
        // the maps need no clearing (a row reads only the entries it wrote): the
        // one-shot rows' column scratch, dead once compacted into C, holds them when
        // it is large enough
        DevBuf<int> posmap_own;
        int *posmap = tcol.get();
        if (tcol.n < (size_t)slots * per_slot)
        {
            posmap_own.reset((size_t)slots * per_slot);
            posmap = posmap_own.get();
        }
        NumArgs na{d.Lp, d.Li, d.L_map, d.L_m, P.n_L, Lx, dvec, d.Ap, d.Ai, Ax, P.Cp.get(), P.Ci.get(), Cx.get(),
                   rt.d_error};
        // the large rows by term count, largest first, handed out by a counter: the
        // largest rows start first and no CTA is left with several of them (only the
        // large rows' counts come to the host)
        const int nbr = cnt[SYM_BITMAP];
        std::vector<int> hrows(nbr);
        std::vector<long long> hub(nbr);
        {
            DevBuf<long long> big_terms((size_t)nbr);
            SDL_LAUNCH(k_gather_row_terms, grid_for(nbr, 256, rt.num_sms * 4), 256, 0, s,
                       lists.get() + off[SYM_BITMAP], nbr, P.row_terms.get() ? P.row_terms.get() : ub.get(),
                       big_terms.get());
            SDL_CUDA(cudaMemcpyAsync(hrows.data(), lists.get() + off[SYM_BITMAP], (size_t)nbr * sizeof(int),
                                     cudaMemcpyDeviceToHost, s));
            SDL_CUDA(cudaMemcpyAsync(hub.data(), big_terms.get(), (size_t)nbr * sizeof(long long),
                                     cudaMemcpyDeviceToHost, s));
            SDL_CUDA(cudaStreamSynchronize(s));
        }
        std::vector<int> idx(nbr);
        for (int q = 0; q < nbr; ++q) idx[q] = q;
        std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return hub[x] > hub[y]; });
        {
            std::vector<int> sorted(nbr);
            for (int q = 0; q < nbr; ++q) sorted[q] = hrows[idx[q]];
            hrows.swap(sorted);
        }
        DevBuf<int> order((size_t)nbr), counter(1);
        SDL_CUDA(cudaMemcpyAsync(order.get(), hrows.data(), (size_t)nbr * sizeof(int), cudaMemcpyHostToDevice, s));
        SDL_CUDA(cudaMemsetAsync(counter.get(), 0, sizeof(int), s));
        const size_t sm = gmem_smem_bytes();
        set_smem(k_num_gmem<true>, sm);
        SDL_LAUNCH(k_num_gmem<true>, slots, GMEM_THREADS, sm, s, order.get(), nbr, na, posmap, P.n, nullptr,
                   counter.get());
        SDL_CUDA(cudaStreamSynchronize(s)); // hrows / hub and the queue are freed on return
        if (take_device_error(s)) fail(SDL_ERR_INTERNAL, "one-shot product: a term column is missing from its row");
    }
    {
        DevBuf<unsigned long long> hits(1);
        SDL_CUDA(cudaMemsetAsync(hits.get(), 0, 8, s));
        SDL_LAUNCH(k_class_hits, grid_for(m_out, 256, rt.num_sms * 4), 256, 0, s, pcls.get(), P.Cp.get(), m_out,
                   hits.get());
        unsigned long long h = 0;
        SDL_CUDA(cudaMemcpyAsync(&h, hits.get(), 8, cudaMemcpyDeviceToHost, s));
        SDL_CUDA(cudaStreamSynchronize(s));
        st.class_hits = (long long)h;
        st.rows = m_out;
    }
    P.scratch_bytes = (long long)(tcol.bytes() + tval.bytes() + fcol.bytes() + fval.bytes());
    P.row_terms = std::move(ub);
    SDL_CUDA(cudaStreamSynchronize(s));
}

void product_complete_plan(Product &P, cudaStream_t s)
{
    if (P.plan_ready) return;
    if (P.m_out > 0) build_schedule(P.desc, P, P.row_terms.get(), s);
    SDL_CUDA(cudaStreamSynchronize(s));
    P.plan_ready = true;
}

namespace {
__global__ void k_rebase_tiles(const TileDesc *__restrict__ src, int n, int prod, TileDesc *__restrict__ dst)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
    {
        TileDesc d = src[t];
        d.prod = prod;
        dst[t] = d;
    }
}
} // namespace

ProdSched sched_of(const Product &P)
{
    const ProductDesc &d = P.desc;
    ProdSched S{};
    S.W = P.W.get();
    S.X = P.X.get();
    S.V = P.V.get();
    S.ES = P.ES.get();
    S.kv = P.kv.get();
    S.Li = d.Li;
    S.L_map = d.L_map;
    S.nV = (long long)d.L_nnz * d.blocks;
    S.nA = d.A_nnz;
    S.L_nnz = d.L_nnz;
    S.n_L = P.n_L;
    S.blocks = d.blocks;
    return S;
}

void entry_values(const ProdSched &S, const ProdPtrs &vals, cudaStream_t s)
{
    if (S.nV <= 0 || (!vals.Lx && !vals.d)) return; // unit product: every value is 1.0
    SDL_LAUNCH(k_entry_values, grid_for(S.nV, 256 * EV_ILP, runtime().num_sms * 8), 256, 0, s, S, vals);
}

void entry_values_batched(const EntChunk *chunks, int nchunks, const ProdPtrs *ptrs, const ProdSched *scheds,
                          cudaStream_t s)
{
    if (nchunks <= 0) return;
    SDL_LAUNCH(k_entry_values_batched, nchunks, 256, 0, s, chunks, ptrs, scheds);
}

void append_entry_chunks(long long nV, int prod, int chunk, std::vector<EntChunk> &out)
{
    for (long long b = 0; b < nV; b += chunk)
        out.push_back(EntChunk{b, (int)std::min<long long>(chunk, nV - b), prod});
}

void rebase_tiles(const TileDesc *src, int n, int prod, TileDesc *dst, cudaStream_t s)
{
    if (n <= 0) return;
    SDL_LAUNCH(k_rebase_tiles, grid_for(n, 256, runtime().num_sms * 4), 256, 0, s, src, n, prod, dst);
}

namespace {
// Resident refill CTAs per SM of one kernel instance (its attributes are set on the
// first call, which is an eager one).
template <bool BATCHED, int NT, bool ESS>
int refill_per_sm(size_t smem)
{
    // resident CTAs per SM for each (device, shared-memory size) met; the kernel's
    // shared-memory attribute is set on each device the first time
    static std::map<std::pair<int, size_t>, int> cache;
    static std::mutex mu;
    // the last answer of this thread, without the lock (launches repeat the same key)
    thread_local int last_dev = -1, last_val = 0;
    thread_local size_t last_smem = 0;
    int dev = 0;
    SDL_CUDA(cudaGetDevice(&dev));
    if (dev == last_dev && smem == last_smem) return last_val;
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find({dev, smem});
    if (it != cache.end())
    {
        last_dev = dev;
        last_smem = smem;
        last_val = it->second;
        return last_val;
    }
    if (ESS)
        SDL_CUDA(cudaFuncSetAttribute(k_tile_refill<BATCHED, NT, ESS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)STAGED_SMEM_MAX));
    else
        set_smem(k_tile_refill<BATCHED, NT, ESS>, smem);
    int n = 0;
    SDL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tile_refill<BATCHED, NT, ESS>, NT, smem));
    const int per_sm = std::max(1, n);
    cache[{dev, smem}] = per_sm;
    last_dev = dev;
    last_smem = smem;
    last_val = per_sm;
    return per_sm;
}

template <bool BATCHED, int NT, bool ESS = false>
void launch_refill(const TileDesc *tiles, int ntiles, const ProdPtrs *ptrs, const ProdSched *scheds,
                   cudaStream_t s, const ProdPtrs &vals, const ProdSched &sched, int ctas_per_sm,
                   const int *tile_nent = nullptr, int wcap = 0, int ecap = 0)
{
    const size_t smem = ESS ? staged_smem_bytes(NT, wcap, ecap) : refill_smem_bytes<NT>();
    const int per_sm = refill_per_sm<BATCHED, NT, ESS>(smem);
    const int use = ctas_per_sm > 0 ? std::min(ctas_per_sm, per_sm) : per_sm;
    const int grid = std::min(ntiles, runtime().num_sms * use);
    if (BATCHED)
    {
        SDL_LAUNCH((k_tile_refill<BATCHED, NT, ESS>), grid, NT, smem, s, tiles, ntiles, ptrs, scheds, vals, sched,
                   runtime().d_error, tile_nent, wcap, ecap);
        return;
    }
    // programmatic dependent launch: the CTAs start while the entry-value kernel
    // ahead of it on the stream drains (the kernel waits before reading V)
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SDL_CUDA(cudaLaunchKernelEx(&cfg, k_tile_refill<BATCHED, NT, ESS>, tiles, ntiles, ptrs, scheds, vals, sched,
                                runtime().d_error, tile_nent, wcap, ecap));
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

} // namespace

bool small_tile_refill(const Product &P)
{
    return P.cfg.refill_threads == REFILL_THREADS_SMALL && P.max_tile_out <= win_of<REFILL_THREADS_SMALL>();
}

// Slot capacities of the staged refill for P's tiles: the largest tile's words and
// records, each rounded up to a 16-byte multiple plus the 16 bytes a run's rounded
// start can add.
void staged_caps(const Product &P, int &wcap, int &ecap)
{
    wcap = ((P.max_tile_terms + 3) & ~3) + 4;
    ecap = ((P.max_tile_ent + 1) & ~1) + 2;
}

bool es_refill(const Product &P)
{
    if (!P.cfg.refill_es || P.ntiles <= 0 || !P.tile_nent.get() || pipe_refill(P)) return false;
    int wcap = 0, ecap = 0;
    staged_caps(P, wcap, ecap);
    const int nt = small_tile_refill(P) ? REFILL_THREADS_SMALL : REFILL_THREADS;
    return staged_smem_bytes(nt, wcap, ecap) <= STAGED_SMEM_MAX;
}

bool pipe_refill(const Product &P)
{
    return P.cfg.refill_pipe && P.ntiles > 0 && P.max_tile_terms <= PIPE_T && P.max_tile_ent <= PIPE_E &&
           P.max_tile_out <= PIPE_WIN;
}

void launch_refill_pipe(const Product &P, cudaStream_t s, const ProdPtrs &vals, const ProdSched &sched)
{
    static int per_sm = 0;
    if (!per_sm)
    {
        set_smem(k_tile_refill_pipe, pipe_smem_bytes());
        int n = 0;
        SDL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tile_refill_pipe, PIPE_NT, pipe_smem_bytes()));
        per_sm = std::max(1, n);
    }
    const int use = P.cfg.refill_ctas_per_sm > 0 ? std::min(P.cfg.refill_ctas_per_sm, per_sm) : per_sm;
    const int grid = std::min(P.ntiles, runtime().num_sms * use);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(PIPE_NT);
    cfg.dynamicSmemBytes = pipe_smem_bytes();
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SDL_CUDA(cudaLaunchKernelEx(&cfg, k_tile_refill_pipe, (const TileDesc *)P.tiles.get(), P.ntiles,
                                (const int *)P.tile_nent.get(), vals, sched, runtime().d_error));
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

void tile_refill(const TileDesc *tiles, int ntiles, const ProdPtrs *ptrs, const ProdSched *scheds,
                 cudaStream_t s, ProdPtrs vals, ProdSched sched, int ctas_per_sm, bool small, const int *tile_nent,
                 int wcap, int ecap)
{
    if (ntiles <= 0) return;
    if (ptrs)
        launch_refill<true, REFILL_THREADS>(tiles, ntiles, ptrs, scheds, s, vals, sched, ctas_per_sm);
    else if (tile_nent && small)
        launch_refill<false, REFILL_THREADS_SMALL, true>(tiles, ntiles, ptrs, scheds, s, vals, sched, ctas_per_sm,
                                                         tile_nent, wcap, ecap);
    else if (tile_nent)
        launch_refill<false, REFILL_THREADS, true>(tiles, ntiles, ptrs, scheds, s, vals, sched, ctas_per_sm,
                                                   tile_nent, wcap, ecap);
    else if (small)
        launch_refill<false, REFILL_THREADS_SMALL>(tiles, ntiles, ptrs, scheds, s, vals, sched, ctas_per_sm);
    else
        launch_refill<false, REFILL_THREADS>(tiles, ntiles, ptrs, scheds, s, vals, sched, ctas_per_sm);
}

void big_rows_refill(const Product &P, const double *Lx, const double *dvec, const double *Ax,
                     double *Cx, cudaStream_t s, const ProdPtrs *vals)
{
    Runtime &rt = runtime();
    const ProductDesc &d = P.desc;
    NumArgs na{d.Lp, d.Li, d.L_map, d.L_m, P.n_L, Lx, dvec, d.Ap, d.Ai, Ax, P.Cp.get(), P.Ci.get(),
               Cx, rt.d_error};
    const int *rows = P.num_rows.get();
    const int *off = P.num_offset;
    const int *cnt = P.num_count;
    const int cap = rt.num_sms * 16;
    if (cnt[NUM_C2K])
    {
        int th = 256;
        size_t sm = 2048 * 16 + (size_t)th * 8 + (3 * th + 32) * 4;
        set_smem(k_num_cta<2048>, sm);
        SDL_LAUNCH(k_num_cta<2048>, grid_for(cnt[NUM_C2K], 1, cap), th, sm, s, rows + off[NUM_C2K],
                   cnt[NUM_C2K], na, vals);
    }
    if (cnt[NUM_C8K])
    {
        int th = 512;
        size_t sm = 8192 * 16 + (size_t)th * 8 + (3 * th + 32) * 4;
        set_smem(k_num_cta<8192>, sm);
        SDL_LAUNCH(k_num_cta<8192>, grid_for(cnt[NUM_C8K], 1, cap), th, sm, s, rows + off[NUM_C8K],
                   cnt[NUM_C8K], na, vals);
    }
    if (cnt[NUM_GMEM])
    {
        const int th = GMEM_THREADS;
        const size_t sm = gmem_smem_bytes();
        set_smem(k_num_gmem<false>, sm);
        SDL_LAUNCH(k_num_gmem<false>, P.gmem_slots, th, sm, s, rows + off[NUM_GMEM], cnt[NUM_GMEM], na,
                   P.gmem_scratch.get(), P.n, vals, nullptr);
    }
}

void big_rows_refill_scratch(const Product &P, const double *Lx, const double *dvec, const double *Ax,
                             double *Cx, int *posmap, int slots, cudaStream_t s)
{
    Runtime &rt = runtime();
    const ProductDesc &d = P.desc;
    NumArgs na{d.Lp, d.Li, d.L_map, d.L_m, P.n_L, Lx, dvec, d.Ap, d.Ai, Ax, P.Cp.get(), P.Ci.get(),
               Cx, rt.d_error};
    const int *rows = P.num_rows.get();
    const int *off = P.num_offset;
    const int *cnt = P.num_count;
    const int cap = rt.num_sms * 16;
    if (cnt[NUM_C2K])
    {
        int th = 256;
        size_t sm = 2048 * 16 + (size_t)th * 8 + (3 * th + 32) * 4;
        set_smem(k_num_cta<2048>, sm);
        SDL_LAUNCH(k_num_cta<2048>, grid_for(cnt[NUM_C2K], 1, cap), th, sm, s, rows + off[NUM_C2K],
                   cnt[NUM_C2K], na, nullptr);
    }
    if (cnt[NUM_C8K])
    {
        int th = 512;
        size_t sm = 8192 * 16 + (size_t)th * 8 + (3 * th + 32) * 4;
        set_smem(k_num_cta<8192>, sm);
        SDL_LAUNCH(k_num_cta<8192>, grid_for(cnt[NUM_C8K], 1, cap), th, sm, s, rows + off[NUM_C8K],
                   cnt[NUM_C8K], na, nullptr);
    }
    if (cnt[NUM_GMEM])
    {
        const int th = GMEM_THREADS;
        const size_t sm = gmem_smem_bytes();
        set_smem(k_num_gmem<false>, sm);
        SDL_LAUNCH(k_num_gmem<false>, std::min(slots, cnt[NUM_GMEM]), th, sm, s, rows + off[NUM_GMEM],
                   cnt[NUM_GMEM], na, posmap, P.n, nullptr, nullptr);
    }
}

// Whether a single product's entry values are L.x itself: no d, one block, and the
// values kept in L's value order (L_map a permutation) or no L_map at all. The refill
// then reads L.x where it would read V, and the entry-value launch is skipped.
bool entry_values_are_lx(const Product &P, const double *Lx, const double *dvec)
{
    return Lx && !dvec && P.desc.blocks == 1 && (P.kv.get() || !P.desc.L_map);
}

void product_numeric(const Product &P, const double *Lx, const double *dvec, const double *Ax,
                     double *Cx, cudaStream_t s)
{
    NvtxRange nvtx_range_("sdl: refill");
    if (!P.plan_ready)
        fail(SDL_ERR_INVALID, "product from the learned one-shot pass: build its refill plan first "
                              "(sdl_product_complete_plan)");
    if (P.nnz == 0) return;
    ProdSched S = sched_of(P);
    const ProdPtrs vals{Lx, dvec, Ax, Cx};
    const bool direct = entry_values_are_lx(P, Lx, dvec);
    if (direct) S.V = const_cast<double *>(Lx); // read only
    if (P.num_count[NUM_TILE])
    {
        if (!direct) entry_values(S, vals, s);
        if (pipe_refill(P))
            launch_refill_pipe(P, s, vals, S);
        else
        {
            int wcap = 0, ecap = 0;
            staged_caps(P, wcap, ecap);
            tile_refill(P.tiles.get(), P.ntiles, nullptr, nullptr, s, vals, S, P.cfg.refill_ctas_per_sm,
                        small_tile_refill(P), es_refill(P) ? P.tile_nent.get() : nullptr, wcap, ecap);
        }
    }
    if (P.big_lists)
    {
        if (!P.num_count[NUM_TILE] && !direct) entry_values(S, vals, s);
        big_lists_refill(P, nullptr, s, vals, S.V);
    }
    else
        big_rows_refill(P, Lx, dvec, Ax, Cx, s);
}

void big_lists_refill(const Product &P, const ProdPtrs *ptrs, cudaStream_t s, ProdPtrs vals, const double *V)
{
    if (!P.big_lists || P.big_outputs == 0) return;
    const int grid = (P.big_outputs + 255) / 256;
    const long long nV = (long long)P.desc.L_nnz * P.desc.blocks;
    if (!V) V = P.V.get();
    if (ptrs)
        SDL_LAUNCH(k_big_refill<true>, grid, 256, 0, s, P.brows.get(), P.nbig, P.bout_off.get(), P.big_outputs,
                   P.bostart.get(), P.bpairs.get(), P.Cp.get(), ptrs, vals, V, nV, (long long)P.desc.A_nnz,
                   runtime().d_error);
    else
        SDL_LAUNCH(k_big_refill<false>, grid, 256, 0, s, P.brows.get(), P.nbig, P.bout_off.get(), P.big_outputs,
                   P.bostart.get(), P.bpairs.get(), P.Cp.get(), ptrs, vals, V, nV, (long long)P.desc.A_nnz,
                   runtime().d_error);
}

} // namespace sdl

// ------------------------------------------------------------------ autotuner
namespace sdl {
namespace {
__global__ void k_tune_diff(const int *__restrict__ a, const int *__restrict__ b, long long n, int *__restrict__ err)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (a[i] != b[i]) atomicOr(err, 8);
}

__global__ void k_tune_fill(double *x, long long n, double v)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = v;
}
} // namespace

void product_replan(Product &P, const TuneConfig &c, cudaStream_t s)
{
    if (c.refill_threads != REFILL_THREADS && c.refill_threads != REFILL_THREADS_SMALL)
        fail(SDL_ERR_INVALID, "refill threads must be 256 or 128");
    if (c.tile_budget < 0 || c.tile_budget > TILE_T || c.tile_max_terms < 0 || c.tile_max_terms > TILE_T ||
        c.refill_ctas_per_sm < 0)
        fail(SDL_ERR_INVALID, "tile budget / largest tile row must lie in [0, TILE_T]");
    if (P.m_out == 0) return;
    Runtime &rt = runtime();
    Product Q;
    product_symbolic(P.desc, c, Q, s);
    if (Q.nnz != P.nnz || Q.m_out != P.m_out) fail(SDL_ERR_INTERNAL, "replan: the plan has another structure");
    SDL_LAUNCH(k_tune_diff, grid_for(P.m_out + 1, 256, rt.num_sms * 8), 256, 0, s, Q.Cp.get(), P.Cp.get(),
               (long long)P.m_out + 1, rt.d_error);
    if (P.nnz > 0)
        SDL_LAUNCH(k_tune_diff, grid_for(P.nnz, 256, rt.num_sms * 8), 256, 0, s, Q.Ci.get(), P.Ci.get(),
                   (long long)P.nnz, rt.d_error);
    if (take_device_error(s)) fail(SDL_ERR_INTERNAL, "replan: the plan has another structure");
    P = std::move(Q);
}

TuneResult product_autotune(Product &P, int reps, cudaStream_t s)
{
    TuneResult R;
    R.best = P.cfg;
    if (P.m_out == 0 || P.nnz == 0) return R;
    reps = std::max(1, std::min(reps, 50));
    Runtime &rt = runtime();
    const auto t_start = std::chrono::steady_clock::now();
    const ProductDesc d = P.desc;
    // placeholder values: d = A.x = 1 (the entry-value kernel runs as in a real refill)
    DevBuf<double> dv((size_t)std::max(1, d.A_m)), ax((size_t)std::max(1, d.A_nnz)), cx((size_t)P.nnz);
    SDL_LAUNCH(k_tune_fill, grid_for(std::max(1, d.A_m), 256, rt.num_sms * 8), 256, 0, s, dv.get(),
               (long long)std::max(1, d.A_m), 1.0);
    SDL_LAUNCH(k_tune_fill, grid_for(std::max(1, d.A_nnz), 256, rt.num_sms * 8), 256, 0, s, ax.get(),
               (long long)std::max(1, d.A_nnz), 1.0);
    DevBuf<unsigned char> flush((size_t)256 << 20); // larger than L2: each timed refill starts cold
    cudaEvent_t e0, e1;
    SDL_CUDA(cudaEventCreate(&e0));
    SDL_CUDA(cudaEventCreate(&e1));
    auto refill_us = [&](const Product &Q) -> double {
        product_numeric(Q, nullptr, dv.get(), ax.get(), cx.get(), s);
        double best = 1e30;
        for (int r = 0; r < reps; ++r)
        {
            SDL_CUDA(cudaMemsetAsync(flush.get(), r & 0xff, flush.bytes(), s));
            SDL_CUDA(cudaEventRecord(e0, s));
            product_numeric(Q, nullptr, dv.get(), ax.get(), cx.get(), s);
            SDL_CUDA(cudaEventRecord(e1, s));
            SDL_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            SDL_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, 1e3 * ms);
        }
        ++R.candidates;
        return best;
    };
    auto build = [&](const TuneConfig &c, Product &out) -> double {
        const auto t0 = std::chrono::steady_clock::now();
        product_symbolic(d, c, out, s);
        SDL_CUDA(cudaStreamSynchronize(s));
        if (out.nnz != P.nnz || out.m_out != P.m_out)
            fail(SDL_ERR_INTERNAL, "autotune: a candidate plan has another structure");
        SDL_LAUNCH(k_tune_diff, grid_for(P.m_out + 1, 256, rt.num_sms * 8), 256, 0, s, out.Cp.get(), P.Cp.get(),
                   (long long)P.m_out + 1, rt.d_error);
        SDL_LAUNCH(k_tune_diff, grid_for(P.nnz, 256, rt.num_sms * 8), 256, 0, s, out.Ci.get(), P.Ci.get(),
                   (long long)P.nnz, rt.d_error);
        if (take_device_error(s)) fail(SDL_ERR_INTERNAL, "autotune: a candidate plan has another structure");
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    // the plan as given (default configuration) is the first candidate
    R.default_refill_us = refill_us(P);
    // stage 1: symbolic bin thresholds (warp-kernel threshold, warps per CTA)
    const TuneConfig base = P.cfg;
    const int sym_cand[][2] = {{512, 8}, {512, 4}, {512, 16}, {128, 8}};
    TuneConfig sym_best = base;
    double sym_best_ms = 1e30;
    Product stage1;
    for (const auto &sc : sym_cand)
    {
        TuneConfig c = base;
        c.warp_max_terms = sc[0];
        c.rows_per_cta_warp = sc[1];
        Product Q;
        const double ms = build(c, Q);
        if (ms < sym_best_ms)
        {
            sym_best_ms = ms;
            sym_best = c;
            stage1 = std::move(Q);
        }
    }
    R.sym_ms = sym_best_ms;
    // stage 2: tile budget x refill CTAs per SM, on the chosen symbolic configuration
    double best_us = R.default_refill_us;
    TuneConfig best_cfg = base;
    bool have_best = false;
    Product best;
    const int budgets[] = {TILE_T, 3 * TILE_T / 4, TILE_T / 2};
    const int ctas[] = {0, 4, 3};
    for (int b : budgets)
    {
        Product Q;
        TuneConfig c = sym_best;
        c.tile_budget = b == TILE_T ? 0 : b;
        if (b == TILE_T && (c.tile_budget == stage1.cfg.tile_budget))
            Q = std::move(stage1);
        else
            build(c, Q);
        bool kept = false;
        for (int k : ctas)
        {
            Q.cfg.refill_ctas_per_sm = k;
            const double us = refill_us(Q);
            if (us < best_us)
            {
                best_us = us;
                best_cfg = Q.cfg;
                kept = true;
            }
        }
        if (kept)
        {
            Q.cfg = best_cfg;
            best = std::move(Q);
            have_best = true;
        }
    }
    // stage 3: the small-tile refill (128-thread CTAs, tiles and tile rows of at most
    // TILE_T / 2 terms; larger rows leave the tiles), when its windows fit
    {
        Product Q;
        TuneConfig c = sym_best;
        c.tile_budget = TILE_T / 2;
        c.tile_max_terms = TILE_T / 2;
        c.refill_threads = REFILL_THREADS_SMALL;
        c.refill_ctas_per_sm = 0;
        build(c, Q);
        if (small_tile_refill(Q))
        {
            // the direct refill and, when the tiles fit its stages, the pipelined one
            double us = refill_us(Q);
            Q.cfg.refill_pipe = 1;
            if (pipe_refill(Q))
            {
                const double us_pipe = refill_us(Q);
                if (us_pipe < us)
                    us = us_pipe;
                else
                    Q.cfg.refill_pipe = 0;
            }
            else
                Q.cfg.refill_pipe = 0;
            // and the staged direct refill, when its slots fit the largest tile
            if (!Q.cfg.refill_pipe)
            {
                Q.cfg.refill_es = 1;
                if (es_refill(Q))
                {
                    const double us_es = refill_us(Q);
                    if (us_es < us)
                        us = us_es;
                    else
                        Q.cfg.refill_es = 0;
                }
                else
                    Q.cfg.refill_es = 0;
            }
            if (us < best_us)
            {
                best_us = us;
                best_cfg = Q.cfg;
                best = std::move(Q);
                have_best = true;
            }
        }
    }
    SDL_CUDA(cudaEventDestroy(e0));
    SDL_CUDA(cudaEventDestroy(e1));
    if (have_best)
    {
        P = std::move(best);
        R.best = best_cfg;
    }
    else
        R.best = P.cfg;
    R.refill_us = best_us;
    R.tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    return R;
}


// ------------------------------------------------------------------ pattern key
// Statistics of a product's pattern that the tuning table is keyed on: rows of C,
// columns of A, terms per row, terms per output, and the histogram of row lengths
// of C over power-of-two classes. Patterns with equal keys share a tuned plan.
namespace {
__global__ void k_rowlen_hist(const int *__restrict__ Cp, int m, unsigned long long *__restrict__ hist)
{
    __shared__ unsigned long long h[33];
    for (int q = threadIdx.x; q < 33; q += blockDim.x) h[q] = 0;
    __syncthreads();
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m; r += (long long)gridDim.x * blockDim.x)
    {
        const int len = Cp[r + 1] - Cp[r];
        atomicAdd(&h[len > 0 ? 32 - __clz(len) : 0], 1ULL);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 33; q += blockDim.x)
        if (h[q]) atomicAdd(&hist[q], h[q]);
}
} // namespace

std::string product_pattern_key(const Product &P, cudaStream_t s)
{
    Runtime &rt = runtime();
    unsigned long long hist[33] = {0};
    if (P.m_out > 0)
    {
        DevBuf<unsigned long long> dh(33);
        SDL_CUDA(cudaMemsetAsync(dh.get(), 0, dh.bytes(), s));
        SDL_LAUNCH(k_rowlen_hist, grid_for(P.m_out, 256, rt.num_sms * 4), 256, 0, s, P.Cp.get(), P.m_out, dh.get());
        SDL_CUDA(cudaMemcpyAsync(hist, dh.get(), sizeof(hist), cudaMemcpyDeviceToHost, s));
        SDL_CUDA(cudaStreamSynchronize(s));
    }
    auto lg = [](double v) { return (int)std::floor(std::log2(v + 1.0)); };
    const double rows = std::max(1, P.m_out);
    char buf[96];
    std::snprintf(buf, sizeof buf, "m%d.n%d.t%d.c%d.h", lg(P.m_out), lg(P.n),
                  (int)std::lround(2.0 * std::log2((double)P.terms / rows + 1.0)),
                  (int)std::min<long long>(64, std::llround(4.0 * (double)P.terms / std::max(1, P.nnz))));
    std::string key(buf);
    for (int b = 0; b < 33; ++b)
    {
        const int eighths = (int)std::lround(8.0 * (double)hist[b] / rows);
        if (eighths > 0) key += std::to_string(b) + ":" + std::to_string(eighths) + ",";
    }
    return key;
}

} // namespace sdl
