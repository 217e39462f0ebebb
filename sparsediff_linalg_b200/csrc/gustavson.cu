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
//   numeric:  warp + shared accumulator (<= 512 terms), CTA + shared accumulator
//             (<= 8192 output entries), CTA + accumulator in C.x itself with a
//             global column->position map (larger rows).
#include <algorithm>
#include <climits>
#include <cstring>
#include <string>

#include "sdl_device.cuh"
#include "sdl_internal.h"

namespace sdl {

void segment_sort_u64(unsigned long long *d_keys, const int *d_off, int nseg, int nkeys,
                      cudaStream_t s);

namespace {

struct SymArgs
{
    const int *Lp, *Li;
    int L_m, n_L, n;
    const int *Ap, *Ai;
    const long long *ub_off;
    int *tmp;
    int *row_nnz;
};

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

__global__ void k_sym_classify(const long long *__restrict__ ub, int m_out,
                               unsigned char *__restrict__ cls)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
    {
        long long u = ub[r];
        int c = u == 0 ? 255 : u <= 32 ? SYM_W32 : u <= 128 ? SYM_W128 : u <= 512 ? SYM_W512
                         : u <= 2048 ? SYM_C2K : u <= 8192 ? SYM_C8K : SYM_BITMAP;
        cls[r] = (unsigned char)c;
    }
}

__global__ void k_num_classify(const long long *__restrict__ ub, const int *__restrict__ Cp,
                               int m_out, unsigned char *__restrict__ cls, long long *__restrict__ plan_len)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
    {
        long long u = ub[r];
        int nr = Cp[r + 1] - Cp[r];
        int c;
        if (u == 0)
            c = 255;
        else if (u <= 32)
            c = NUM_W32;
        else if (u <= 64)
            c = NUM_W64;
        else if (u <= 128)
            c = NUM_W128;
        else if (u <= 256)
            c = NUM_W256;
        else if (u <= 512)
            c = NUM_W512;
        else if (nr <= 2048)
            c = NUM_C2K;
        else if (nr <= 8192)
            c = NUM_C8K;
        else
            c = NUM_GMEM;
        cls[r] = (unsigned char)c;
        plan_len[r] = c < NUM_WARP_CLASSES ? u : 0;
    }
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
        long long off = a.ub_off[row];
        int nn = 0;
        for (int base = 0; base < cnt; base += 32)
        {
            int q = base + lane;
            bool flag = q < cnt && (q == 0 || buf[q] != buf[q - 1]);
            unsigned bal = __ballot_sync(FULL_MASK, flag);
            if (flag) a.tmp[off + nn + __popc(bal & lanemask_lt())] = buf[q];
            nn += __popc(bal);
        }
        if (lane == 0) a.row_nnz[row] = nn;
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
        long long off = a.ub_off[row];
        int nn = 0;
        for (int base = 0; base < cnt; base += blockDim.x)
        {
            int q = base + threadIdx.x;
            int flag = (q < cnt && (q == 0 || buf[q] != buf[q - 1])) ? 1 : 0;
            int incl = block_incl_scan_int(flag, ch.scr);
            if (flag) a.tmp[off + nn + incl - 1] = buf[q];
            if (threadIdx.x == blockDim.x - 1) tot_sh = incl;
            __syncthreads();
            nn += tot_sh;
            __syncthreads();
        }
        if (threadIdx.x == 0) a.row_nnz[row] = nn;
        __syncthreads();
    }
}

// Large rows: mark columns in a shared-memory bitmap, one column window at a time;
// reading the bitmap word by word yields the columns in ascending order.
__global__ void k_sym_bitmap(const int *__restrict__ rows, int count, SymArgs a, int words)
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
    const int wbits = words * 32;
    for (int it = blockIdx.x; it < count; it += gridDim.x)
    {
        int row = rows[it];
        int b = row / a.L_m, r = row - b * a.L_m;
        int ls = a.Lp[r], le = a.Lp[r + 1];
        long long off = a.ub_off[row];
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
                    a.tmp[pos++] = (int)(ws + q * 32 + bit);
                    word &= word - 1;
                }
            }
            if (threadIdx.x == blockDim.x - 1) tot_sh = incl;
            __syncthreads();
            running += tot_sh;
            __syncthreads();
        }
        if (threadIdx.x == 0) a.row_nnz[row] = running;
        __syncthreads();
    }
}

__global__ void k_compact(const long long *__restrict__ ub_off, const int *__restrict__ row_nnz,
                          const int *__restrict__ Cp, const int *__restrict__ tmp,
                          int *__restrict__ Ci, int m_out)
{
    const int lane = lane_id(), wpb = blockDim.x >> 5;
    for (long long row = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); row < m_out;
         row += (long long)gridDim.x * wpb)
    {
        int nn = row_nnz[row];
        const int *src = tmp + ub_off[row];
        int *dst = Ci + Cp[row];
        for (int q = lane; q < nn; q += 32) dst[q] = src[q];
    }
}

// ------------------------------------------------------------ numeric kernels
// Apply acc[pos] += prod for the valid lanes, lanes sharing a position one after
// another in lane (= term) order.
__device__ __forceinline__ void warp_ordered_add(double *acc, int pos, double prod, bool valid)
{
    unsigned key = valid ? (unsigned)pos : (0x80000000u | (unsigned)lane_id());
    unsigned peers = __match_any_sync(FULL_MASK, key);
    int rank = __popc(peers & lanemask_lt());
    unsigned rounds = __reduce_max_sync(FULL_MASK, valid ? (unsigned)__popc(peers) : 1u);
    for (unsigned q = 0; q < rounds; ++q)
    {
        if (valid && rank == (int)q) acc[pos] = __dadd_rn(acc[pos], prod);
        __syncwarp();
    }
}

// Plan of a warp-class row, built once per pattern: the terms are visited exactly
// as k_num_warp_plan visits them (L entries in chunks of 32, their terms in windows
// of 32), and every term gets its position inside the output row (found by binary
// search in the sorted row), plus bit 15 when its window has two terms on one
// position (so the numeric kernel must apply that window in term order).
template <int CAP>
__global__ void k_build_plan(const int *__restrict__ rows, int count, NumArgs a,
                             unsigned short *__restrict__ plan, const long long *__restrict__ plan_off)
{
    extern __shared__ int sci[];
    const int lane = lane_id(), wpb = blockDim.x >> 5;
    int *ci = sci + (threadIdx.x >> 5) * CAP;
    for (long long it = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); it < count;
         it += (long long)gridDim.x * wpb)
    {
        int row = rows[it];
        int b = row / a.L_m, r = row - b * a.L_m;
        int cs = a.Cp[row], nr = a.Cp[row + 1] - cs;
        for (int q = lane; q < nr; q += 32) ci[q] = a.Ci[cs + q];
        __syncwarp();
        long long po = plan_off[row];
        int ls = a.Lp[r], le = a.Lp[r + 1], cum = 0;
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
                bool valid = u < total;
                int e = warp_entry_of(incl, u);
                int se = __shfl_sync(FULL_MASK, s, e);
                int ie = __shfl_sync(FULL_MASK, incl, e);
                int lne = __shfl_sync(FULL_MASK, len, e);
                int pos = 0;
                if (valid)
                {
                    int j = a.Ai[se + u - (ie - lne)];
                    pos = lower_bound_dev(ci, nr, j);
                    if (pos >= nr || ci[pos] != j)
                    {
                        atomicOr(a.err, 1);
                        pos = 0x7fff; // rejected by the numeric kernel's range check
                    }
                }
                unsigned key = valid ? (unsigned)pos : (0x80000000u | (unsigned)lane);
                unsigned peers = __match_any_sync(FULL_MASK, key);
                bool dup = __any_sync(FULL_MASK, valid && __popc(peers) > 1);
                if (valid) plan[po + cum + u] = (unsigned short)(pos | (dup ? 0x8000 : 0));
            }
            cum += total;
        }
        __syncwarp();
    }
}

// Warp-class numeric refill through the plan: per term only the value of A is
// gathered (no column index, no search); the loads of up to BATCH windows are
// issued before their accumulations so their latencies overlap. Windows without a
// duplicated position are applied in one step, the others lane by lane in term
// order.
template <int CAP, int BATCH>
__global__ void k_num_warp_plan(const int *__restrict__ rows, int count, NumArgs a,
                                const unsigned short *__restrict__ plan,
                                const long long *__restrict__ plan_off)
{
    extern __shared__ __align__(16) double sacc[];
    const int lane = lane_id(), wpb = blockDim.x >> 5;
    double *acc = sacc + (threadIdx.x >> 5) * CAP;
    for (long long it = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); it < count;
         it += (long long)gridDim.x * wpb)
    {
        int row = rows[it];
        int b = row / a.L_m, r = row - b * a.L_m;
        int cs = a.Cp[row], nr = a.Cp[row + 1] - cs;
        for (int q = lane; q < nr; q += 32) acc[q] = 0.0;
        __syncwarp();
        long long po = plan_off[row];
        int ls = a.Lp[r], le = a.Lp[r + 1], cum = 0;
        for (int c = ls; c < le; c += 32)
        {
            int ii = c + lane, s = 0, len = 0;
            double v = 0.0;
            if (ii < le)
            {
                int k = a.Li[ii] + b * a.n_L;
                s = a.Ap[k];
                len = a.Ap[k + 1] - s;
                double lx = a.Lx ? a.Lx[a.L_map ? a.L_map[ii] : ii] : 1.0;
                v = a.d ? __dmul_rn(lx, a.d[k]) : lx;
            }
            int incl = warp_incl_scan(len);
            int total = __shfl_sync(FULL_MASK, incl, 31);
            for (int b0 = 0; b0 < total; b0 += 32 * BATCH)
            {
                int pos_r[BATCH];
                double prod_r[BATCH];
                unsigned dup_r = 0;
#pragma unroll
                for (int k = 0; k < BATCH; ++k)
                {
                    pos_r[k] = -1;
                    prod_r[k] = 0.0;
                    int base = b0 + 32 * k;
                    if (base < total)
                    {
                        int u = base + lane;
                        int e = warp_entry_of(incl, u);
                        int se = __shfl_sync(FULL_MASK, s, e);
                        int ie = __shfl_sync(FULL_MASK, incl, e);
                        int lne = __shfl_sync(FULL_MASK, len, e);
                        double ve = __shfl_sync(FULL_MASK, v, e);
                        if (u < total)
                        {
                            unsigned pe = plan[po + cum + u];
                            prod_r[k] = __dmul_rn(ve, a.Ax[se + u - (ie - lne)]);
                            pos_r[k] = (int)(pe & 0x7fffu);
                            dup_r |= (pe >> 15) << k;
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < BATCH; ++k)
                {
                    if (b0 + 32 * k < total)
                    {
                        int pos = pos_r[k];
                        bool valid = pos >= 0;
                        if (valid && pos >= nr)
                        {
                            atomicOr(a.err, 1);
                            valid = false;
                        }
                        if (__any_sync(FULL_MASK, (dup_r >> k) & 1u))
                        {
                            warp_ordered_add(acc, pos, prod_r[k], valid);
                        }
                        else
                        {
                            if (valid) acc[pos] = __dadd_rn(acc[pos], prod_r[k]);
                            __syncwarp();
                        }
                    }
                }
            }
            cum += total;
        }
        __syncwarp();
        for (int q = lane; q < nr; q += 32) a.Cx[cs + q] = acc[q];
        __syncwarp();
    }
}

// Medium rows: one CTA per row, shared accumulator indexed by output position;
// a claim table orders same-position terms of a chunk by term index.
template <int CAP>
__global__ void k_num_cta(const int *__restrict__ rows, int count, NumArgs a)
{
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

constexpr int GMEM_CLAIM = 4096;

// Large rows: accumulate straight into C.x; a per-CTA global map column -> position
// (only this row's columns are ever read, so it never needs clearing) and a hashed
// claim table keep same-position terms in order.
__global__ void k_num_gmem(const int *__restrict__ rows, int count, NumArgs a,
                           int *__restrict__ posmap_all, int n)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    CtaChunk ch;
    ch.v = (double *)smraw;
    int *claim = (int *)(ch.v + blockDim.x);
    ch.incl = claim + GMEM_CLAIM;
    ch.s = ch.incl + blockDim.x;
    ch.len = ch.s + blockDim.x;
    ch.scr = ch.len + blockDim.x;
    int *posmap = posmap_all + (long long)blockIdx.x * n;
    for (int it = blockIdx.x; it < count; it += gridDim.x)
    {
        int row = rows[it];
        int b = row / a.L_m, r = row - b * a.L_m;
        int cs = a.Cp[row], nr = a.Cp[row + 1] - cs;
        double *acc = a.Cx + cs;
        for (int q = threadIdx.x; q < nr; q += blockDim.x)
        {
            posmap[a.Ci[cs + q]] = q;
            acc[q] = 0.0;
        }
        for (int q = threadIdx.x; q < GMEM_CLAIM; q += blockDim.x) claim[q] = INT_MAX;
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
                    pos = posmap[j];
                    if (pos < 0 || pos >= nr)
                    {
                        atomicOr(a.err, 1);
                        pending = false;
                    }
                }
                int slot = pos & (GMEM_CLAIM - 1);
                while (true)
                {
                    if (pending) atomicMin(&claim[slot], u);
                    __syncthreads();
                    bool won = pending && claim[slot] == u;
                    if (won) acc[pos] = __dadd_rn(acc[pos], prod);
                    __syncthreads();
                    if (won)
                    {
                        claim[slot] = INT_MAX;
                        pending = false;
                    }
                    if (!__syncthreads_or(pending)) break;
                }
            }
            __syncthreads();
        }
        __syncthreads();
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

void product_symbolic(const ProductDesc &d, const TuneConfig &cfg, Product &P, cudaStream_t s,
                      bool keep_row_terms)
{
    Runtime &rt = runtime();
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
               cls.get());
    DevBuf<int> lists;
    int cnt[SYM_NBINS], off[SYM_NBINS + 1];
    bin_items(cls.get(), m_out, SYM_NBINS, lists, cnt, off, s);

    SymArgs sa{d.Lp, d.Li, d.L_m, P.n_L, d.A_n, d.Ap, d.Ai, ub_off.get(), tmp.get(), row_nnz.get()};
    const int cap = rt.num_sms * 16;
    const int wpb = 8;
    if (cnt[SYM_W32])
        SDL_LAUNCH(k_sym_warp<32>, grid_for(cnt[SYM_W32], wpb, cap), wpb * 32, wpb * 32 * 4, s,
                   lists.get() + off[SYM_W32], cnt[SYM_W32], sa);
    if (cnt[SYM_W128])
        SDL_LAUNCH(k_sym_warp<128>, grid_for(cnt[SYM_W128], wpb, cap), wpb * 32, wpb * 128 * 4, s,
                   lists.get() + off[SYM_W128], cnt[SYM_W128], sa);
    if (cnt[SYM_W512])
        SDL_LAUNCH(k_sym_warp<512>, grid_for(cnt[SYM_W512], wpb, cap), wpb * 32, wpb * 512 * 4, s,
                   lists.get() + off[SYM_W512], cnt[SYM_W512], sa);
    if (cnt[SYM_C2K])
    {
        int th = 256;
        size_t sm = 2048 * 4 + (3 * th + 32) * 4;
        SDL_LAUNCH(k_sym_cta<2048>, grid_for(cnt[SYM_C2K], 1, cap), th, sm, s,
                   lists.get() + off[SYM_C2K], cnt[SYM_C2K], sa);
    }
    if (cnt[SYM_C8K])
    {
        int th = 512;
        size_t sm = 8192 * 4 + (3 * th + 32) * 4;
        set_smem(k_sym_cta<8192>, sm);
        SDL_LAUNCH(k_sym_cta<8192>, grid_for(cnt[SYM_C8K], 1, cap), th, sm, s,
                   lists.get() + off[SYM_C8K], cnt[SYM_C8K], sa);
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
        SDL_LAUNCH(k_sym_bitmap, grid_for(cnt[SYM_BITMAP], 1, rt.num_sms * 2), th, sm, s,
                   lists.get() + off[SYM_BITMAP], cnt[SYM_BITMAP], sa, words);
    }

    P.nnz = exclusive_scan_i32_checked(row_nnz.get(), P.Cp.get(), m_out, s);
    P.Ci.reset(std::max(1, P.nnz));
    if (P.nnz > 0)
        SDL_LAUNCH(k_compact, grid_for(m_out, 8, rt.num_sms * 16), 256, 0, s, ub_off.get(),
                   row_nnz.get(), P.Cp.get(), tmp.get(), P.Ci.get(), m_out);

    DevBuf<long long> plan_len(m_out);
    SDL_LAUNCH(k_num_classify, grid_for(m_out, 256, rt.num_sms * 8), 256, 0, s, ub.get(),
               P.Cp.get(), m_out, cls.get(), plan_len.get());
    bin_items(cls.get(), m_out, NUM_NBINS, P.num_rows, P.num_count, P.num_offset, s);
    P.plan_off.reset((size_t)m_out + 1);
    long long plan_total = exclusive_scan_i64(plan_len.get(), P.plan_off.get(), m_out, s);
    P.plan.reset(std::max<long long>(1, plan_total));
    {
        NumArgs na{d.Lp, d.Li, d.L_map, d.L_m, P.n_L, nullptr, nullptr, d.Ap, d.Ai, nullptr,
                   P.Cp.get(), P.Ci.get(), nullptr, rt.d_error};
        const int *rows = P.num_rows.get();
        const int wpb_b = 8;
#define SDL_BUILD_PLAN(CLS, CAPV)                                                                   \
    if (P.num_count[CLS])                                                                           \
        SDL_LAUNCH(k_build_plan<CAPV>, grid_for(P.num_count[CLS], wpb_b, cap), wpb_b * 32,            \
                   wpb_b * (CAPV) * 4, s, rows + P.num_offset[CLS], P.num_count[CLS], na, P.plan.get(), \
                   P.plan_off.get());
        SDL_BUILD_PLAN(NUM_W32, 32)
        SDL_BUILD_PLAN(NUM_W64, 64)
        SDL_BUILD_PLAN(NUM_W128, 128)
        SDL_BUILD_PLAN(NUM_W256, 256)
        SDL_BUILD_PLAN(NUM_W512, 512)
#undef SDL_BUILD_PLAN
    }
    if (take_device_error(s)) fail(SDL_ERR_INTERNAL, "product plan: a term column is missing from its row");
    if (P.num_count[NUM_GMEM])
    {
        long long per_slot = std::max(1, P.n);
        long long max_slots = std::max<long long>(1, (2LL << 30) / (per_slot * 4));
        P.gmem_slots = (int)std::min<long long>({(long long)rt.num_sms, max_slots,
                                                 (long long)P.num_count[NUM_GMEM]});
        P.gmem_scratch.reset((size_t)P.gmem_slots * per_slot);
    }
    if (keep_row_terms) P.row_terms = std::move(ub);
    SDL_CUDA(cudaStreamSynchronize(s));
}

void product_numeric(const Product &P, const double *Lx, const double *dvec, const double *Ax,
                     double *Cx, cudaStream_t s)
{
    Runtime &rt = runtime();
    if (P.nnz == 0) return;
    const ProductDesc &d = P.desc;
    NumArgs na{d.Lp, d.Li, d.L_map, d.L_m, P.n_L, Lx, dvec, d.Ap, d.Ai, Ax, P.Cp.get(), P.Ci.get(),
               Cx, rt.d_error};
    const int *rows = P.num_rows.get();
    const int *off = P.num_offset;
    const int *cnt = P.num_count;
    const int cap = rt.num_sms * 16;
    const int wpb = 8;
#define SDL_NUM_WARP(CLS, CAPV, BATCHV)                                                        \
    if (cnt[CLS])                                                                              \
        SDL_LAUNCH((k_num_warp_plan<CAPV, BATCHV>), grid_for(cnt[CLS], wpb, cap), wpb * 32,      \
                   wpb * (CAPV) * 8, s, rows + off[CLS], cnt[CLS], na, P.plan.get(), P.plan_off.get());
    SDL_NUM_WARP(NUM_W32, 32, 1)
    SDL_NUM_WARP(NUM_W64, 64, 2)
    SDL_NUM_WARP(NUM_W128, 128, 4)
    SDL_NUM_WARP(NUM_W256, 256, 8)
    SDL_NUM_WARP(NUM_W512, 512, 8)
#undef SDL_NUM_WARP
    if (cnt[NUM_C2K])
    {
        int th = 256;
        size_t sm = 2048 * 16 + (size_t)th * 8 + (3 * th + 32) * 4;
        set_smem(k_num_cta<2048>, sm);
        SDL_LAUNCH(k_num_cta<2048>, grid_for(cnt[NUM_C2K], 1, cap), th, sm, s, rows + off[NUM_C2K],
                   cnt[NUM_C2K], na);
    }
    if (cnt[NUM_C8K])
    {
        int th = 512;
        size_t sm = 8192 * 16 + (size_t)th * 8 + (3 * th + 32) * 4;
        set_smem(k_num_cta<8192>, sm);
        SDL_LAUNCH(k_num_cta<8192>, grid_for(cnt[NUM_C8K], 1, cap), th, sm, s, rows + off[NUM_C8K],
                   cnt[NUM_C8K], na);
    }
    if (cnt[NUM_GMEM])
    {
        int th = 512;
        size_t sm = (size_t)th * 8 + GMEM_CLAIM * 4 + (3 * th + 32) * 4;
        set_smem(k_num_gmem, sm);
        SDL_LAUNCH(k_num_gmem, P.gmem_slots, th, sm, s, rows + off[NUM_GMEM], cnt[NUM_GMEM], na,
                   P.gmem_scratch.get(), P.n);
    }
}

} // namespace sdl
