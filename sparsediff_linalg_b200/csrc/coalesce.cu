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
                q0[j] = ostart[o];
                q1[j] = ostart[o + 1];
            }
        }
        int t[COAL_ILP];
#pragma unroll
        for (int j = 0; j < COAL_ILP; ++j) t[j] = q0[j] < q1[j] ? perm[q0[j]] : -1;
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
                const int tq = perm[q];
                acc = __dadd_rn(acc, f ? __dmul_rn(f[tq], x[tq]) : x[tq]);
            }
            C[o] = acc;
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

} // namespace sdl
