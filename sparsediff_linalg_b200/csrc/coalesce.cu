// Value refill of a COO coalescing plan (and of the matrix sums built on it), as a
// gather in output order: at plan time every triplet's output position is found
// (binary search of its column in its output row) and the triplets are sorted by
// it with the stable radix sort, so each output's triplets sit together in
// ascending triplet order; a refill is then one thread per output summing its
// triplets' values (times their factors, when given) from +0.0 in that order --
// upstream's memset + accumulator order, bit for bit -- with the triplet-to-output
// permutation read in order and the values gathered once each.
#include <algorithm>

#include "sdl_device.cuh"
#include "sdl_internal.h"

namespace sdl {

void sum_positions(const int *rows, const int *cols, int n, const int *Cp, const int *Ci, int *map, cudaStream_t s);
void radix_sort_pairs(unsigned *keys, uint2 *vals, unsigned *keys_tmp, uint2 *vals_tmp, int n, int key_bits,
                      cudaStream_t s);

namespace {

int grid_coal(long long n, int per_block)
{
    long long g = (n + per_block - 1) / per_block;
    return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 32));
}

__global__ void k_coal_keys(const int *__restrict__ map, int n, unsigned *__restrict__ keys, uint2 *__restrict__ vals)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    {
        keys[t] = (unsigned)map[t];
        vals[t] = make_uint2((unsigned)t, 0u);
    }
}

// perm[q] = triplet of sorted slot q; ostart[o] = first slot of output o.
__global__ void k_coal_starts(const unsigned *__restrict__ keys, const uint2 *__restrict__ vals, int n, int nout,
                              int *__restrict__ perm, int *__restrict__ ostart, int *__restrict__ err)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    {
        perm[q] = (int)vals[q].x;
        const unsigned k = keys[q];
        if (k >= (unsigned)nout)
        {
            atomicOr(err, 1);
            continue;
        }
        if (q == 0 || keys[q - 1] != k) ostart[k] = (int)q;
        if (q == 0 && k != 0) atomicOr(err, 1); // output 0 has no triplet
        if (q > 0 && keys[q - 1] != k && k != keys[q - 1] + 1) atomicOr(err, 1); // an output without triplets
        if (q == n - 1 && k != (unsigned)nout - 1) atomicOr(err, 1);             // the last outputs without triplets
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) ostart[nout] = n;
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

} // namespace

void coalesce_order_build(const int *rows, const int *cols, int n, const int *Cp, const int *Ci, int nout,
                          DevBuf<int> &perm, DevBuf<int> &ostart, cudaStream_t s)
{
    perm.reset((size_t)std::max(1, n));
    ostart.reset((size_t)nout + 1);
    if (n == 0)
    {
        SDL_CUDA(cudaMemsetAsync(ostart.get(), 0, ((size_t)nout + 1) * sizeof(int), s));
        return;
    }
    DevBuf<int> map((size_t)n);
    sum_positions(rows, cols, n, Cp, Ci, map.get(), s);
    if (take_device_error(s)) fail(SDL_ERR_INTERNAL, "coalesce plan: a triplet's column is missing from its row");
    DevBuf<unsigned> keys((size_t)n), keys_tmp((size_t)n);
    DevBuf<uint2> vals((size_t)n), vals_tmp((size_t)n);
    SDL_LAUNCH(k_coal_keys, grid_coal(n, 256), 256, 0, s, map.get(), n, keys.get(), vals.get());
    int bits = 1;
    while (bits < 32 && ((long long)1 << bits) < (long long)nout) ++bits;
    radix_sort_pairs(keys.get(), vals.get(), keys_tmp.get(), vals_tmp.get(), n, bits, s);
    SDL_LAUNCH(k_coal_starts, grid_coal(n, 256), 256, 0, s, keys.get(), vals.get(), n, nout, perm.get(), ostart.get(),
               runtime().d_error);
    if (take_device_error(s)) fail(SDL_ERR_INTERNAL, "coalesce plan: inconsistent output order");
}

void coalesce_order_fill(const int *ostart, const int *perm, const double *x, const double *f, int nout, double *C,
                         cudaStream_t s)
{
    if (nout <= 0) return;
    SDL_LAUNCH(k_coal_fill, grid_coal(nout, 256), 256, 0, s, ostart, perm, x, f, nout, C);
}

} // namespace sdl
