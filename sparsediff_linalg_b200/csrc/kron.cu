// y = kron(I_p, A) x (upstream src/matmul_kron_dispatchers.c:18-27 ->
// src/sparse/linalg_sparse_matmuls.c:25-50 for a sparse A,
// src/permuted_dense/permuted_dense.c:131-150 for a full permuted_dense A).
#include <algorithm>

#include "sdl_device.cuh"
#include "sdl_internal.h"

namespace sdl {
namespace {

// One thread per (block b, row i): the row's entries in CSR order, from +0.0
// (bit-identical to upstream's loop).
__global__ void k_kron_vec_csr(const int *__restrict__ Ap, const int *__restrict__ Ai, const double *__restrict__ Ax,
                               int m, int n, int p, const double *__restrict__ x, double *__restrict__ y)
{
    const long long total = (long long)m * p;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int b = (int)(t / m), i = (int)(t - (long long)b * m);
        const double *xb = x + (long long)b * n;
        double acc = 0.0;
        for (int q = Ap[i]; q < Ap[i + 1]; ++q) acc = __dadd_rn(acc, __dmul_rn(Ax[q], xb[Ai[q]]));
        y[t] = acc;
    }
}

// One warp per (block b, row i) of y = X A^T for a dense m x n A (upstream calls
// cblas_dgemm here, whose summation order is unspecified): lanes take strided
// columns, then a shuffle reduction.
__global__ void k_kron_vec_dense(const double *__restrict__ A, int m, int n, int p, const double *__restrict__ x,
                                 double *__restrict__ y)
{
    const long long total = (long long)m * p;
    const int lane = threadIdx.x & 31;
    for (long long t = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; t < total;
         t += ((long long)gridDim.x * blockDim.x) >> 5)
    {
        const int b = (int)(t / m), i = (int)(t - (long long)b * m);
        const double *xb = x + (long long)b * n, *ai = A + (long long)i * n;
        double acc = 0.0;
        for (int j = lane; j < n; j += 32) acc = __dadd_rn(acc, __dmul_rn(ai[j], xb[j]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(FULL_MASK, acc, o));
        if (lane == 0) y[t] = acc;
    }
}

int grid_kron(long long n, int per_block)
{
    long long g = (n + per_block - 1) / per_block;
    return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 32));
}

} // namespace

void kron_vec_csr(const int *Ap, const int *Ai, const double *Ax, int m, int n, int p, const double *x, double *y,
                  cudaStream_t s)
{
    if ((long long)m * p <= 0) return;
    SDL_LAUNCH(k_kron_vec_csr, grid_kron((long long)m * p, 256), 256, 0, s, Ap, Ai, Ax, m, n, p, x, y);
}

void kron_vec_dense(const double *A, int m, int n, int p, const double *x, double *y, cudaStream_t s)
{
    if ((long long)m * p <= 0) return;
    SDL_LAUNCH(k_kron_vec_dense, grid_kron((long long)m * p * 32, 256), 256, 0, s, A, m, n, p, x, y);
}

} // namespace sdl
