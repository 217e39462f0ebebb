// Device kernels of the matrix sums and vstack (capi_sum.cpp).
#include <algorithm>

#include "sdl_internal.h"

namespace sdl {
namespace {

int grid_sum(long long n, int per_block)
{
    long long g = (n + per_block - 1) / per_block;
    return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 32));
}

// Output position of each input triplet: its column's place in the coalesced row.
__global__ void k_sum_positions(const int *__restrict__ rows, const int *__restrict__ cols, int n,
                                const int *__restrict__ Cp, const int *__restrict__ Ci, int *__restrict__ map,
                                int *__restrict__ err)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    {
        int lo = Cp[rows[t]], hi = Cp[rows[t] + 1];
        const int c = cols[t];
        while (lo < hi)
        {
            const int mid = (lo + hi) >> 1;
            if (Ci[mid] < c)
                lo = mid + 1;
            else
                hi = mid;
        }
        if (lo >= Cp[rows[t] + 1] || Ci[lo] != c)
        {
            atomicOr(err, 1);
            lo = -1;
        }
        map[t] = lo;
    }
}

// Per-triplet factor of a scaled two-operand sum: d1[row] for the first operand's
// triplets, d2[row] for the second's.
__global__ void k_sum_factors(const int *__restrict__ rows, int n, int split, const double *__restrict__ d1,
                              const double *__restrict__ d2, double *__restrict__ f)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        f[t] = t < split ? d1[rows[t]] : d2[rows[t]];
}

// C[map[j]] += x[j]; map is injective within one operand, so no two threads share a cell.
__global__ void k_scatter_add(const int *__restrict__ map, const double *__restrict__ x, int n,
                              double *__restrict__ C)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        C[map[j]] = __dadd_rn(C[map[j]], x[j]);
}

// C[pos[j]] = x[j] (a stacked_pd's block-major values into CSR order).
__global__ void k_scatter_copy(const int *__restrict__ pos, const double *__restrict__ x, int n,
                               double *__restrict__ C)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) C[pos[j]] = x[j];
}

} // namespace

void sum_positions(const int *rows, const int *cols, int n, const int *Cp, const int *Ci, int *map, cudaStream_t s)
{
    if (n <= 0) return;
    SDL_LAUNCH(k_sum_positions, grid_sum(n, 256), 256, 0, s, rows, cols, n, Cp, Ci, map, runtime().d_error);
}

void sum_factors(const int *rows, int n, int split, const double *d1, const double *d2, double *f, cudaStream_t s)
{
    if (n <= 0) return;
    SDL_LAUNCH(k_sum_factors, grid_sum(n, 256), 256, 0, s, rows, n, split, d1, d2, f);
}

void scatter_add(const int *map, const double *x, int n, double *C, cudaStream_t s)
{
    if (n <= 0) return;
    SDL_LAUNCH(k_scatter_add, grid_sum(n, 256), 256, 0, s, map, x, n, C);
}

void scatter_copy(const int *pos, const double *x, int n, double *C, cudaStream_t s)
{
    if (n <= 0) return;
    SDL_LAUNCH(k_scatter_copy, grid_sum(n, 256), 256, 0, s, pos, x, n, C);
}

} // namespace sdl
