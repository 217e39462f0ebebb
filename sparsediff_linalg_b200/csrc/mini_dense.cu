// Dense-vector helpers of upstream include/sparsediff_linalg/dense.h
// (src/support/mini_numpy.c), on the device: host arrays in and out, one thread
// per output value, each sum over its terms in upstream's loop order from +0.0
// (bit-identical).
#include <algorithm>

#include "capi_common.h"
#include "sparsediff_linalg/dense.h"

namespace sdl {
namespace {

int grid_mini(long long n)
{
    long long g = (n + 255) / 256;
    return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 32));
}

#define SDL_GRID_STRIDE(i, n)                                                                  \
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n);              \
         i += (long long)gridDim.x * blockDim.x)

__global__ void k_repeat(double *r, const double *a, int len, int reps)
{
    SDL_GRID_STRIDE(i, (long long)len * reps) r[i] = a[i / reps];
}

__global__ void k_tile(double *r, const double *a, int len, int tiles)
{
    SDL_GRID_STRIDE(i, (long long)len * tiles) r[i] = a[i % len];
}

__global__ void k_fill(double *r, long long n, double v)
{
    SDL_GRID_STRIDE(i, n) r[i] = v;
}

// AT[j m + i] = A[i n + j]; thread per output value, reading along A's columns.
__global__ void k_transpose_dense(double *AT, const double *A, int m, int n)
{
    SDL_GRID_STRIDE(e, (long long)m * n)
    {
        const long long j = e / m, i = e - j * m;
        AT[e] = A[i * n + j];
    }
}

// v[row + j m] = sum over col of Y[j + col k] * w[row + col m]
__global__ void k_y_kron_i(int m, int k, int n, const double *Y, const double *w, double *v)
{
    SDL_GRID_STRIDE(e, (long long)m * k)
    {
        const int j = (int)(e / m), row = (int)(e - (long long)j * m);
        double sum = 0.0;
        for (int col = 0; col < n; ++col)
            sum = __dadd_rn(sum, __dmul_rn(Y[j + (long long)col * k], w[row + (long long)col * m]));
        v[e] = sum;
    }
}

// v[j + col k] = sum over row of X[row + j m] * w[row + col m]
__global__ void k_i_kron_xt(int m, int k, int n, const double *X, const double *w, double *v)
{
    SDL_GRID_STRIDE(e, (long long)k * n)
    {
        const int col = (int)(e / k), j = (int)(e - (long long)col * k);
        double sum = 0.0;
        for (int row = 0; row < m; ++row)
            sum = __dadd_rn(sum, __dmul_rn(X[row + (long long)j * m], w[row + (long long)col * m]));
        v[e] = sum;
    }
}

cudaStream_t S() { return runtime().stream; }

DevBuf<double> up(const double *h, long long n, cudaStream_t s)
{
    DevBuf<double> b((size_t)std::max<long long>(1, n));
    if (n > 0) h2d(b.get(), h, (size_t)n, s);
    return b;
}

void down(double *h, const DevBuf<double> &b, long long n, cudaStream_t s)
{
    if (n > 0) d2h(h, b.get(), (size_t)n, s);
    SDL_CUDA(cudaStreamSynchronize(s));
}

void check_sizes(long long a, long long b, const char *what)
{
    if (a < 0 || b < 0) fail(SDL_ERR_INVALID, std::string(what) + ": negative size");
}

} // namespace
} // namespace sdl

using namespace sdl;

extern "C" void repeat(double *result, const double *a, int len, int repeats)
{
    guard_upstream_void("repeat", [&]() {
        check_sizes(len, repeats, "repeat");
        const long long n = (long long)len * repeats;
        if (!n) return;
        cudaStream_t s = S();
        DevBuf<double> da = up(a, len, s), dr((size_t)n);
        SDL_LAUNCH(k_repeat, grid_mini(n), 256, 0, s, dr.get(), da.get(), len, repeats);
        down(result, dr, n, s);
    });
}

extern "C" void tile_double(double *result, const double *a, int len, int tiles)
{
    guard_upstream_void("tile_double", [&]() {
        check_sizes(len, tiles, "tile_double");
        const long long n = (long long)len * tiles;
        if (!n) return;
        cudaStream_t s = S();
        DevBuf<double> da = up(a, len, s), dr((size_t)n);
        SDL_LAUNCH(k_tile, grid_mini(n), 256, 0, s, dr.get(), da.get(), len, tiles);
        down(result, dr, n, s);
    });
}

extern "C" void scaled_ones(double *result, int size, double value)
{
    guard_upstream_void("scaled_ones", [&]() {
        check_sizes(size, 0, "scaled_ones");
        if (!size) return;
        cudaStream_t s = S();
        DevBuf<double> dr((size_t)size);
        SDL_LAUNCH(k_fill, grid_mini(size), 256, 0, s, dr.get(), (long long)size, value);
        down(result, dr, size, s);
    });
}

extern "C" void A_transpose(double *AT, const double *A, int m, int n)
{
    guard_upstream_void("A_transpose", [&]() {
        check_sizes(m, n, "A_transpose");
        const long long N = (long long)m * n;
        if (!N) return;
        cudaStream_t s = S();
        DevBuf<double> dA = up(A, N, s), dT((size_t)N);
        SDL_LAUNCH(k_transpose_dense, grid_mini(N), 256, 0, s, dT.get(), dA.get(), m, n);
        down(AT, dT, N, s);
    });
}

extern "C" void Y_kron_I_vec(int m, int k, int n, const double *Y, const double *w, double *v)
{
    guard_upstream_void("Y_kron_I_vec", [&]() {
        check_sizes((long long)m * k, n, "Y_kron_I_vec");
        const long long N = (long long)m * k;
        if (!N) return;
        cudaStream_t s = S();
        DevBuf<double> dY = up(Y, (long long)k * n, s), dw = up(w, (long long)m * n, s), dv((size_t)N);
        SDL_LAUNCH(k_y_kron_i, grid_mini(N), 256, 0, s, m, k, n, dY.get(), dw.get(), dv.get());
        down(v, dv, N, s);
    });
}

extern "C" void I_kron_XT_vec(int m, int k, int n, const double *X, const double *w, double *v)
{
    guard_upstream_void("I_kron_XT_vec", [&]() {
        check_sizes((long long)k * n, m, "I_kron_XT_vec");
        const long long N = (long long)k * n;
        if (!N) return;
        cudaStream_t s = S();
        DevBuf<double> dX = up(X, (long long)m * k, s), dw = up(w, (long long)m * n, s), dv((size_t)N);
        SDL_LAUNCH(k_i_kron_xt, grid_mini(N), 256, 0, s, m, k, n, dX.get(), dw.get(), dv.get());
        down(v, dv, N, s);
    });
}
