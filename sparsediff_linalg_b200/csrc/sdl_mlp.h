// Shapes and host entry points of the learned row scheduler (mlp.cu).
#pragma once

#include "sdl_internal.h"
#ifdef __CUDACC__
#include "sdl_device.cuh"
#endif

namespace sdl {

constexpr int MLP_IN = 8, MLP_H = 32, MLP_OUT = 4;
// parameter layout (row-major weights, W[out][in])
constexpr int MLP_W1 = 0;
constexpr int MLP_B1 = MLP_W1 + MLP_H * MLP_IN;
constexpr int MLP_W2 = MLP_B1 + MLP_H;
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;
constexpr int MLP_W3 = MLP_B2 + MLP_H;
constexpr int MLP_B3 = MLP_W3 + MLP_OUT * MLP_H;
constexpr int MLP_NPARAMS = MLP_B3 + MLP_OUT;

// accumulator class of a row with `nnz` outputs (the classifier's label)
__host__ __device__ inline int mlp_class_of(long long nnz) { return nnz <= 512 ? 0 : nnz <= 8192 ? 1 : 2; }

struct Mlp
{
    DevBuf<float> params, m1, m2, grad;
    explicit Mlp(unsigned long long seed);
};

// Features (n_rows x MLP_IN) of every output row of the product, and with Cp the
// labels (n_rows x 2: log1p(nnz), class) the exact symbolic pass produced.
void row_features(const ProductDesc &d, const int *Cp, float *feat, float *label, cudaStream_t s);
// Loss and gradient (device, MLP_NPARAMS floats) of the mean loss over rows idx[0..n)
// (idx may be null: rows 0..n). Synchronises.
float mlp_gradient(const Mlp &net, const float *feat, const float *label, const int *idx, int n,
                   float *grad_out_dev, cudaStream_t s);
// Adam over shuffled mini-batches; returns the mean loss of the last epoch.
float mlp_train(Mlp &net, const float *feat, const float *label, long long n, int epochs, int batch,
                float lr, unsigned long long seed, cudaStream_t s);
// out (n x MLP_OUT): raw outputs (log1p(nnz), 3 class logits).
void mlp_predict(const Mlp &net, const float *feat, long long n, float *out, cudaStream_t s);

#ifdef __CUDACC__
// Inference by one warp: lane q < MLP_IN holds feature q; lane j computes hidden
// unit j; on return lanes 0..3 hold the four outputs. Same summation order as the
// training kernel (bias first, inputs ascending).
__device__ __forceinline__ float mlp_row_forward(const float *P, float f)
{
    const int lane = lane_id();
    float a = P[MLP_B1 + lane];
#pragma unroll
    for (int q = 0; q < MLP_IN; ++q) a += P[MLP_W1 + lane * MLP_IN + q] * __shfl_sync(FULL_MASK, f, q);
    const float h1 = a > 0.f ? a : 0.f;
    float a2 = P[MLP_B2 + lane];
#pragma unroll 8
    for (int q = 0; q < MLP_H; ++q) a2 += P[MLP_W2 + lane * MLP_H + q] * __shfl_sync(FULL_MASK, h1, q);
    const float h2 = a2 > 0.f ? a2 : 0.f;
    const int o = lane & (MLP_OUT - 1);
    float a3 = P[MLP_B3 + o];
#pragma unroll 8
    for (int q = 0; q < MLP_H; ++q) a3 += P[MLP_W3 + o * MLP_H + q] * __shfl_sync(FULL_MASK, h2, q);
    return a3;
}
#endif

} // namespace sdl
