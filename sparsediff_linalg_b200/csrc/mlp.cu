// Learned row scheduler: an 8 -> 32 -> 32 -> 4 FP32 MLP over per-row statistics of
// a row-wise product that predicts the row's output size (log1p(nnz), regression)
// and its accumulator class (3 logits: <= 512, <= 8192, > 8192 outputs). Training
// and inference are this file's own CUDA kernels:
//   * k_row_features: per output row, the features the exact symbolic pass knows
//     before it runs (L-row length, term count = sum of referenced A-row lengths,
//     longest referenced A row, A's width) and, optionally, the labels it produces;
//   * k_mlp_train_step: forward + backward of a mini-batch, one sample per thread,
//     weight gradients reduced across each warp with shuffles and then across the
//     grid with atomics; k_adam: the Adam update;
//   * k_mlp_predict / mlp_row_forward: inference, one warp per row with one
//     hidden unit per lane (fused into the learned row-binning kernel).
// The schedule is the only thing the network changes: the exact symbolic pass
// stays the fallback and the judge (see product_symbolic_learned).
#include <cmath>
#include <vector>

#include "sdl_device.cuh"
#include "sdl_internal.h"
#include "sdl_mlp.h"

namespace sdl {
namespace {

__device__ __forceinline__ float relu(float v) { return v > 0.f ? v : 0.f; }

// features of one output row (layout shared with the CPU oracle, oracle/mlp_oracle.py)
__device__ __forceinline__ void row_features(int lrow_len, long long ub, int maxlen, int n, float *f)
{
    float lu = log1pf((float)ub);
    float lm = log1pf((float)maxlen);
    float ln = log1pf((float)n);
    f[0] = log1pf((float)lrow_len);
    f[1] = lu;
    f[2] = lm;
    f[3] = ln;
    f[4] = fminf(4.f, (float)ub / (float)max(1, n));
    f[5] = lu - lm;
    f[6] = lu - ln;
    f[7] = 1.f;
}

__global__ void k_row_features(const int *__restrict__ Lp, const int *__restrict__ Li, int L_m, int n_L,
                               int m_out, const int *__restrict__ Ap, int n, const int *__restrict__ Cp,
                               float *__restrict__ feat, float *__restrict__ label)
{
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
        if (lane == 0)
        {
            float f[MLP_IN];
            row_features(Lp[r + 1] - Lp[r], sum, mx, n, f);
            for (int q = 0; q < MLP_IN; ++q) feat[row * MLP_IN + q] = f[q];
            if (label && Cp)
            {
                int nnz = Cp[row + 1] - Cp[row];
                label[row * 2 + 0] = log1pf((float)nnz);
                label[row * 2 + 1] = (float)mlp_class_of(nnz);
            }
        }
    }
}

// Forward + backward of one mini-batch (sample per thread). Gradients are summed
// over the warp with shuffles, then added to the global gradient with one atomic
// per warp and parameter.
__global__ void k_mlp_train_step(const float *__restrict__ P, const float *__restrict__ feat,
                                 const float *__restrict__ label, const int *__restrict__ idx, int nb,
                                 float inv_n, float *__restrict__ grad, float *__restrict__ loss)
{
    extern __shared__ float sp[]; // parameters
    for (int q = threadIdx.x; q < MLP_NPARAMS; q += blockDim.x) sp[q] = P[q];
    __syncthreads();
    const float *W1 = sp + MLP_W1, *b1 = sp + MLP_B1, *W2 = sp + MLP_W2, *b2 = sp + MLP_B2,
                *W3 = sp + MLP_W3, *b3 = sp + MLP_B3;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = s < nb;
    float x[MLP_IN], z1[MLP_H], h1[MLP_H], z2[MLP_H], h2[MLP_H], y[MLP_OUT], dy[MLP_OUT];
    float l = 0.f;
    if (valid)
    {
        const int r = idx ? idx[s] : s;
        for (int q = 0; q < MLP_IN; ++q) x[q] = feat[(long long)r * MLP_IN + q];
        for (int j = 0; j < MLP_H; ++j)
        {
            float a = b1[j];
            for (int q = 0; q < MLP_IN; ++q) a += W1[j * MLP_IN + q] * x[q];
            z1[j] = a;
            h1[j] = relu(a);
        }
        for (int j = 0; j < MLP_H; ++j)
        {
            float a = b2[j];
            for (int q = 0; q < MLP_H; ++q) a += W2[j * MLP_H + q] * h1[q];
            z2[j] = a;
            h2[j] = relu(a);
        }
        for (int o = 0; o < MLP_OUT; ++o)
        {
            float a = b3[o];
            for (int q = 0; q < MLP_H; ++q) a += W3[o * MLP_H + q] * h2[q];
            y[o] = a;
        }
        const float t0 = label[(long long)r * 2], tc = label[(long long)r * 2 + 1];
        const float e = y[0] - t0;
        float m = fmaxf(y[1], fmaxf(y[2], y[3]));
        float p1 = expf(y[1] - m), p2 = expf(y[2] - m), p3 = expf(y[3] - m);
        float z = p1 + p2 + p3;
        p1 /= z;
        p2 /= z;
        p3 /= z;
        int c = (int)tc;
        float pc = c == 0 ? p1 : c == 1 ? p2 : p3;
        l = 0.5f * e * e - logf(fmaxf(pc, 1e-30f));
        dy[0] = e * inv_n;
        dy[1] = (p1 - (c == 0 ? 1.f : 0.f)) * inv_n;
        dy[2] = (p2 - (c == 1 ? 1.f : 0.f)) * inv_n;
        dy[3] = (p3 - (c == 2 ? 1.f : 0.f)) * inv_n;
    }
    else
    {
        for (int q = 0; q < MLP_IN; ++q) x[q] = 0.f;
        for (int j = 0; j < MLP_H; ++j) z1[j] = h1[j] = z2[j] = h2[j] = 0.f;
        for (int o = 0; o < MLP_OUT; ++o) dy[o] = 0.f;
    }
    // warp-reduce a gradient term and add it once per warp
    auto acc = [&](int at, float v) {
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
        if (lane_id() == 0 && v != 0.f) atomicAdd(&grad[at], v);
    };
    // layer 3
    float dh2[MLP_H];
    for (int q = 0; q < MLP_H; ++q) dh2[q] = 0.f;
    for (int o = 0; o < MLP_OUT; ++o)
    {
        acc(MLP_B3 + o, dy[o]);
        for (int q = 0; q < MLP_H; ++q)
        {
            acc(MLP_W3 + o * MLP_H + q, dy[o] * h2[q]);
            dh2[q] += W3[o * MLP_H + q] * dy[o];
        }
    }
    // layer 2
    float dz2[MLP_H], dh1[MLP_H];
    for (int j = 0; j < MLP_H; ++j) dz2[j] = z2[j] > 0.f ? dh2[j] : 0.f;
    for (int q = 0; q < MLP_H; ++q) dh1[q] = 0.f;
    for (int j = 0; j < MLP_H; ++j)
    {
        acc(MLP_B2 + j, dz2[j]);
        for (int q = 0; q < MLP_H; ++q)
        {
            acc(MLP_W2 + j * MLP_H + q, dz2[j] * h1[q]);
            dh1[q] += W2[j * MLP_H + q] * dz2[j];
        }
    }
    // layer 1
    for (int j = 0; j < MLP_H; ++j)
    {
        float dz1 = z1[j] > 0.f ? dh1[j] : 0.f;
        acc(MLP_B1 + j, dz1);
        for (int q = 0; q < MLP_IN; ++q) acc(MLP_W1 + j * MLP_IN + q, dz1 * x[q]);
    }
    // loss (mean over the batch)
    float lv = l * inv_n;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) lv += __shfl_xor_sync(FULL_MASK, lv, o);
    if (lane_id() == 0 && loss) atomicAdd(loss, lv);
}

__global__ void k_adam(float *__restrict__ P, const float *__restrict__ g, float *__restrict__ m1,
                       float *__restrict__ m2, float lr, float b1c, float b2c)
{
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < MLP_NPARAMS; q += gridDim.x * blockDim.x)
    {
        float gq = g[q];
        float a = beta1 * m1[q] + (1.f - beta1) * gq;
        float b = beta2 * m2[q] + (1.f - beta2) * gq * gq;
        m1[q] = a;
        m2[q] = b;
        P[q] -= lr * (a / b1c) / (sqrtf(b / b2c) + eps);
    }
}

__global__ void k_mlp_predict(const float *__restrict__ P, const float *__restrict__ feat, long long n,
                              float *__restrict__ out)
{
    extern __shared__ float sp[];
    for (int q = threadIdx.x; q < MLP_NPARAMS; q += blockDim.x) sp[q] = P[q];
    __syncthreads();
    const int wpb = blockDim.x >> 5;
    for (long long row = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); row < n;
         row += (long long)gridDim.x * wpb)
    {
        float f = lane_id() < MLP_IN ? feat[row * MLP_IN + lane_id()] : 0.f;
        float y = mlp_row_forward(sp, f);
        if (lane_id() < MLP_OUT) out[row * MLP_OUT + lane_id()] = y;
    }
}

} // namespace

// ------------------------------------------------------------------ host side
Mlp::Mlp(unsigned long long seed)
{
    params.reset(MLP_NPARAMS);
    m1.reset(MLP_NPARAMS);
    m2.reset(MLP_NPARAMS);
    grad.reset(MLP_NPARAMS);
    std::vector<float> h(MLP_NPARAMS, 0.f);
    // He-uniform initialisation from a splitmix64 stream (deterministic per seed)
    unsigned long long st = seed ? seed : 0x9e3779b97f4a7c15ULL;
    auto next = [&]() {
        st += 0x9e3779b97f4a7c15ULL;
        unsigned long long z = st;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int at, int count, int fan_in) {
        double lim = std::sqrt(6.0 / fan_in);
        for (int q = 0; q < count; ++q) h[at + q] = (float)((2.0 * next() - 1.0) * lim);
    };
    fill(MLP_W1, MLP_H * MLP_IN, MLP_IN);
    fill(MLP_W2, MLP_H * MLP_H, MLP_H);
    fill(MLP_W3, MLP_OUT * MLP_H, MLP_H);
    cudaStream_t s = runtime().stream;
    SDL_CUDA(cudaMemcpyAsync(params.get(), h.data(), MLP_NPARAMS * 4, cudaMemcpyHostToDevice, s));
    SDL_CUDA(cudaMemsetAsync(m1.get(), 0, MLP_NPARAMS * 4, s));
    SDL_CUDA(cudaMemsetAsync(m2.get(), 0, MLP_NPARAMS * 4, s));
    SDL_CUDA(cudaStreamSynchronize(s));
}

void row_features(const ProductDesc &d, const int *Cp, float *feat, float *label, cudaStream_t s)
{
    Runtime &rt = runtime();
    long long m_out = (long long)d.L_m * d.blocks;
    if (m_out == 0) return;
    int grid = (int)std::max<long long>(1, std::min<long long>((m_out + 7) / 8, rt.num_sms * 16LL));
    SDL_LAUNCH(k_row_features, grid, 256, 0, s, d.Lp, d.Li, d.L_m, d.A_m / d.blocks, (int)m_out, d.Ap,
               d.A_n, Cp, feat, label);
}

float mlp_gradient(const Mlp &net, const float *feat, const float *label, const int *idx, int n,
                   float *grad_out_dev, cudaStream_t s)
{
    DevBuf<float> loss(1);
    SDL_CUDA(cudaMemsetAsync(grad_out_dev, 0, MLP_NPARAMS * 4, s));
    SDL_CUDA(cudaMemsetAsync(loss.get(), 0, 4, s));
    if (n > 0)
        SDL_LAUNCH(k_mlp_train_step, (n + 255) / 256, 256, MLP_NPARAMS * 4, s, net.params.get(), feat,
                   label, idx, n, 1.f / (float)n, grad_out_dev, loss.get());
    float h = 0.f;
    SDL_CUDA(cudaMemcpyAsync(&h, loss.get(), 4, cudaMemcpyDeviceToHost, s));
    SDL_CUDA(cudaStreamSynchronize(s));
    return h;
}

float mlp_train(Mlp &net, const float *feat, const float *label, long long n, int epochs, int batch,
                float lr, unsigned long long seed, cudaStream_t s)
{
    if (n <= 0) return 0.f;
    // a fixed shuffled order per epoch (host permutation, uploaded once)
    std::vector<int> perm((size_t)n);
    for (long long q = 0; q < n; ++q) perm[q] = (int)q;
    unsigned long long st = seed * 2654435761ULL + 1;
    DevBuf<int> didx((size_t)n);
    DevBuf<float> loss(1);
    float last = 0.f;
    long long step = 0;
    for (int ep = 0; ep < epochs; ++ep)
    {
        for (long long q = n - 1; q > 0; --q)
        {
            st = st * 6364136223846793005ULL + 1442695040888963407ULL;
            long long j = (long long)((st >> 33) % (unsigned long long)(q + 1));
            std::swap(perm[q], perm[j]);
        }
        SDL_CUDA(cudaMemcpyAsync(didx.get(), perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
        SDL_CUDA(cudaMemsetAsync(loss.get(), 0, 4, s));
        int nbatches = 0;
        for (long long b0 = 0; b0 < n; b0 += batch)
        {
            int nb = (int)std::min<long long>(batch, n - b0);
            SDL_CUDA(cudaMemsetAsync(net.grad.get(), 0, MLP_NPARAMS * 4, s));
            SDL_LAUNCH(k_mlp_train_step, (nb + 255) / 256, 256, MLP_NPARAMS * 4, s, net.params.get(), feat,
                       label, didx.get() + b0, nb, 1.f / (float)nb, net.grad.get(), loss.get());
            ++step;
            float b1c = 1.f - std::pow(0.9f, (float)step), b2c = 1.f - std::pow(0.999f, (float)step);
            SDL_LAUNCH(k_adam, (MLP_NPARAMS + 255) / 256, 256, 0, s, net.params.get(), net.grad.get(),
                       net.m1.get(), net.m2.get(), lr, b1c, b2c);
            ++nbatches;
        }
        float h = 0.f;
        SDL_CUDA(cudaMemcpyAsync(&h, loss.get(), 4, cudaMemcpyDeviceToHost, s));
        SDL_CUDA(cudaStreamSynchronize(s));
        last = h / (float)std::max(1, nbatches);
    }
    return last;
}

void mlp_predict(const Mlp &net, const float *feat, long long n, float *out, cudaStream_t s)
{
    if (n <= 0) return;
    Runtime &rt = runtime();
    int grid = (int)std::max<long long>(1, std::min<long long>((n + 7) / 8, rt.num_sms * 16LL));
    SDL_LAUNCH(k_mlp_predict, grid, 256, MLP_NPARAMS * 4, s, net.params.get(), feat, n, out);
}

} // namespace sdl
