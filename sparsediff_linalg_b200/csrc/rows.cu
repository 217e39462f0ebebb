// Row-wise copy kernels: row_gather (upstream src/sparse/sparse_matrix.c:79-134)
// and the diagonal row scaling C = diag(d) A (upstream src/sparse/CSR_matrix.c:86-97).
#include <algorithm>

#include "sdl_device.cuh"
#include "sdl_internal.h"

namespace sdl {
namespace {

__global__ void k_gather_lengths(const int *__restrict__ Ap, const int *__restrict__ map, int m_out,
                                 int *__restrict__ len)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < m_out;
         r += (long long)gridDim.x * blockDim.x)
    {
        int s = map[r];
        len[r] = Ap[s + 1] - Ap[s];
    }
}

template <class T>
__global__ void k_gather_segments(const int *__restrict__ Ap, const T *__restrict__ src,
                                  const int *__restrict__ map, const int *__restrict__ Cp, int m_out,
                                  T *__restrict__ dst)
{
    const int lane = lane_id(), wpb = blockDim.x >> 5;
    for (long long r = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); r < m_out;
         r += (long long)gridDim.x * wpb)
    {
        int s = Ap[map[r]];
        int c = Cp[r], len = Cp[r + 1] - c;
        for (int q = lane; q < len; q += 32) dst[c + q] = src[s + q];
    }
}

__global__ void k_scale_rows(const int *__restrict__ Ap, int m, const double *__restrict__ d,
                             const double *__restrict__ Ax, double *__restrict__ Cx)
{
    const int lane = lane_id(), wpb = blockDim.x >> 5;
    for (long long r = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); r < m;
         r += (long long)gridDim.x * wpb)
    {
        double dr = d[r];
        for (int q = Ap[r] + lane; q < Ap[r + 1]; q += 32) Cx[q] = __dmul_rn(Ax[q], dr);
    }
}

int grid_of(long long items, int per_block)
{
    Runtime &rt = runtime();
    long long g = (items + per_block - 1) / per_block;
    return (int)std::max<long long>(1, std::min<long long>(g, (long long)rt.num_sms * 16));
}

} // namespace

int gather_rows_structure(const int *d_Ap, const int *d_Ai, const int *d_map, int m_out,
                          DevBuf<int> &Cp, DevBuf<int> &Ci, cudaStream_t s)
{
    Cp.reset((size_t)m_out + 1);
    DevBuf<int> len(std::max(1, m_out));
    if (m_out > 0) SDL_LAUNCH(k_gather_lengths, grid_of(m_out, 256), 256, 0, s, d_Ap, d_map, m_out, len.get());
    int nnz = exclusive_scan_i32_checked(len.get(), Cp.get(), m_out, s);
    Ci.reset(std::max(1, nnz));
    if (nnz > 0)
        SDL_LAUNCH(k_gather_segments<int>, grid_of(m_out, 8), 256, 0, s, d_Ap, d_Ai, d_map, Cp.get(),
                   m_out, Ci.get());
    SDL_CUDA(cudaStreamSynchronize(s));
    return nnz;
}

void gather_rows_values(const int *d_Ap, const double *d_Ax, const int *d_map, const int *d_Cp,
                        int m_out, double *d_Cx, cudaStream_t s)
{
    if (m_out > 0)
        SDL_LAUNCH(k_gather_segments<double>, grid_of(m_out, 8), 256, 0, s, d_Ap, d_Ax, d_map, d_Cp,
                   m_out, d_Cx);
}

void scale_rows(const int *d_Ap, int m, const double *d_d, const double *d_Ax, double *d_Cx,
                cudaStream_t s)
{
    if (m > 0) SDL_LAUNCH(k_scale_rows, grid_of(m, 8), 256, 0, s, d_Ap, m, d_d, d_Ax, d_Cx);
}

} // namespace sdl
