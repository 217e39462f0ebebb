// Dense blocks times a sparse CSR on the GPU: C_k = B_k S[col_perm_k, :]
// (upstream src/permuted_dense/permuted_dense_linalg.c:313-430 BA_pd_csr_*,
// src/stacked_pd/stacked_pd_linalg.c:657-671 BA_spd_csr_*).
//
// Upstream's structure: C_k's columns are the union of the patterns of S's rows
// col_perm_k (ascending), and the fill sums, for every output (i, c), the terms
// B_k[i, r] * S[col_perm_k[r], c] over the compact CSC of S[col_perm_k, :] in its
// order (r ascending), from +0.0, one rounding per product and per sum. Here a
// warp computes whole output columns with its lanes on the block's rows, reading
// the block's columns contiguously from a transposed copy, and each output is
// summed in exactly that order (__dmul_rn / __dadd_rn: no FMA, as the upstream
// build has none). The kernel is bound by the writes of C.
#include <algorithm>
#include <climits>
#include <map>

#include "capi_common.h"
#include "dense_plan.h"
#include "sdl_device.cuh"

namespace sdl {
namespace {

int grid_cap(long long work_items, int per_block, int cap)
{
    long long g = (work_items + per_block - 1) / per_block;
    return (int)std::max<long long>(1, std::min<long long>(g, cap));
}

constexpr int BC_THREADS = 256;

__global__ void k_gather_vals(const int *__restrict__ pos, const double *__restrict__ Sx, long long n,
                              double *__restrict__ vals)
{
    for (long long d = blockIdx.x * (long long)blockDim.x + threadIdx.x; d < n;
         d += (long long)gridDim.x * blockDim.x)
        vals[d] = Sx[pos[d]];
}

// BT = the source blocks transposed (each n0 x m0 row-major), so that one column of
// a block is contiguous.
__global__ void k_transpose_blocks(const BlkDesc *__restrict__ descs, int nblk, const double *__restrict__ B,
                                   double *__restrict__ BT)
{
    __shared__ double t[32][33];
    const BlkDesc D = descs[blockIdx.z];
    const int i0 = blockIdx.y * 32, r0 = blockIdx.x * 32;
    if (i0 >= D.m0 || r0 >= D.n0_B) return;
    const double *src = B + D.b_off;
    double *dst = BT + D.b_off;
    for (int y = threadIdx.y; y < 32; y += blockDim.y)
    {
        const int i = i0 + y, r = r0 + threadIdx.x;
        if (i < D.m0 && r < D.n0_B) t[y][threadIdx.x] = src[(long long)i * D.n0_B + r];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y)
    {
        const int r = r0 + y, i = i0 + threadIdx.x;
        if (r < D.n0_B && i < D.m0) dst[(long long)r * D.m0 + i] = t[threadIdx.x][y];
    }
}

#ifndef SDL_BC_COLS
#define SDL_BC_COLS 32
#endif
constexpr int BC_COLS = SDL_BC_COLS; // output columns of a CTA tile
constexpr int BC_ROWS = 64; // block rows per pass (two per lane)

// One CTA: output columns [c0, c0 + 32) of one block; each warp takes four columns
// one after the other, its lanes the block's rows (two per lane): every term of a
// column is a broadcast (row r of the block, value of S) times a contiguous read of
// column r of the block (BT). The 64 x 32 results go through shared memory and are
// written row by row, 256 bytes per row.
__global__ void __launch_bounds__(BC_THREADS) k_blocks_csr(const BlkTile *__restrict__ tiles,
                                                           const BlkDesc *__restrict__ descs,
                                                           const int *__restrict__ cp_all,
                                                           const int *__restrict__ rows_all,
                                                           const double *__restrict__ vals_all,
                                                           const double *__restrict__ BT_vals,
                                                           double *__restrict__ C_vals)
{
    __shared__ double tile[BC_ROWS][BC_COLS + 1];
    const BlkTile t = tiles[blockIdx.x];
    const BlkDesc D = descs[t.blk];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int *cp = cp_all + D.cp_off;
    const int *rows = rows_all + D.d_off;
    const double *vals = vals_all + D.d_off;
    const double *BT = BT_vals + D.b_off;
    const int ncol = min(BC_COLS, D.n0_C - t.c0);
    for (int i0 = 0; i0 < D.m0; i0 += BC_ROWS)
    {
        const int ia = i0 + lane, ib = i0 + 32 + lane;
        for (int cl = warp; cl < BC_COLS; cl += BC_THREADS / 32)
        {
            double a0 = 0.0, a1 = 0.0;
            if (cl < ncol)
            {
                const int c = t.c0 + cl;
                const int d1 = cp[c + 1];
                for (int d = cp[c]; d < d1; ++d)
                {
                    const double *col = BT + (long long)rows[d] * D.m0;
                    const double v = vals[d];
                    if (ia < D.m0) a0 = __dadd_rn(a0, __dmul_rn(col[ia], v));
                    if (ib < D.m0) a1 = __dadd_rn(a1, __dmul_rn(col[ib], v));
                }
            }
            tile[lane][cl] = a0;
            tile[32 + lane][cl] = a1;
        }
        __syncthreads();
        const int nrow = min(BC_ROWS, D.m0 - i0);
        double *C = C_vals + D.c_off + (long long)i0 * D.n0_C + t.c0;
        for (int e = threadIdx.x; e < nrow * BC_COLS; e += BC_THREADS)
        {
            const int ri = e / BC_COLS, cl = e % BC_COLS;
            if (cl < ncol) C[(long long)ri * D.n0_C + cl] = tile[ri][cl];
        }
        __syncthreads();
    }
}

} // namespace

std::unique_ptr<BlocksCsrPlan> blocks_csr_build(int n_src, const int *m0, const int *n0,
                                                const int *const *col_perm, const int *Sp, const int *Si,
                                                int S_m, int S_n, bool keep_empty, cudaStream_t s)
{
    if (n_src < 0 || S_m < 0 || S_n < 0) fail(SDL_ERR_INVALID, "blocks x CSR: negative size");
    auto P = std::make_unique<BlocksCsrPlan>();
    P->S_m = S_m;
    P->S_n = S_n;
    P->S_nnz = S_m ? Sp[S_m] : 0;
    P->n_src = n_src;
    // compact CSCs, one per distinct col_perm (upstream builds one per block)
    struct Csc
    {
        std::vector<int> col_perm_C, cp, rows, pos;
        long long cp_off = 0, d_off = 0;
    };
    std::map<std::vector<int>, int> seen;
    std::vector<Csc> cscs;
    std::vector<int> csc_of(n_src);
    std::vector<int> mark(std::max(1, S_n));
    for (int k = 0; k < n_src; ++k)
    {
        if (m0[k] < 0 || n0[k] < 0) fail(SDL_ERR_INVALID, "blocks x CSR: negative block shape");
        std::vector<int> key(col_perm[k], col_perm[k] + n0[k]);
        for (int r = 0; r < n0[k]; ++r)
            if (key[r] < 0 || key[r] >= S_m || (r && key[r] <= key[r - 1]))
                fail(SDL_ERR_INVALID, "blocks x CSR: a col_perm is not strictly increasing rows of S");
        auto it = seen.find(key);
        if (it != seen.end())
        {
            csc_of[k] = it->second;
            continue;
        }
        Csc cc;
        std::fill(mark.begin(), mark.end(), -1);
        long long nnz_K = 0;
        for (int row : key)
        {
            for (int q = Sp[row]; q < Sp[row + 1]; ++q)
            {
                if (Si[q] < 0 || Si[q] >= S_n) fail(SDL_ERR_INVALID, "blocks x CSR: column index of S out of range");
                mark[Si[q]] = 0;
            }
            nnz_K += Sp[row + 1] - Sp[row];
        }
        if (nnz_K > INT_MAX) fail(SDL_ERR_OVERFLOW, "blocks x CSR: compact CSC exceeds INT_MAX entries");
        for (int j = 0; j < S_n; ++j)
            if (mark[j] >= 0)
            {
                mark[j] = (int)cc.col_perm_C.size();
                cc.col_perm_C.push_back(j);
            }
        const int n0C = (int)cc.col_perm_C.size();
        cc.cp.assign((size_t)n0C + 1, 0);
        for (int row : key)
            for (int q = Sp[row]; q < Sp[row + 1]; ++q) cc.cp[mark[Si[q]] + 1]++;
        for (int c = 0; c < n0C; ++c) cc.cp[c + 1] += cc.cp[c];
        cc.rows.resize((size_t)nnz_K);
        cc.pos.resize((size_t)nnz_K);
        std::vector<int> next(cc.cp.begin(), cc.cp.end() - 1);
        for (int r = 0; r < (int)key.size(); ++r)
            for (int q = Sp[key[r]]; q < Sp[key[r] + 1]; ++q)
            {
                const int dd = next[mark[Si[q]]]++;
                cc.rows[dd] = r;
                cc.pos[dd] = q;
            }
        csc_of[k] = (int)cscs.size();
        seen.emplace(std::move(key), csc_of[k]);
        cscs.push_back(std::move(cc));
    }
    long long cp_total = 0;
    for (Csc &cc : cscs)
    {
        cc.cp_off = cp_total;
        cc.d_off = P->d_total;
        cp_total += (long long)cc.cp.size();
        P->d_total += (long long)cc.rows.size();
    }
    std::vector<int> h_cp((size_t)std::max<long long>(1, cp_total)), h_rows((size_t)std::max<long long>(1, P->d_total)),
        h_pos((size_t)std::max<long long>(1, P->d_total));
    for (const Csc &cc : cscs)
    {
        std::copy(cc.cp.begin(), cc.cp.end(), h_cp.begin() + cc.cp_off);
        std::copy(cc.rows.begin(), cc.rows.end(), h_rows.begin() + cc.d_off);
        std::copy(cc.pos.begin(), cc.pos.end(), h_pos.begin() + cc.d_off);
    }
    // output blocks and their work tiles
    std::vector<BlkDesc> descs;
    std::vector<BlkTile> tiles;
    long long b_off = 0;
    for (int k = 0; k < n_src; ++k)
    {
        const Csc &cc = cscs[csc_of[k]];
        const int n0C = (int)cc.col_perm_C.size();
        const long long bk = (long long)m0[k] * n0[k];
        if ((n0C > 0 && m0[k] > 0) || keep_empty)
        {
            if ((long long)m0[k] * n0C > INT_MAX) fail(SDL_ERR_OVERFLOW, "blocks x CSR: output block exceeds INT_MAX values");
            BlkDesc D{};
            D.b_off = b_off;
            D.c_off = P->c_total;
            D.cp_off = cc.cp_off;
            D.d_off = cc.d_off;
            D.m0 = m0[k];
            D.n0_B = n0[k];
            D.n0_C = n0C;
            const int blk = (int)descs.size();
            for (int c0 = 0; c0 < n0C && m0[k] > 0; c0 += BC_COLS) tiles.push_back(BlkTile{blk, c0});
            descs.push_back(D);
            P->src.push_back(k);
            P->col_perm.push_back(cc.col_perm_C);
            P->m0.push_back(m0[k]);
            P->n0_C.push_back(n0C);
            P->c_total += (long long)m0[k] * n0C;
        }
        b_off += bk;
    }
    P->b_total = b_off;
    P->ntiles = (int)tiles.size();
    P->cp = upload(h_cp.data(), h_cp.size(), s);
    P->rows = upload(h_rows.data(), h_rows.size(), s);
    P->pos = upload(h_pos.data(), h_pos.size(), s);
    P->vals.reset((size_t)std::max<long long>(1, P->d_total));
    P->BT.reset((size_t)std::max<long long>(1, P->b_total));
    // transpose work: every block as 32 x 32 tiles (grid.z = output block)
    for (size_t q = 0; q < descs.size(); ++q)
    {
        P->tr_x = std::max(P->tr_x, (descs[q].n0_B + 31) / 32);
        P->tr_y = std::max(P->tr_y, (descs[q].m0 + 31) / 32);
    }
    P->desc = upload(descs.data(), std::max<size_t>(1, descs.size()), s);
    P->tiles = upload(tiles.data(), std::max<size_t>(1, tiles.size()), s);
    SDL_CUDA(cudaStreamSynchronize(s));
    return P;
}

void blocks_csr_fill(const BlocksCsrPlan &P, const double *B_vals, const double *S_x, double *C_vals,
                     cudaStream_t s)
{
    if (P.ntiles == 0) return;
    Runtime &rt = runtime();
    if (P.d_total > 0)
        SDL_LAUNCH(k_gather_vals, grid_cap(P.d_total, 256, rt.num_sms * 8), 256, 0, s, P.pos.get(), S_x,
                   P.d_total, P.vals.get());
    // the output blocks' sources, transposed (a source feeding two outputs is
    // transposed twice: outputs and sources are one to one here)
    const dim3 tg(std::max(1, P.tr_x), std::max(1, P.tr_y), (unsigned)P.src.size());
    SDL_LAUNCH(k_transpose_blocks, tg, dim3(32, 8), 0, s, P.desc.get(), (int)P.src.size(), B_vals, P.BT.get());
    SDL_LAUNCH(k_blocks_csr, P.ntiles, BC_THREADS, 0, s, P.tiles.get(), P.desc.get(), P.cp.get(),
               P.rows.get(), P.vals.get(), P.BT.get(), C_vals);
}

} // namespace sdl
