// A^T diag(d) A of dense blocks on the FP64 tensor cores (upstream
// src/permuted_dense/permuted_dense_linalg.c:87-112 ATA_pd_* / ATDA_pd_*, and
// src/stacked_pd/stacked_pd_linalg.c:197-237 ATA_spd_* / ATDA_spd_* with the
// coalescing of src/stacked_pd/stacked_pd_coalesce.c:150-381).
//
// Upstream forms dwork = diag(d_perm) X (one rounding per product) and calls
// cblas_dgemm for X^T dwork, whose summation order BLAS leaves unspecified; here
// the same dwork products feed mma.sync.m8n8k4 f64 tiles (the K loop in ascending
// row order). Partials are then summed cell by cell in upstream's block order,
// from +0.0. The dgemm part is therefore equal to upstream's within rounding
// (tests compare at 1e-12 of the sum of |terms|), everything around it exactly.
#include <algorithm>
#include <climits>
#include <map>

#include "capi_common.h"
#include "dense_plan.h"

namespace sdl {
namespace {

int grid_cap2(long long work_items, int per_block, int cap)
{
    long long g = (work_items + per_block - 1) / per_block;
    return (int)std::max<long long>(1, std::min<long long>(g, cap));
}

__device__ __forceinline__ void mma_f64(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// One CTA (4 warps) per 64 x 64 tile (a0, b0) of partial P_k = X^T diag(d_perm) X.
// The block's rows are taken ATA_KC at a time through a two-stage cp.async
// pipeline: columns a0.. and b0.. of the next ATA_KC rows (and their d values) are
// copied into shared memory while the current ones feed the tensor cores. Each
// warp runs its 32 x 32 quarter as 4 x 4 m8n8k4 accumulators: per step of 4 rows,
// 4 A and 4 B fragments from shared memory feed 16 MMAs. The B fragments are
// dwork = d * X, formed as they are read (upstream's one rounding per product). The
// K order (rows ascending, 4 per MMA) is the same for every output.
//   A fragment (8 x 4, row-major): lane holds A[lane / 4][lane % 4] = X[k + lane % 4][a + lane / 4]
//   B fragment (4 x 8, col-major): lane holds B[lane % 4][lane / 4] = d * X[k + lane % 4][b + lane / 4]
//   C (8 x 8): lane holds C[lane / 4][2 (lane % 4) + {0, 1}]
constexpr int ATA_T = 64;   // output tile edge
constexpr int ATA_KC = 16;  // rows staged at a time
constexpr int ATA_LD = 68;  // shared row stride (doubles)
constexpr int ATA_STAGE = 2 * ATA_KC * ATA_LD + ATA_KC; // A panel, B panel, d values
constexpr int ATA_SMEM = 2 * ATA_STAGE * (int)sizeof(double);

__device__ __forceinline__ unsigned ata_smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void ata_cp8(double *dst, const double *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(ata_smem_u32(dst)), "l"(src));
}

// Copies rows k0 .. k0 + ATA_KC - 1 of the tile's two column panels (zeros past
// the block's rows or columns) and the rows' d values into one stage.
__device__ __forceinline__ void ata_stage(double *st, const double *X, const int *rp, const double *d, int m0,
                                          int n0, int a0, int b0, int k0)
{
    double *As = st, *Bs = st + ATA_KC * ATA_LD, *ds = st + 2 * ATA_KC * ATA_LD;
#pragma unroll 4
    for (int e = threadIdx.x; e < ATA_KC * ATA_T; e += 128)
    {
        const int r = e / ATA_T, col = e % ATA_T;
        const int i = k0 + r;
        const double *row = X + (long long)i * n0;
        if (i < m0 && a0 + col < n0)
            ata_cp8(&As[r * ATA_LD + col], row + a0 + col);
        else
            As[r * ATA_LD + col] = 0.0;
        if (i < m0 && b0 + col < n0)
            ata_cp8(&Bs[r * ATA_LD + col], row + b0 + col);
        else
            Bs[r * ATA_LD + col] = 0.0;
    }
    if (d && threadIdx.x < ATA_KC)
    {
        const int i = k0 + threadIdx.x;
        if (i < m0)
            ata_cp8(&ds[threadIdx.x], d + rp[i]);
        else
            ds[threadIdx.x] = 0.0;
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__global__ void __launch_bounds__(128) k_ata_partials(const int4 *__restrict__ mtiles, int nmt,
                                                      const long long *__restrict__ x_off,
                                                      const long long *__restrict__ p_off,
                                                      const int *__restrict__ m0d, const int *__restrict__ n0d,
                                                      const int *__restrict__ rowperm_all,
                                                      const long long *__restrict__ rowperm_off,
                                                      const double *__restrict__ X_vals,
                                                      const double *__restrict__ d, double *__restrict__ P)
{
    extern __shared__ double ata_sm[];
    if (blockIdx.x >= nmt) return;
    const int4 t = mtiles[blockIdx.x];
    const int k = t.x, a0 = t.y, b0 = t.z;
    const int m0 = m0d[k], n0 = n0d[k];
    const double *X = X_vals + x_off[k];
    const int *rp = rowperm_all + rowperm_off[k];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, q = lane & 3;
    const int wa = 32 * (w >> 1), wb = 32 * (w & 1);
    double c[4][4][2] = {};
    const int nch = (m0 + ATA_KC - 1) / ATA_KC;
    if (nch > 0) ata_stage(ata_sm, X, rp, d, m0, n0, a0, b0, 0);
    for (int ch = 0; ch < nch; ++ch)
    {
        if (ch + 1 < nch)
        {
            ata_stage(ata_sm + ((ch + 1) & 1) * ATA_STAGE, X, rp, d, m0, n0, a0, b0, (ch + 1) * ATA_KC);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        }
        else
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();
        const double *As = ata_sm + (ch & 1) * ATA_STAGE;
        const double *Bs = As + ATA_KC * ATA_LD, *ds = As + 2 * ATA_KC * ATA_LD;
        const int kend = min(ATA_KC, m0 - ch * ATA_KC);
        for (int kk = 0; kk < kend; kk += 4)
        {
            double af[4], bf[4];
            const double dq = d ? ds[kk + q] : 1.0;
#pragma unroll
            for (int h = 0; h < 4; ++h)
            {
                af[h] = As[(kk + q) * ATA_LD + wa + 8 * h + g];
                const double x = Bs[(kk + q) * ATA_LD + wb + 8 * h + g];
                bf[h] = d ? __dmul_rn(x, dq) : x; // dwork = diag(d_perm) X, as upstream
            }
#pragma unroll
            for (int ha = 0; ha < 4; ++ha)
#pragma unroll
                for (int hb = 0; hb < 4; ++hb) mma_f64(c[ha][hb][0], c[ha][hb][1], af[ha], bf[hb]);
        }
        __syncthreads(); // this stage is free for the chunk after next
    }
    double *Pk = P + p_off[k];
#pragma unroll
    for (int ha = 0; ha < 4; ++ha)
#pragma unroll
        for (int hb = 0; hb < 4; ++hb)
#pragma unroll
            for (int e = 0; e < 2; ++e)
            {
                const int r = a0 + wa + 8 * ha + g, cc = b0 + wb + 8 * hb + 2 * q + e;
                if (r < n0 && cc < n0) Pk[(long long)r * n0 + cc] = c[ha][hb][e];
            }
}

// One warp per (block k, active column c of B): row c of the partial,
// P_k[c, j] = sum over B's column c (CSC order, rows of block k only) of
// B.x * (d[row] * X_k[kk, j]) -- upstream's two roundings -- or B.x * X_k[kk, j]
// without d, from +0.0. Lanes take the columns j of the block.
__global__ void __launch_bounds__(256) k_btda_partials(const int2 *__restrict__ wtask, int nwt,
                                                       const int *__restrict__ ent_off, const int *__restrict__ ent_kk,
                                                       const int *__restrict__ ent_pos,
                                                       const long long *__restrict__ x_off,
                                                       const long long *__restrict__ p_off,
                                                       const int *__restrict__ m0d, const int *__restrict__ n0d,
                                                       const int *__restrict__ rowperm_all,
                                                       const long long *__restrict__ rowperm_off,
                                                       const double *__restrict__ X_vals, const double *__restrict__ d,
                                                       const double *__restrict__ Bx, int B_nnz,
                                                       double *__restrict__ P, int *__restrict__ err)
{
    const int t = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (t >= nwt) return;
    const int lane = threadIdx.x & 31;
    const int2 wt = wtask[t];
    const int k = wt.x, a = wt.y;
    const int m0 = m0d[k], n0 = n0d[k];
    const double *X = X_vals + x_off[k];
    const int *rp = rowperm_all + rowperm_off[k];
    const int e0 = ent_off[t], e1 = ent_off[t + 1];
    double *Pk = P + p_off[k] + (long long)a * n0;
    for (int j = lane; j < n0; j += 32)
    {
        double acc = 0.0;
        for (int e = e0; e < e1; ++e)
        {
            const int kk = ent_kk[e], pos = ent_pos[e];
            if (kk < 0 || kk >= m0 || pos < 0 || pos >= B_nnz)
            {
                atomicOr(err, 1);
                continue;
            }
            const double x = X[(long long)kk * n0 + j];
            const double w = d ? __dmul_rn(d[rp[kk]], x) : x;
            acc = __dadd_rn(acc, __dmul_rn(Bx[pos], w));
        }
        Pk[j] = acc;
    }
}

// Output cells: the partials that hold the cell, summed from +0.0 in block order.
// A CTA takes GATHER_THREADS consecutive cells of one output block (one per
// thread); the sources' partial offsets and strides are staged in shared memory
// GATHER_CHUNK at a time, and each thread issues the loads of GATHER_BATCH sources
// before it adds them, so the partials (just written, mostly in L2) stream with
// that many loads in flight per thread instead of one. An absent cell reads as
// -0.0, which leaves every round-to-nearest sum bit-for-bit unchanged (x + -0.0 = x,
// +0.0 + -0.0 = +0.0), so the sum equals the one that skips it.
constexpr int GATHER_THREADS = 256;
constexpr int GATHER_CHUNK = 64;
constexpr int GATHER_BATCH = 16;

__global__ void __launch_bounds__(GATHER_THREADS) k_ata_gather(const BlocksAtaPlan::OutDesc *__restrict__ outd,
                                                               int o_base, const int *__restrict__ srcs,
                                                               const int *__restrict__ maps,
                                                               const long long *__restrict__ p_off,
                                                               const int *__restrict__ n0d,
                                                               const double *__restrict__ P,
                                                               double *__restrict__ C)
{
    __shared__ long long sbase[GATHER_CHUNK];
    __shared__ int sn0[GATHER_CHUNK];
    const BlocksAtaPlan::OutDesc D = outd[o_base + blockIdx.y];
    const long long cells = (long long)D.m0 * D.n0;
    const int ms = D.m0 + D.n0;
    for (long long eb = (long long)blockIdx.x * GATHER_THREADS; eb < cells;
         eb += (long long)gridDim.x * GATHER_THREADS)
    {
        const long long e = eb + threadIdx.x;
        const bool live = e < cells;
        const int i = live ? (int)(e / D.n0) : 0;
        const int j = live ? (int)(e - (long long)i * D.n0) : 0;
        double acc = 0.0;
        for (int t0 = D.s_begin; t0 < D.s_end; t0 += GATHER_CHUNK)
        {
            const int nt = min(GATHER_CHUNK, D.s_end - t0);
            __syncthreads();
            if (threadIdx.x < nt)
            {
                const int k = srcs[t0 + threadIdx.x];
                sbase[threadIdx.x] = p_off[k];
                sn0[threadIdx.x] = n0d[k];
            }
            __syncthreads();
            if (!live) continue;
            const int *mp = maps + D.map_off + (long long)(t0 - D.s_begin) * ms;
            for (int u0 = 0; u0 < nt; u0 += GATHER_BATCH)
            {
                double v[GATHER_BATCH];
#pragma unroll
                for (int u = 0; u < GATHER_BATCH; ++u)
                {
                    v[u] = -0.0;
                    if (u0 + u < nt)
                    {
                        if (D.direct)
                            v[u] = P[sbase[u0 + u] + e];
                        else
                        {
                            const int *m = mp + (long long)(u0 + u) * ms;
                            const int si = m[i], sj = m[D.m0 + j];
                            if (si >= 0 && sj >= 0) v[u] = P[sbase[u0 + u] + (long long)si * sn0[u0 + u] + sj];
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < GATHER_BATCH; ++u)
                    if (u0 + u < nt) acc = __dadd_rn(acc, v[u]);
            }
        }
        if (live) C[D.c_off + e] = acc;
    }
}

} // namespace

// Upstream's coalescing of per-block partials (src/stacked_pd/stacked_pd_coalesce.c:
// 150-381): partial k covers rows prow[k] x columns pcol[k] (both ascending) of a
// nrows x ncols result. The signature of a row is the list of partials holding it,
// in partial order; rows with the same signature form one output block (blocks in
// order of first appearance scanning rows ascending), whose columns are the union
// of those partials' columns. Fills the output blocks of P and, per output block
// and contributing partial, its row and column maps (-1: absent).
void coalesce_partials(const std::vector<std::vector<int>> &prow, const std::vector<std::vector<int>> &pcol,
                       int nrows, int ncols, BlocksAtaPlan &P, std::vector<BlocksAtaPlan::OutDesc> &od,
                       std::vector<int> &h_srcs, std::vector<int> &h_maps)
{
    const int n_src = (int)prow.size();
    std::vector<std::vector<int>> row_blocks(std::max(1, nrows));
    for (int k = 0; k < n_src; ++k)
        for (int r : prow[k]) row_blocks[r].push_back(k);
    std::map<std::vector<int>, int> sig_id;
    P.out_rows.clear();
    P.out_cols.clear();
    P.out_srcs.clear();
    for (int r = 0; r < nrows; ++r)
    {
        if (row_blocks[r].empty()) continue;
        auto it = sig_id.find(row_blocks[r]);
        int sid;
        if (it == sig_id.end())
        {
            sid = (int)P.out_rows.size();
            sig_id.emplace(row_blocks[r], sid);
            P.out_rows.emplace_back();
            P.out_srcs.push_back(row_blocks[r]);
        }
        else
            sid = it->second;
        P.out_rows[sid].push_back(r);
    }
    P.n_out = (int)P.out_rows.size();
    P.c_total = 0;
    std::vector<int> rpos(std::max(1, nrows), -1), cpos(std::max(1, ncols), -1);
    for (int o = 0; o < P.n_out; ++o)
    {
        std::vector<int> cols;
        for (int k : P.out_srcs[o]) cols.insert(cols.end(), pcol[k].begin(), pcol[k].end());
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        P.out_cols.push_back(cols);
        BlocksAtaPlan::OutDesc D{};
        D.c_off = P.c_total;
        D.m0 = (int)P.out_rows[o].size();
        D.n0 = (int)cols.size();
        if ((long long)D.m0 * D.n0 > INT_MAX) fail(SDL_ERR_OVERFLOW, "dense blocks: output block exceeds INT_MAX values");
        D.s_begin = (int)h_srcs.size();
        D.map_off = (long long)h_maps.size();
        D.direct = 1;
        for (int k : P.out_srcs[o])
        {
            h_srcs.push_back(k);
            for (size_t q = 0; q < prow[k].size(); ++q) rpos[prow[k][q]] = (int)q;
            for (size_t q = 0; q < pcol[k].size(); ++q) cpos[pcol[k][q]] = (int)q;
            if (prow[k].size() != (size_t)D.m0 || pcol[k].size() != (size_t)D.n0) D.direct = 0;
            for (size_t q = 0; q < P.out_rows[o].size(); ++q)
            {
                h_maps.push_back(rpos[P.out_rows[o][q]]);
                if (rpos[P.out_rows[o][q]] != (int)q) D.direct = 0;
            }
            for (size_t q = 0; q < cols.size(); ++q)
            {
                h_maps.push_back(cpos[cols[q]]);
                if (cpos[cols[q]] != (int)q) D.direct = 0;
            }
            for (int r : prow[k]) rpos[r] = -1;
            for (int c : pcol[k]) cpos[c] = -1;
        }
        D.s_end = (int)h_srcs.size();
        od.push_back(D);
        P.c_total += (long long)D.m0 * D.n0;
    }
}

std::unique_ptr<BlocksAtaPlan> blocks_ata_build(int n_src, const int *m0, const int *n0,
                                                const int *const *row_perm, const int *const *col_perm,
                                                int m, int n, cudaStream_t s)
{
    if (n_src < 0 || m < 0 || n < 0) fail(SDL_ERR_INVALID, "blocks A^T D A: negative size");
    auto P = std::make_unique<BlocksAtaPlan>();
    P->m = m;
    P->n = n;
    P->n_src = n_src;
    std::vector<long long> x_off(std::max(1, n_src)), p_off(std::max(1, n_src)), rp_off(std::max(1, n_src));
    std::vector<int> h_m0(std::max(1, n_src)), h_n0(std::max(1, n_src)), h_rp;
    std::vector<int4> mt;
    for (int k = 0; k < n_src; ++k)
    {
        if (m0[k] < 0 || n0[k] < 0) fail(SDL_ERR_INVALID, "blocks A^T D A: negative block shape");
        for (int r = 0; r < m0[k]; ++r)
            if (row_perm[k][r] < 0 || row_perm[k][r] >= m) fail(SDL_ERR_INVALID, "blocks A^T D A: row_perm out of range");
        for (int c = 0; c < n0[k]; ++c)
            if (col_perm[k][c] < 0 || col_perm[k][c] >= n || (c && col_perm[k][c] <= col_perm[k][c - 1]))
                fail(SDL_ERR_INVALID, "blocks A^T D A: col_perm is not strictly increasing columns");
        x_off[k] = P->x_total;
        p_off[k] = P->p_total;
        rp_off[k] = (long long)h_rp.size();
        h_m0[k] = m0[k];
        h_n0[k] = n0[k];
        h_rp.insert(h_rp.end(), row_perm[k], row_perm[k] + m0[k]);
        P->x_total += (long long)m0[k] * n0[k];
        P->p_total += (long long)n0[k] * n0[k];
        for (int a = 0; a < n0[k]; a += ATA_T)
            for (int b = 0; b < n0[k]; b += ATA_T) mt.push_back(make_int4(k, a, b, 0));
    }
    // upstream's coalescing of the partials (row_perm = col_perm = col_perm_k)
    std::vector<std::vector<int>> prow(n_src), pcol(n_src);
    for (int k = 0; k < n_src; ++k)
    {
        prow[k].assign(col_perm[k], col_perm[k] + n0[k]);
        pcol[k] = prow[k];
    }
    std::vector<BlocksAtaPlan::OutDesc> od;
    std::vector<int> h_srcs, h_maps;
    coalesce_partials(prow, pcol, n, n, *P, od, h_srcs, h_maps);
    P->x_off = upload(x_off.data(), x_off.size(), s);
    P->p_off = upload(p_off.data(), p_off.size(), s);
    P->m0d = upload(h_m0.data(), h_m0.size(), s);
    P->n0d = upload(h_n0.data(), h_n0.size(), s);
    P->rowperm_all = upload(h_rp.data(), std::max<size_t>(1, h_rp.size()), s);
    P->rowperm_off = upload(rp_off.data(), rp_off.size(), s);
    P->P.reset((size_t)std::max<long long>(1, P->p_total));
    P->nmtiles = (int)mt.size();
    P->mtiles = upload(mt.data(), std::max<size_t>(1, mt.size()), s);
    // the partials' two pipeline stages exceed the default 48 KB of dynamic shared
    // memory (set on the device the plan, and so its fills, live on)
    SDL_CUDA(cudaFuncSetAttribute(k_ata_partials, cudaFuncAttributeMaxDynamicSharedMemorySize, ATA_SMEM));
    P->outd = upload(od.data(), std::max<size_t>(1, od.size()), s);
    P->srcs = upload(h_srcs.data(), std::max<size_t>(1, h_srcs.size()), s);
    P->maps = upload(h_maps.data(), std::max<size_t>(1, h_maps.size()), s);
    SDL_CUDA(cudaStreamSynchronize(s));
    return P;
}

void blocks_ata_fill(const BlocksAtaPlan &P, const double *X_vals, const double *d, double *C_vals,
                     cudaStream_t s)
{
    if (P.c_total == 0) return;
    if (P.nmtiles > 0)
        SDL_LAUNCH(k_ata_partials, P.nmtiles, 128, ATA_SMEM, s, P.mtiles.get(), P.nmtiles, P.x_off.get(),
                   P.p_off.get(), P.m0d.get(), P.n0d.get(), P.rowperm_all.get(), P.rowperm_off.get(), X_vals, d,
                   P.P.get());
    long long maxcells = 0;
    // grid.x covers the largest output block; grid.y = output blocks
    // (cells of block o: P.out_rows[o].size() * P.out_cols[o].size())
    for (int o = 0; o < P.n_out; ++o)
        maxcells = std::max(maxcells, (long long)P.out_rows[o].size() * (long long)P.out_cols[o].size());
    for (int o = 0; o < P.n_out; o += 65535)
    {
        const dim3 grid(grid_cap2(maxcells, GATHER_THREADS, 4096), (unsigned)std::min(65535, P.n_out - o));
        SDL_LAUNCH(k_ata_gather, grid, GATHER_THREADS, 0, s, P.outd.get(), o, P.srcs.get(), P.maps.get(), P.p_off.get(),
                   P.n0d.get(), P.P.get(), C_vals);
    }
}

std::unique_ptr<BlocksAtaPlan> blocks_btda_build(int n_src, const int *m0, const int *n0,
                                                 const int *const *row_perm, const int *const *col_perm, int m,
                                                 int n, const int *Bp, const int *Bi, int nB, cudaStream_t s)
{
    if (n_src < 0 || m < 0 || n < 0 || nB < 0) fail(SDL_ERR_INVALID, "B^T D A (dense blocks): negative size");
    auto P = std::make_unique<BlocksAtaPlan>();
    P->btda = true;
    P->m = m;
    P->n = n;
    P->nB = nB;
    P->n_src = n_src;
    P->B_nnz = m ? Bp[m] : 0;
    // row -> (block, local row); a stacked_pd's blocks own disjoint rows
    std::vector<int> rb(std::max(1, m), -1), rl(std::max(1, m), -1);
    std::vector<long long> x_off(std::max(1, n_src)), p_off(std::max(1, n_src)), rp_off(std::max(1, n_src));
    std::vector<int> h_m0(std::max(1, n_src)), h_n0(std::max(1, n_src)), h_rp;
    for (int k = 0; k < n_src; ++k)
    {
        if (m0[k] < 0 || n0[k] < 0) fail(SDL_ERR_INVALID, "B^T D A (dense blocks): negative block shape");
        for (int r = 0; r < m0[k]; ++r)
        {
            const int row = row_perm[k][r];
            if (row < 0 || row >= m) fail(SDL_ERR_INVALID, "B^T D A (dense blocks): row_perm out of range");
            if (rb[row] >= 0) fail(SDL_ERR_INVALID, "B^T D A (dense blocks): two blocks share a row");
            rb[row] = k;
            rl[row] = r;
        }
        for (int c = 0; c < n0[k]; ++c)
            if (col_perm[k][c] < 0 || col_perm[k][c] >= n || (c && col_perm[k][c] <= col_perm[k][c - 1]))
                fail(SDL_ERR_INVALID, "B^T D A (dense blocks): col_perm is not strictly increasing columns");
        x_off[k] = P->x_total;
        rp_off[k] = (long long)h_rp.size();
        h_m0[k] = m0[k];
        h_n0[k] = n0[k];
        h_rp.insert(h_rp.end(), row_perm[k], row_perm[k] + m0[k]);
        P->x_total += (long long)m0[k] * n0[k];
    }
    // B's entries column by column, rows ascending (its CSC order), with CSR positions
    std::vector<int> ccnt((size_t)nB + 1, 0);
    for (int i = 0; i < m; ++i)
        for (int q = Bp[i]; q < Bp[i + 1]; ++q)
        {
            if (Bi[q] < 0 || Bi[q] >= nB) fail(SDL_ERR_INVALID, "B^T D A (dense blocks): column index of B out of range");
            ccnt[Bi[q] + 1]++;
        }
    for (int c = 0; c < nB; ++c) ccnt[c + 1] += ccnt[c];
    std::vector<int> crow((size_t)std::max(1, P->B_nnz)), cpos((size_t)std::max(1, P->B_nnz));
    {
        std::vector<int> nx(ccnt.begin(), ccnt.end() - 1);
        for (int i = 0; i < m; ++i)
            for (int q = Bp[i]; q < Bp[i + 1]; ++q)
            {
                const int e = nx[Bi[q]]++;
                crow[e] = i;
                cpos[e] = q;
            }
    }
    // per block: the active columns of B and their entries
    P->act.assign(n_src, {});
    std::vector<std::vector<int>> ekk(n_src), epos(n_src), eoff(n_src);
    for (int c = 0; c < nB; ++c)
        for (int e = ccnt[c]; e < ccnt[c + 1]; ++e)
        {
            const int k = rb[crow[e]];
            if (k < 0) continue;
            if (P->act[k].empty() || P->act[k].back() != c)
            {
                P->act[k].push_back(c);
                eoff[k].push_back((int)ekk[k].size());
            }
            ekk[k].push_back(rl[crow[e]]);
            epos[k].push_back(cpos[e]);
        }
    std::vector<int2> wt;
    std::vector<int> h_off(1, 0), h_kk, h_pos;
    for (int k = 0; k < n_src; ++k)
    {
        p_off[k] = P->p_total;
        P->p_total += (long long)P->act[k].size() * n0[k];
        eoff[k].push_back((int)ekk[k].size());
        for (size_t a = 0; a < P->act[k].size(); ++a)
        {
            wt.push_back(make_int2(k, (int)a));
            h_kk.insert(h_kk.end(), ekk[k].begin() + eoff[k][a], ekk[k].begin() + eoff[k][a + 1]);
            h_pos.insert(h_pos.end(), epos[k].begin() + eoff[k][a], epos[k].begin() + eoff[k][a + 1]);
            h_off.push_back((int)h_kk.size());
        }
    }
    // upstream's coalescing of the partials (rows = active columns of B, columns = col_perm_k)
    std::vector<std::vector<int>> pcol(n_src);
    for (int k = 0; k < n_src; ++k) pcol[k].assign(col_perm[k], col_perm[k] + n0[k]);
    std::vector<BlocksAtaPlan::OutDesc> od;
    std::vector<int> h_srcs, h_maps;
    coalesce_partials(P->act, pcol, nB, n, *P, od, h_srcs, h_maps);
    P->x_off = upload(x_off.data(), x_off.size(), s);
    P->p_off = upload(p_off.data(), p_off.size(), s);
    P->m0d = upload(h_m0.data(), h_m0.size(), s);
    P->n0d = upload(h_n0.data(), h_n0.size(), s);
    P->rowperm_all = upload(h_rp.data(), std::max<size_t>(1, h_rp.size()), s);
    P->rowperm_off = upload(rp_off.data(), rp_off.size(), s);
    P->P.reset((size_t)std::max<long long>(1, P->p_total));
    P->nwtask = (int)wt.size();
    P->wtask = upload(wt.data(), std::max<size_t>(1, wt.size()), s);
    P->ent_off = upload(h_off.data(), h_off.size(), s);
    P->ent_kk = upload(h_kk.data(), std::max<size_t>(1, h_kk.size()), s);
    P->ent_pos = upload(h_pos.data(), std::max<size_t>(1, h_pos.size()), s);
    P->outd = upload(od.data(), std::max<size_t>(1, od.size()), s);
    P->srcs = upload(h_srcs.data(), std::max<size_t>(1, h_srcs.size()), s);
    P->maps = upload(h_maps.data(), std::max<size_t>(1, h_maps.size()), s);
    SDL_CUDA(cudaStreamSynchronize(s));
    return P;
}

void blocks_btda_fill(const BlocksAtaPlan &P, const double *X_vals, const double *d, const double *B_x,
                      double *C_vals, cudaStream_t s)
{
    if (P.c_total == 0) return;
    if (P.nwtask > 0)
        SDL_LAUNCH(k_btda_partials, (P.nwtask + 7) / 8, 256, 0, s, P.wtask.get(), P.nwtask, P.ent_off.get(),
                   P.ent_kk.get(), P.ent_pos.get(), P.x_off.get(), P.p_off.get(), P.m0d.get(), P.n0d.get(),
                   P.rowperm_all.get(), P.rowperm_off.get(), X_vals, d, B_x, P.B_nnz, P.P.get(), runtime().d_error);
    long long maxcells = 0;
    for (int o = 0; o < P.n_out; ++o)
        maxcells = std::max(maxcells, (long long)P.out_rows[o].size() * (long long)P.out_cols[o].size());
    for (int o = 0; o < P.n_out; o += 65535)
    {
        const dim3 grid(grid_cap2(maxcells, GATHER_THREADS, 4096), (unsigned)std::min(65535, P.n_out - o));
        SDL_LAUNCH(k_ata_gather, grid, GATHER_THREADS, 0, s, P.outd.get(), o, P.srcs.get(), P.maps.get(), P.p_off.get(),
                   P.n0d.get(), P.P.get(), C_vals);
    }
}

} // namespace sdl
