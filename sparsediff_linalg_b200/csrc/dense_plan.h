// Products of dense blocks (permuted_dense / the blocks of a stacked_pd) with a
// sparse CSR: C_k = B_k S[col_perm_k, :] for every block k (upstream
// src/permuted_dense/permuted_dense_linalg.c:313-430 BA_pd_csr_*,
// src/stacked_pd/stacked_pd_linalg.c:657-671 BA_spd_csr_*).
#pragma once

#include <memory>
#include <vector>

#include "sdl_internal.h"

namespace sdl {

// Device descriptor of one output block.
struct BlkDesc
{
    long long b_off; // first value of the source block in the B value array
    long long c_off; // first value of the output block in the C value array
    long long cp_off; // column offsets of its compact CSC (n0_C + 1)
    long long d_off;  // its compact CSC entries (rows, vals)
    int m0, n0_B, n0_C, pad;
};

// One CTA's share: columns [c0, c0 + 32) of output block `blk`.
struct BlkTile
{
    int blk, c0;
};

struct BlocksCsrPlan
{
    int S_m = 0, S_n = 0, S_nnz = 0;
    int n_src = 0;
    // output blocks: the source blocks whose product has at least one column
    // (upstream spd_map_filter_blocks drops the empty ones)
    std::vector<int> src;                   // source block of each output block
    std::vector<std::vector<int>> col_perm; // col_perm of each output block (host)
    std::vector<int> m0, n0_C;
    long long c_total = 0, b_total = 0, d_total = 0;
    // compact CSC of S restricted to a block's col_perm rows, shared by blocks whose
    // col_perms are equal: column offsets, local row in the block, position in S.x
    DevBuf<int> cp, rows, pos;
    DevBuf<double> vals; // S.x gathered in compact order (refill scratch)
    DevBuf<double> BT;   // the source blocks transposed (refill scratch)
    int tr_x = 0, tr_y = 0; // transpose grid: 32 x 32 tiles of the largest block
    DevBuf<BlkDesc> desc;
    DevBuf<BlkTile> tiles;
    int ntiles = 0;
};

// Builds the plan of C_k = B_k S[col_perm_k, :] for n_src source blocks of shape
// m0[k] x n0[k] (col_perm[k] strictly increasing rows of S); S given by its host CSR
// structure (S_m x S_n). When keep_empty, every source block gets an output block
// (a single permuted_dense), else blocks without columns are dropped.
std::unique_ptr<BlocksCsrPlan> blocks_csr_build(int n_src, const int *m0, const int *n0,
                                                const int *const *col_perm, const int *Sp, const int *Si,
                                                int S_m, int S_n, bool keep_empty, cudaStream_t s);
// C values (output blocks in order, each m0 x n0_C row-major) from the B values
// (source blocks in order, each m0 x n0 row-major) and S.x; all device pointers.
void blocks_csr_fill(const BlocksCsrPlan &P, const double *B_vals, const double *S_x, double *C_vals,
                     cudaStream_t s);

} // namespace sdl

namespace sdl {

// A^T diag(d) A for dense blocks A_k (m0[k] x n0[k], rows row_perm[k] of an m-row
// matrix, columns col_perm[k] of n): the partial of every block,
// P_k = X_k^T diag(d[row_perm_k]) X_k (n0 x n0, rows and columns col_perm_k), on the
// FP64 tensor cores, then upstream's coalescing (src/stacked_pd/
// stacked_pd_coalesce.c:150-381): output blocks grouped by the set of blocks that
// contain a row (its signature), each cell the sum of the partials that hold it,
// from +0.0 in block order (upstream ATA_spd_* in src/stacked_pd/
// stacked_pd_linalg.c:197-237; ATA_pd_* in permuted_dense_linalg.c:87-112 is the
// one-block case).
struct BlocksAtaPlan
{
    int n = 0, m = 0, n_src = 0;
    // output blocks (signatures): rows, columns, contributing source blocks
    std::vector<std::vector<int>> out_rows, out_cols, out_srcs;
    std::vector<int> src_p; // out k's sources: out_srcs flattened, src_p offsets
    long long c_total = 0, p_total = 0, x_total = 0;
    DevBuf<long long> x_off, p_off;       // per source block: its values / its partial
    DevBuf<int> m0d, n0d;                 // per source block
    DevBuf<int> rowperm_all;              // per source block, concatenated
    DevBuf<long long> rowperm_off;
    DevBuf<double> P;                     // partials (refill scratch)
    DevBuf<int4> mtiles;                  // 64 x 64 tiles of the partials: (block, a0, b0, -)
    int nmtiles = 0;
    // gather of the output cells: per output block, per source: row / column maps
    struct OutDesc
    {
        long long c_off; // first value of the output block
        int m0, n0;
        int s_begin, s_end; // its sources in srcs
        long long map_off;  // row maps then column maps of its sources
        int direct;         // 1: every source is exactly this block (cell e of the
                            // block is value e of each partial): no map lookups
    };
    DevBuf<OutDesc> outd;
    DevBuf<int> srcs;   // source block ids
    DevBuf<int> maps;   // per (output block, source): m0 row positions, n0 column positions (-1: absent)
    int n_out = 0;
    // B^T diag(d) A_k partials (blocks_btda_build): one warp task per (block, active
    // column of B); its entries (block row, position in B's CSR values) in B's CSC order
    bool btda = false;
    int nB = 0, B_nnz = 0, nwtask = 0;
    std::vector<std::vector<int>> act; // per block: the columns of B that reach its rows (host)
    DevBuf<int2> wtask;                // (block, index of the active column)
    DevBuf<int> ent_off, ent_kk, ent_pos;
};

std::unique_ptr<BlocksAtaPlan> blocks_ata_build(int n_src, const int *m0, const int *n0,
                                                const int *const *row_perm, const int *const *col_perm,
                                                int m, int n, cudaStream_t s);
// C values (output blocks in order, row-major) from the source values X_vals
// (blocks in order, row-major) and d (m values, or null for the identity).
void blocks_ata_fill(const BlocksAtaPlan &P, const double *X_vals, const double *d, double *C_vals,
                     cudaStream_t s);

// B^T diag(d) A for B sparse (m x nB, host CSR structure) and A dense blocks (rows
// row_perm[k] of m, pairwise disjoint; columns col_perm[k] of n): per block the
// partial B^T diag(d) A_k over the columns of B that reach its rows (upstream
// BTA_csc_pd_* / BTDA_csc_pd_*, src/permuted_dense/permuted_dense_linalg.c:646-741,
// each output a sum over B's column in CSC order from +0.0: bit-identical), then
// upstream's coalescing (BTA_csc_spd_* / BTDA_csc_spd_*, src/stacked_pd/
// stacked_pd_linalg.c:594-608).
std::unique_ptr<BlocksAtaPlan> blocks_btda_build(int n_src, const int *m0, const int *n0,
                                                 const int *const *row_perm, const int *const *col_perm, int m,
                                                 int n, const int *Bp, const int *Bi, int nB, cudaStream_t s);
// C values from the blocks' values, d (or null: B^T A) and B's CSR values (device).
void blocks_btda_fill(const BlocksAtaPlan &P, const double *X_vals, const double *d, const double *B_x,
                      double *C_vals, cudaStream_t s);

} // namespace sdl
