// Fill programs over dense blocks: the device side of every permuted_dense /
// stacked_pd operation that is not a dedicated kernel elsewhere (upstream
// src/permuted_dense/permuted_dense.c, permuted_dense_linalg.c, src/stacked_pd/
// stacked_pd.c, stacked_pd_linalg.c, stacked_pd_coalesce.c).
//
// A program runs in two stages. Stage 1 writes partial blocks into a partial
// buffer P: row copies / scalings / sums, block transposes, gathered GEMMs on the
// FP64 tensor cores, and sparse x dense vectors. Stage 2, present when the output
// is a coalesced stacked_pd (or a permuted_dense accumulated from several
// partials), gathers every output cell from the partials that hold it: a sum from
// +0.0 in partial order (upstream's memset + accumulating scatter) or the single
// holder's value (upstream's plain scatter). A program without stage 2 writes its
// partials straight into the output values (P is the output).
//
// The host builds a program once per output (the alloc); the fill uploads the
// operands' values and runs it. All value arrays are block-major and row-major
// within a block, as upstream stores them.
#pragma once

#include <memory>
#include <vector>

#include "capi_common.h"

namespace sdl {

enum DpRowMode : int
{
    DP_ROW_COPY = 0,  // dst = src (one source)
    DP_ROW_SCALE = 1, // dst = src * d[scale_row] (one source)
    DP_ROW_SUM = 2,   // dst = sum of the sources from +0.0, in list order
};

// One output row of `len` values at P + dst; sources XL + src[e] for e in
// [e_begin, e_end).
struct DpRowTask
{
    long long dst;
    int len, e_begin, e_end, scale_row, mode;
};

// P + dst (n0 x m0) = (XL + src, an m0 x n0 block)^T.
struct DpTrTask
{
    long long src, dst;
    int m0, n0;
};

// P[p + i * nj + j] = sum over t < s of L(i, t) * R(t, j), on mma.m8n8k4 f64:
//   L(i, t) = XL[l_off + (l_trans ? lidx[t] * l_ld + i : i * l_ld + lidx[t])]
//   R(t, j) = XR[r_off + ridx[t] * r_ld + j], times d[drow[t]] (one rounding, as
//             upstream's dscal of the gathered rows) when d is given
// with t indexing idx_off + t in the lidx / ridx / drow arrays.
struct DpGemmTask
{
    long long l_off, r_off, p, idx_off;
    int l_ld, r_ld, ni, nj, s, l_trans;
};

// Where a fill with d folds d[row] into a sparse x dense term; without d the
// term is S.x * X.
enum DpSpMode : int
{
    DP_SP_D_DENSE = 1, // S.x * (d[row] * X)   (upstream BTDA_csc_pd: d folded into the dense block)
    DP_SP_D_SPARSE = 2 // (d[row] * S.x) * X   (upstream BTDA_pd_csc: d folded into the sparse value)
};

// One vector of `nvec` values: P[p + t * stride] = sum over the entries e in
// [e_begin, e_end) of the term (mode) for S.x[e_pos[e]], the dense value
// X[x_off + e_kk[e] * ld + t] (or X[x_off + t * ld + e_kk[e]] when dense_trans)
// and d[e_row[e]], from +0.0 in entry order. X is XL (dense_right == 0) or XR.
struct DpSpTask
{
    long long x_off, p;
    int ld, nvec, e_begin, e_end, stride, mode, dense_right, dense_trans;
};

// Output block of stage 2: m0 x n0 values at C + c_off; its value sources
// [s_begin, s_end) each with a row map (m0) and a column map (n0) at map_off.
struct DpOut
{
    long long c_off, map_off;
    int m0, n0, s_begin, s_end, accumulate, pad;
};

// One value source of stage 2: the cell (si, sj) of the source is P[p + si * rs + sj * cs].
struct DpSrc
{
    long long p;
    int rs, cs;
};

struct DenseProg
{
    bool gathered = false;      // stage 2 present
    long long p_total = 0;      // partial values (== c_total when not gathered)
    long long c_total = 0;      // output values
    long long nl = 0, nr = 0;   // XL / XR values the fill expects
    int ns = 0;                 // sparse values the fill expects (S.x)
    int d_len = 0;              // length of d when the fill takes one (0: no d)
    bool needs_d = false;       // the fill requires d (row scalings)
    // output structure of a coalesced result (host): per output block its rows,
    // columns and the partials (upstream source blocks) of its signature
    std::vector<std::vector<int>> out_rows, out_cols, out_srcs;
    // stage 1
    int n_row = 0, n_trt = 0, n_gmt = 0, n_sp = 0;
    DevBuf<DpRowTask> row;
    DevBuf<long long> row_src;
    DevBuf<DpTrTask> tr;
    DevBuf<int4> tr_tiles; // (task, r0, c0, -): 32 x 32 tiles
    DevBuf<DpGemmTask> gm;
    DevBuf<int4> gm_tiles; // (task, a0, b0, -): 16 x 16 tiles
    DevBuf<int> lidx, ridx, drow;
    DevBuf<DpSpTask> sp;
    DevBuf<int> e_kk, e_pos, e_row;
    // stage 2
    int n_out = 0;
    long long max_cells = 0;
    DevBuf<DpOut> outd;
    DevBuf<DpSrc> srcs;
    DevBuf<int> maps;
    DevBuf<double> P; // partial scratch (gathered programs)
};

// Host-side builder.
struct DpBuilder
{
    std::vector<DpRowTask> row;
    std::vector<long long> row_src;
    std::vector<DpTrTask> tr;
    std::vector<DpGemmTask> gm;
    std::vector<int> lidx, ridx, drow;
    std::vector<DpSpTask> sp;
    std::vector<int> e_kk, e_pos, e_row;
    long long p_total = 0;

    long long alloc(long long n)
    {
        const long long off = p_total;
        p_total += n;
        return off;
    }
    void row_copy(long long dst, long long src, int len, int mode = DP_ROW_COPY, int scale_row = -1);
    void row_sum(long long dst, const std::vector<long long> &srcs, int len);
    void transpose(long long src, long long dst, int m0, int n0);
    // P[p + i * nj + j] = sum_t L(i, t) R(t, j), see DpGemmTask
    void gemm(long long p, int ni, int nj, long long l_off, int l_ld, bool l_trans, const std::vector<int> &li,
              long long r_off, int r_ld, const std::vector<int> &ri, const std::vector<int> &dr);
    // one vector; entries (dense row, position of S.x, global row for d)
    void spvec(long long p, int nvec, int stride, long long x_off, int ld, bool dense_right, int mode,
               const std::vector<int> &kk, const std::vector<int> &pos, const std::vector<int> &grow,
               bool dense_trans = false);
};

// A partial of a coalesced result: rows x cols of the result (both ascending),
// whose values come from one or more value sources. Each value source covers all
// of the partial's rows and a subset `cols` of its columns; with several, a cell's
// value is their sum (the inner sum of a nested blockwise product).
struct DpPart
{
    std::vector<int> rows, cols;
    struct Val
    {
        std::vector<int> cols;
        long long p;
        int rs, cs;
    };
    std::vector<Val> vals;
};

// Every program is finished by one of the three calls below (the output side),
// then by dp_finish, which checks every index of stage 1 against the operand
// sizes the fill accepts (XL / XR values, sparse values, length of d; 0 when the
// product takes no d) and uploads the tasks.
void dp_finish(DenseProg &P, DpBuilder &b, long long nl, long long nr, int ns, int d_len, cudaStream_t s);
// Finish a program whose partials are the output itself (no stage 2).
std::unique_ptr<DenseProg> dp_direct(DpBuilder &b, long long c_total, cudaStream_t s);
// Finish a program with upstream's coalescing of `parts` (an nrows x ncols result,
// src/stacked_pd/stacked_pd_coalesce.c:115-381): rows grouped by the list of parts
// that hold them, output blocks in order of first appearance, columns the union of
// the parts' columns; cells summed from +0.0 in part order (accumulate) or copied
// from their single holder.
std::unique_ptr<DenseProg> dp_coalesced(DpBuilder &b, const std::vector<DpPart> &parts, int nrows, int ncols,
                                        bool accumulate, cudaStream_t s);
// Finish a program whose output blocks are the parts themselves, in order (rows
// x cols of each part), each cell the sum of its part's value sources from +0.0.
std::unique_ptr<DenseProg> dp_blocks(DpBuilder &b, const std::vector<DpPart> &parts, cudaStream_t s);
// Finish a program whose one output block (rows x cols) is the sum of `parts`
// (each part's rows a subset of `rows`) from +0.0 in part order.
std::unique_ptr<DenseProg> dp_single(DpBuilder &b, const std::vector<int> &rows, const std::vector<int> &cols,
                                     const std::vector<DpPart> &parts, cudaStream_t s);

// Run: XL / XR dense operand values, Sx sparse values, d (or null), C output values
// (all device pointers).
void dp_fill(DenseProg &P, const double *XL, const double *XR, const double *Sx, const double *d, double *C,
             cudaStream_t s);

} // namespace sdl
