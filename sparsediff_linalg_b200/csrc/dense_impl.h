// Device state bound to a permuted_dense / stacked_pd by the operation that
// allocated it (its plan or fill program, and the device copies of its operands'
// and its own values).
#pragma once

#include <memory>

#include "dense_plan.h"
#include "dense_prog.h"
#include "matrix_kinds.h"

namespace sdl {

// Operations whose fill runs a DenseProg (dense_prog.h).
enum DpOp : int
{
    DP_OP_NONE = 0,
    DP_OP_DA,        // DA_matrices_fill_values
    DP_OP_TRANSPOSE, // transpose_matrices_*
    DP_OP_GATHER,    // row_gather vtable slot
    DP_OP_REDUCE,    // row_reduce vtable slot
    DP_OP_BTA,       // BTA_matrices_alloc (B or A dense-block, the other any kind)
    DP_OP_BA,        // BA_matrices_alloc
    DP_OP_KRON,      // BA_kron_matrices_alloc / BA_dense_kron_I_matrices_alloc (A a full permuted_dense)
};

struct ProgState
{
    int op = DP_OP_NONE;
    std::unique_ptr<DenseProg> prog;
    DevBuf<double> xl, xr, dv, cv; // operand values, d, output values
};

struct PdImpl
{
    std::unique_ptr<BlocksCsrPlan> ba;  // bound by BA_matrices_alloc (B pd, A sparse)
    std::unique_ptr<BlocksAtaPlan> ata; // bound by ATA_matrices_alloc (A pd) or BTA_matrices_alloc (B sparse)
    DevBuf<double> bvals, cvals, dvec;
    ProgState ps;
};

struct SpdImpl
{
    std::unique_ptr<BlocksAtaPlan> ata;
    DevBuf<double> xvals, cvals, dvec;
    ProgState ps;
};

inline ProgState *prog_state(matrix *m)
{
    if (m->kind == MATRIX_PERMUTED_DENSE) return as_pd(m)->impl ? &as_pd(m)->impl->ps : nullptr;
    if (m->kind == MATRIX_STACKED_PD) return as_spd(m)->impl ? &as_spd(m)->impl->ps : nullptr;
    return nullptr;
}

// Fill-program operations (capi_dense_ops.cpp).
matrix *prog_BTA_alloc(matrix *A, matrix *B);
matrix *prog_BA_alloc(const matrix *B, matrix *A);
// Runs the program bound to C: XL = B's values, XR = A's values (dense kinds),
// the sparse operand's values, d (or null).
void prog_product_fill(const matrix *B, const double *d, const matrix *A, matrix *C, int op);
void prog_DA_fill(const double *d, const matrix *A, matrix *C);
matrix *prog_transpose_alloc(const matrix *A);
void prog_transpose_fill(const matrix *A, matrix *AT);
matrix *pd_row_gather_alloc(const matrix *self, const int *map, int m_out);
matrix *spd_row_gather_alloc(const matrix *self, const int *map, int m_out);
matrix *pd_row_reduce_alloc(const matrix *self, const int *group, int m_out);
matrix *spd_row_reduce_alloc(const matrix *self, const int *group, int m_out);
void dense_rows_fill(const matrix *self, matrix *out); // row_gather / row_reduce fill slots
// C = kron(I_p, A) J (a_i = false) or kron(A, I_p) J (a_i = true) for a full
// permuted_dense A and J of any kind; C is a stacked_pd.
matrix *prog_dense_kron_alloc(const matrix *A, int p, matrix *J, bool a_i);
void prog_dense_kron_fill(const matrix *A, int p, const matrix *J, matrix *C);

} // namespace sdl
