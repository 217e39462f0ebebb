// Upstream polymorphic matrix API (matrix.h, matmul.h) with the sparse kind on
// the GPU.
//
// Mirrors of upstream's caches (src/internal/sparse_matrix.h:32-54):
//   * csc_cache  -> a device CSC structure plus the CSR position of every CSC entry
//                   (TransposePlan). Fills read B's values straight from its CSR
//                   through those positions, so the CSC value refresh upstream runs
//                   in sparse_csc_fresh (src/sparse/sparse_matrix.c:62-72) is fused
//                   into the product kernel.
//   * device CSR values, re-uploaded iff base.values_version moved (the same
//     version protocol upstream uses for its CSC mirror).
//   * bound_iwork / bound_dwork -> a BoundOp holding the device plan of the alloc
//     that produced the matrix.
// Every fill leaves the output's host values current and bumps its version; the
// device copy of the output is then known fresh, so chained products do not
// re-upload it.
#include <climits>
#include <memory>

#include "capi_common.h"
#include "matrix_kinds.h"
#include "sparsediff_linalg/matmul.h"
#include "sparsediff_linalg/matrix.h"
#include "sparsediff_linalg/tracked_alloc.h"

namespace sdl {

int gather_rows_structure(const int *d_Ap, const int *d_Ai, const int *d_map, int m_out,
                          DevBuf<int> &Cp, DevBuf<int> &Ci, cudaStream_t s);
void gather_rows_values(const int *d_Ap, const double *d_Ax, const int *d_map, const int *d_Cp,
                        int m_out, double *d_Cx, cudaStream_t s);
void scale_rows(const int *d_Ap, int m, const double *d_d, const double *d_Ax, double *d_Cx,
                cudaStream_t s);

namespace {

cudaStream_t S() { return runtime().stream; }

// ------------------------------------------------------------------ bound ops
struct ProductOp : BoundOp
{
    std::shared_ptr<DevStruct> A;     // right operand structure
    std::shared_ptr<DevStruct> Lrows; // L given by rows of a CSR (B A)
    std::shared_ptr<TransposePlan> Lcsc; // L = CSC mirror (B^T A, A^T A)
    std::shared_ptr<TransposePlan> group; // L = group indicator (row_reduce)
    Product P;
    DevBuf<double> dvec;
    int A_m = 0, A_n = 0, A_nnz = 0, L_src_m = 0, L_src_n = 0, L_src_nnz = 0;
};

struct GatherOp : BoundOp
{
    std::shared_ptr<DevStruct> A;
    DevBuf<int> map;
    int A_m = 0, A_n = 0, A_nnz = 0;
};

struct TransposeOp : BoundOp
{
    std::shared_ptr<TransposePlan> T;
    int A_m = 0, A_n = 0, A_nnz = 0;
};

struct ScaleOp : BoundOp
{
    DevBuf<double> dvec;
};

CSR_matrix *sparse_to_csr(matrix *self) { return as_sparse(self)->csr; }

matrix *sparse_row_gather_alloc(const matrix *self, const int *map, int m_out);
void sparse_row_gather_fill(const matrix *self, matrix *out);
matrix *sparse_row_reduce_alloc(const matrix *self, const int *group, int m_out);
void sparse_row_reduce_fill(const matrix *self, matrix *out);

void sparse_free(sdl_sparse *sm)
{
    delete sm->impl;
    free_CSR_matrix(sm->csr);
    sp_free(sm);
}

void check_sparse(const matrix *M, const char *what)
{
    if (!M) fail(SDL_ERR_INVALID, std::string(what) + " is NULL");
    if (M->kind != MATRIX_SPARSE) fail(SDL_ERR_INVALID, std::string(what) + " must be sparse here");
}

// C = kron(I, L) diag(d) A product output. mode: 0 = L is the CSC mirror of Lsrc
// (B^T A / A^T A), 1 = L is Lsrc's CSR rows (B A).
matrix *sparse_product_alloc(sdl_sparse *Lsrc, int mode, sdl_sparse *A)
{
    cudaStream_t s = S();
    auto op = std::make_unique<ProductOp>();
    op->A = std::shared_ptr<DevStruct>(nullptr);
    const DevStruct &As = sparse_dev_struct(A, s);
    (void)As;
    op->A = A->impl->st;
    ProductDesc d;
    if (mode == 0)
    {
        const TransposePlan &T = sparse_dev_csc(Lsrc, s);
        (void)T;
        op->Lcsc = Lsrc->impl->csc;
        d.Lp = op->Lcsc->Tp.get();
        d.Li = op->Lcsc->Ti.get();
        d.L_map = op->Lcsc->src.get();
        d.L_m = Lsrc->csr->n;
        d.L_nnz = Lsrc->csr->nnz;
        if (Lsrc->csr->m != A->csr->m) fail(SDL_ERR_INVALID, "B^T A: row counts of A and B differ");
    }
    else
    {
        sparse_dev_struct(Lsrc, s);
        op->Lrows = Lsrc->impl->st;
        d.Lp = op->Lrows->p.get();
        d.Li = op->Lrows->i.get();
        d.L_m = Lsrc->csr->m;
        d.L_nnz = Lsrc->csr->nnz;
        if (Lsrc->csr->n != A->csr->m) fail(SDL_ERR_INVALID, "B A: inner dimensions differ");
    }
    d.blocks = 1;
    d.Ap = op->A->p.get();
    d.Ai = op->A->i.get();
    d.A_m = A->csr->m;
    d.A_n = A->csr->n;
    d.A_nnz = A->csr->nnz;
    product_symbolic(d, TuneConfig{}, op->P, s);
    op->dvec.reset(std::max(1, A->csr->m));
    op->A_m = A->csr->m;
    op->A_n = A->csr->n;
    op->A_nnz = A->csr->nnz;
    op->L_src_m = Lsrc->csr->m;
    op->L_src_n = Lsrc->csr->n;
    op->L_src_nnz = Lsrc->csr->nnz;
    sdl_sparse *C = new_output(op->P.m_out, op->P.n, op->P.nnz, op->P.Cp.get(), op->P.Ci.get(), s);
    C->impl->bound = std::move(op);
    return &C->base;
}

void sparse_product_fill(sdl_sparse *Lsrc, const double *d, sdl_sparse *A, sdl_sparse *C)
{
    cudaStream_t s = S();
    auto *op = dynamic_cast<ProductOp *>(C->impl->bound.get());
    if (!op) fail(SDL_ERR_INVALID, "C was not produced by the matching alloc");
    if (op->A_m != A->csr->m || op->A_n != A->csr->n || op->A_nnz != A->csr->nnz ||
        op->L_src_m != Lsrc->csr->m || op->L_src_n != Lsrc->csr->n || op->L_src_nnz != Lsrc->csr->nnz)
        fail(SDL_ERR_INVALID, "operands do not match the ones C was allocated for");
    const double *Ax, *Lx;
    {
        NvtxRange r("sdl: operand values to the device");
        Ax = sparse_dev_values(A, s);
        Lx = sparse_dev_values(Lsrc, s);
        if (d) h2d(op->dvec.get(), d, A->csr->m, s);
    }
    product_numeric(op->P, Lx, d ? op->dvec.get() : nullptr, Ax, C->impl->vals.x.get(), s);
    publish_output(C, s);
}

// ------------------------------------------------------------------ row gather
matrix *sparse_row_gather_alloc(const matrix *self, const int *map, int m_out)
{
    return guard_upstream<matrix *>("row_gather_alloc", nullptr, [&]() -> matrix * {
        sdl_sparse *A = as_sparse(self);
        cudaStream_t s = S();
        if (m_out < 0) fail(SDL_ERR_INVALID, "negative m_out");
        auto op = std::make_unique<GatherOp>();
        sparse_dev_struct(A, s);
        op->A = A->impl->st;
        op->map = upload(map, m_out, s);
        validate_compressed(nullptr, op->map.get(), 0, A->csr->m, m_out, "row_gather map", s);
        DevBuf<int> Cp, Ci;
        int nnz = gather_rows_structure(op->A->p.get(), op->A->i.get(), op->map.get(), m_out, Cp, Ci, s);
        op->A_m = A->csr->m;
        op->A_n = A->csr->n;
        op->A_nnz = A->csr->nnz;
        sdl_sparse *C = new_output(m_out, A->csr->n, nnz, Cp.get(), Ci.get(), s);
        C->impl->st = std::make_shared<DevStruct>();
        C->impl->st->rows = m_out;
        C->impl->st->cols = A->csr->n;
        C->impl->st->nnz = nnz;
        C->impl->st->p = std::move(Cp);
        C->impl->st->i = std::move(Ci);
        C->impl->bound = std::move(op);
        return &C->base;
    });
}

void sparse_row_gather_fill(const matrix *self, matrix *out)
{
    guard_upstream_void("row_gather_fill_values", [&]() {
        sdl_sparse *A = as_sparse(self);
        sdl_sparse *C = as_sparse(out);
        cudaStream_t s = S();
        auto *op = dynamic_cast<GatherOp *>(C->impl->bound.get());
        if (!op) fail(SDL_ERR_INVALID, "output was not produced by row_gather_alloc");
        if (op->A_m != A->csr->m || op->A_n != A->csr->n || op->A_nnz != A->csr->nnz)
            fail(SDL_ERR_INVALID, "A does not match the matrix the gather was allocated for");
        const double *Ax = sparse_dev_values(A, s);
        gather_rows_values(op->A->p.get(), Ax, op->map.get(), C->impl->st->p.get(), C->csr->m,
                           C->impl->vals.x.get(), s);
        publish_output(C, s);
    });
}

// ------------------------------------------------------------------ row reduce
// C = G A with G the m_out x m indicator of group (rows of G list their source rows
// in ascending order): a unit-valued row-wise product, which sums every output
// entry's sources in ascending source position from +0.0 exactly as upstream's
// accumulator does (src/sparse/sparse_matrix.c:221-240, CSR_sum.c:150-157).
matrix *sparse_row_reduce_alloc(const matrix *self, const int *group, int m_out)
{
    return guard_upstream<matrix *>("row_reduce_alloc", nullptr, [&]() -> matrix * {
        sdl_sparse *A = as_sparse(self);
        cudaStream_t s = S();
        if (m_out < 0) fail(SDL_ERR_INVALID, "negative m_out");
        int m = A->csr->m;
        auto op = std::make_unique<ProductOp>();
        sparse_dev_struct(A, s);
        op->A = A->impl->st;
        DevBuf<int> g = upload(group, m, s);
        validate_compressed(nullptr, g.get(), 0, m_out, m, "row_reduce group", s);
        op->group = std::make_shared<TransposePlan>();
        transpose_build(nullptr, g.get(), m, m_out, m, *op->group, s);
        ProductDesc d;
        d.Lp = op->group->Tp.get();
        d.Li = op->group->Ti.get();
        d.L_m = m_out;
        d.L_nnz = m;
        d.blocks = 1;
        d.Ap = op->A->p.get();
        d.Ai = op->A->i.get();
        d.A_m = m;
        d.A_n = A->csr->n;
        d.A_nnz = A->csr->nnz;
        product_symbolic(d, TuneConfig{}, op->P, s);
        op->A_m = m;
        op->A_n = A->csr->n;
        op->A_nnz = A->csr->nnz;
        sdl_sparse *C = new_output(m_out, A->csr->n, op->P.nnz, op->P.Cp.get(), op->P.Ci.get(), s);
        C->impl->bound = std::move(op);
        return &C->base;
    });
}

void sparse_row_reduce_fill(const matrix *self, matrix *out)
{
    guard_upstream_void("row_reduce_fill_values", [&]() {
        sdl_sparse *A = as_sparse(self);
        sdl_sparse *C = as_sparse(out);
        cudaStream_t s = S();
        auto *op = dynamic_cast<ProductOp *>(C->impl->bound.get());
        if (!op || !op->group) fail(SDL_ERR_INVALID, "output was not produced by row_reduce_alloc");
        if (op->A_m != A->csr->m || op->A_n != A->csr->n || op->A_nnz != A->csr->nnz)
            fail(SDL_ERR_INVALID, "A does not match the matrix the reduce was allocated for");
        const double *Ax = sparse_dev_values(A, s);
        product_numeric(op->P, nullptr, nullptr, Ax, C->impl->vals.x.get(), s);
        publish_output(C, s);
    });
}

void wire_sparse(sdl_sparse *sm)
{
    sm->base.kind = MATRIX_SPARSE;
    sm->base.to_csr = sparse_to_csr;
    sm->base.row_gather_alloc = sparse_row_gather_alloc;
    sm->base.row_gather_fill_values = sparse_row_gather_fill;
    sm->base.row_reduce_alloc = sparse_row_reduce_alloc;
    sm->base.row_reduce_fill_values = sparse_row_reduce_fill;
}

} // namespace

// Copy the device values of an output into its host CSR and publish them.
void publish_output(sdl_sparse *C, cudaStream_t s)
{
    NvtxRange r("sdl: C.x to the host");
    d2h(C->csr->x, C->impl->vals.x.get(), C->csr->nnz, s);
    check_device_errors(s, "fill");
    matrix_values_changed(&C->base);
    C->impl->vals.seen = C->base.values_version;
    C->impl->vals.valid = true;
}

// New sparse output whose structure is (Cp, Ci) on the device; host copy made.
sdl_sparse *new_output(int m, int n, int nnz, const int *d_Cp, const int *d_Ci, cudaStream_t s)
{
    CSR_matrix *csr = new_CSR_matrix(m, n, nnz);
    d2h(csr->p, d_Cp, (size_t)m + 1, s);
    d2h(csr->i, d_Ci, nnz, s);
    SDL_CUDA(cudaStreamSynchronize(s));
    sdl_sparse *C = as_sparse(sparse_wrap(csr));
    C->impl->vals.x.reset(std::max(1, nnz));
    return C;
}


// ------------------------------------------------------------------ sparse helpers
matrix *sparse_wrap(CSR_matrix *csr)
{
    sdl_sparse *sm = (sdl_sparse *)sp_calloc(1, sizeof(sdl_sparse));
    if (!sm) throw std::bad_alloc();
    sm->base.m = csr->m;
    sm->base.n = csr->n;
    sm->base.nnz = csr->nnz;
    sm->base.x = csr->x;
    sm->csr = csr;
    sm->impl = new SparseImpl();
    wire_sparse(sm);
    return &sm->base;
}

const DevStruct &sparse_dev_struct(sdl_sparse *A, cudaStream_t s)
{
    SparseImpl *im = A->impl;
    if (!im->st)
    {
        auto st = std::make_shared<DevStruct>();
        st->rows = A->csr->m;
        st->cols = A->csr->n;
        st->nnz = A->csr->nnz;
        st->p = upload(A->csr->p, (size_t)A->csr->m + 1, s);
        st->i = upload(A->csr->i, A->csr->nnz, s);
        validate_compressed(st->p.get(), st->i.get(), st->rows, st->cols, st->nnz, "sparse matrix", s);
        im->st = std::move(st);
    }
    return *im->st;
}

const double *sparse_dev_values(sdl_sparse *A, cudaStream_t s)
{
    DevValues &v = A->impl->vals;
    if (!v.x.get() || v.x.n < (size_t)std::max(1, A->csr->nnz)) v.x.reset(std::max(1, A->csr->nnz));
    if (!v.valid || v.seen != A->base.values_version)
    {
        h2d(v.x.get(), A->csr->x, A->csr->nnz, s);
        v.seen = A->base.values_version;
        v.valid = true;
    }
    return v.x.get();
}

const TransposePlan &sparse_dev_csc(sdl_sparse *A, cudaStream_t s)
{
    SparseImpl *im = A->impl;
    if (!im->csc)
    {
        const DevStruct &st = sparse_dev_struct(A, s);
        auto T = std::make_shared<TransposePlan>();
        transpose_build(st.p.get(), st.i.get(), st.rows, st.cols, st.nnz, *T, s);
        im->csc = std::move(T);
    }
    return *im->csc;
}

} // namespace sdl

using namespace sdl;

// ====================================================================== constructors
extern "C" matrix *new_sparse_matrix(CSR_matrix *A)
{
    return guard_upstream<matrix *>("new_sparse_matrix", nullptr, [&]() { return sparse_wrap(A); });
}

extern "C" matrix *new_sparse_matrix_alloc(int m, int n, int nnz)
{
    return new_sparse_matrix(new_CSR_matrix(m, n, nnz));
}

extern "C" void free_matrix(matrix *m)
{
    if (!m) return;
    if (m->kind == MATRIX_PERMUTED_DENSE)
        pd_free(as_pd(m));
    else if (m->kind == MATRIX_STACKED_PD)
        spd_free(as_spd(m));
    else
        sparse_free(as_sparse(m));
}

extern "C" matrix *copy_sparsity_matrices_alloc(const matrix *A)
{
    return guard_upstream<matrix *>("copy_sparsity_matrices_alloc", nullptr, [&]() -> matrix * {
        if (A->kind == MATRIX_PERMUTED_DENSE) return pd_copy_sparsity(as_pd(A));
        if (A->kind == MATRIX_STACKED_PD) return spd_copy_sparsity(as_spd(A));
        const CSR_matrix *src = as_sparse(A)->csr;
        CSR_matrix *csr = new_CSR_matrix(src->m, src->n, src->nnz);
        std::memcpy(csr->p, src->p, ((size_t)src->m + 1) * sizeof(int));
        if (src->nnz) std::memcpy(csr->i, src->i, (size_t)src->nnz * sizeof(int));
        matrix *C = sparse_wrap(csr);
        // share the device structure when A has one already
        as_sparse(C)->impl->st = as_sparse(A)->impl->st;
        return C;
    });
}

// ====================================================================== dispatchers
extern "C" matrix *BTA_matrices_alloc(matrix *A, matrix *B)
{
    return guard_upstream<matrix *>("BTA_matrices_alloc", nullptr, [&]() -> matrix * {
        if (!A || !B) fail(SDL_ERR_INVALID, "NULL operand");
        if (B->kind == MATRIX_SPARSE && A->kind == MATRIX_SPARSE)
            return sparse_product_alloc(as_sparse(B), 0, as_sparse(A));
        return dense_BTA_alloc(A, B);
    });
}

extern "C" void BTDA_matrices_fill_values(matrix *A, const double *d, matrix *B, matrix *C)
{
    guard_upstream_void("BTDA_matrices_fill_values", [&]() {
        if (!A || !B || !C) fail(SDL_ERR_INVALID, "NULL operand");
        if (B->kind == MATRIX_SPARSE && A->kind == MATRIX_SPARSE)
        {
            check_sparse(C, "C");
            sparse_product_fill(as_sparse(B), d, as_sparse(A), as_sparse(C));
            return;
        }
        dense_BTDA_fill(A, d, B, C);
    });
}

extern "C" void BTA_matrices_fill_values(matrix *A, matrix *B, matrix *C)
{
    BTDA_matrices_fill_values(A, nullptr, B, C);
}

extern "C" matrix *BA_matrices_alloc(const matrix *B, matrix *A)
{
    return guard_upstream<matrix *>("BA_matrices_alloc", nullptr, [&]() -> matrix * {
        if (!A || !B) fail(SDL_ERR_INVALID, "NULL operand");
        if (B->kind == MATRIX_STACKED_PD) fail(SDL_ERR_INVALID, "BA_matrices_alloc: B must not be stacked_pd");
        if (B->kind == MATRIX_SPARSE && A->kind == MATRIX_SPARSE)
            return sparse_product_alloc(as_sparse(B), 1, as_sparse(A));
        return dense_BA_alloc(B, A);
    });
}

extern "C" void BA_matrices_fill_values(const matrix *B, const matrix *A, matrix *C)
{
    guard_upstream_void("BA_matrices_fill_values", [&]() {
        if (!A || !B || !C) fail(SDL_ERR_INVALID, "NULL operand");
        if (B->kind == MATRIX_STACKED_PD) fail(SDL_ERR_INVALID, "BA_matrices_fill_values: B must not be stacked_pd");
        if (B->kind == MATRIX_SPARSE && A->kind == MATRIX_SPARSE)
        {
            check_sparse(C, "C");
            sparse_product_fill(as_sparse(B), nullptr, as_sparse(A), as_sparse(C));
            return;
        }
        dense_BA_fill(B, A, C);
    });
}

extern "C" matrix *ATA_matrices_alloc(matrix *A)
{
    return guard_upstream<matrix *>("ATA_matrices_alloc", nullptr, [&]() -> matrix * {
        if (!A) fail(SDL_ERR_INVALID, "NULL operand");
        if (A->kind == MATRIX_SPARSE) return sparse_product_alloc(as_sparse(A), 0, as_sparse(A));
        return dense_ATA_alloc(A);
    });
}

extern "C" void ATDA_matrices_fill_values(const matrix *A, const double *d, matrix *C)
{
    guard_upstream_void("ATDA_matrices_fill_values", [&]() {
        if (!A || !C) fail(SDL_ERR_INVALID, "NULL operand");
        if (A->kind != C->kind) fail(SDL_ERR_INVALID, "C must have A's kind");
        if (A->kind == MATRIX_SPARSE)
        {
            sdl_sparse *a = as_sparse(A);
            sparse_product_fill(a, d, a, as_sparse(C));
            return;
        }
        dense_ATDA_fill(A, d, C);
    });
}

extern "C" void DA_matrices_fill_values(const double *d, const matrix *A, matrix *C)
{
    guard_upstream_void("DA_matrices_fill_values", [&]() {
        if (!A || !C || !d) fail(SDL_ERR_INVALID, "NULL operand");
        if (A->kind != C->kind) fail(SDL_ERR_INVALID, "C must have A's kind");
        if (A->kind != MATRIX_SPARSE)
        {
            dense_DA_fill(d, A, C);
            return;
        }
        sdl_sparse *a = as_sparse(A), *c = as_sparse(C);
        if (a->csr->m != c->csr->m || a->csr->nnz != c->csr->nnz)
            fail(SDL_ERR_INVALID, "C must come from copy_sparsity_matrices_alloc(A)");
        cudaStream_t s = S();
        const DevStruct &st = sparse_dev_struct(a, s);
        const double *Ax = sparse_dev_values(a, s);
        auto *op = dynamic_cast<ScaleOp *>(c->impl->bound.get());
        if (!op)
        {
            // first DA fill into this output: set up its device buffers once
            auto fresh = std::make_unique<ScaleOp>();
            fresh->dvec.reset(std::max(1, a->csr->m));
            op = fresh.get();
            c->impl->bound = std::move(fresh);
        }
        if (!c->impl->vals.x.get() || c->impl->vals.x.n < (size_t)std::max(1, c->csr->nnz))
            c->impl->vals.x.reset(std::max(1, c->csr->nnz));
        h2d(op->dvec.get(), d, a->csr->m, s);
        scale_rows(st.p.get(), a->csr->m, op->dvec.get(), Ax, c->impl->vals.x.get(), s);
        publish_output(c, s);
    });
}

extern "C" matrix *transpose_matrices_alloc(const matrix *A)
{
    return guard_upstream<matrix *>("transpose_matrices_alloc", nullptr, [&]() -> matrix * {
        if (!A) fail(SDL_ERR_INVALID, "NULL operand");
        if (A->kind != MATRIX_SPARSE) return dense_transpose_alloc(A);
        sdl_sparse *a = as_sparse(A);
        cudaStream_t s = S();
        const TransposePlan &T = sparse_dev_csc(a, s);
        auto op = std::make_unique<TransposeOp>();
        op->T = a->impl->csc;
        op->A_m = a->csr->m;
        op->A_n = a->csr->n;
        op->A_nnz = a->csr->nnz;
        sdl_sparse *C = new_output(a->csr->n, a->csr->m, a->csr->nnz, T.Tp.get(), T.Ti.get(), s);
        C->impl->bound = std::move(op);
        return &C->base;
    });
}

extern "C" void transpose_matrices_fill_values(const matrix *A, matrix *AT)
{
    guard_upstream_void("transpose_matrices_fill_values", [&]() {
        if (!A || !AT) fail(SDL_ERR_INVALID, "NULL operand");
        if (A->kind != AT->kind) fail(SDL_ERR_INVALID, "AT must have A's kind");
        if (A->kind != MATRIX_SPARSE)
        {
            dense_transpose_fill(A, AT);
            return;
        }
        sdl_sparse *a = as_sparse(A), *c = as_sparse(AT);
        auto *op = dynamic_cast<TransposeOp *>(c->impl->bound.get());
        if (!op) fail(SDL_ERR_INVALID, "AT was not produced by transpose_matrices_alloc");
        if (op->A_m != a->csr->m || op->A_n != a->csr->n || op->A_nnz != a->csr->nnz)
            fail(SDL_ERR_INVALID, "A does not match the matrix AT was allocated for");
        cudaStream_t s = S();
        const double *Ax = sparse_dev_values(a, s);
        gather_values(op->T->src.get(), Ax, c->impl->vals.x.get(), a->csr->nnz, s);
        publish_output(c, s);
    });
}
