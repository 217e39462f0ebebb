// Matrix sums and vstack (upstream include/sparsediff_linalg/matrix_sum.h,
// matrix_vstack.h; src/sparse/matrix_sum.c, src/sparse/CSR_sum.c:1-297,
// src/sparse/matrix_vstack.c).
//
// A sum of n operands is the coalescing of their entries, taken as (row, column,
// value) triplets in operand order: every output entry sums its duplicates from
// +0.0 in ascending triplet order, which is upstream's memset + accumulator over
// the operands in order (each operand holds a cell at most once). The triplets of
// an operand follow its own value array op->x (CSR order for sparse and
// permuted_dense, block-major for stacked_pd, as upstream's composed index maps
// read it), so a fill stages the operands' values back to back and runs the
// coalescing product. The scaled two-operand sum gives each triplet the factor
// d1[row] or d2[row] (one rounding, as upstream's d * x). fill_add scatters one
// operand into the running sum through the triplet -> output position map.
//
// vstack concatenates the operands' CSR views; its fill copies the operands whose
// values_version moved since the previous fill (every operand after C itself was
// written), on the device, and reads back the copied ranges.
#include <climits>
#include <cstring>

#include "capi_common.h"
#include "matrix_kinds.h"
#include "sparsediff_linalg/matrix.h"
#include "sparsediff_linalg/matrix_sum.h"
#include "sparsediff_linalg/matrix_vstack.h"
#include "sparsediff_linalg/tracked_alloc.h"

namespace sdl {

void coalesce_fill_scaled(const sdl_coalesce *C, const double *x, const double *d, double *Cx, cudaStream_t s);
void sum_positions(const int *rows, const int *cols, int n, const int *Cp, const int *Ci, int *map, cudaStream_t s);
void sum_factors(const int *rows, int n, int split, const double *d1, const double *d2, double *f, cudaStream_t s);
void scatter_add(const int *map, const double *x, int n, double *C, cudaStream_t s);
void scatter_copy(const int *pos, const double *x, int n, double *C, cudaStream_t s);

namespace {

cudaStream_t S() { return runtime().stream; }

struct Shape
{
    int m, n, nnz, kind;
    bool operator==(const Shape &o) const { return m == o.m && n == o.n && nnz == o.nnz && kind == o.kind; }
};
Shape shape_of(const matrix *op) { return Shape{op->m, op->n, op->nnz, (int)op->kind}; }

// (row, column) of every entry of an operand, in the order of its value array.
void triplets_of(const matrix *op, std::vector<int> &rows, std::vector<int> &cols)
{
    if (op->kind == MATRIX_SPARSE)
    {
        const CSR_matrix *A = as_sparse(op)->csr;
        for (int r = 0; r < A->m; ++r)
            for (int q = A->p[r]; q < A->p[r + 1]; ++q)
            {
                rows.push_back(r);
                cols.push_back(A->i[q]);
            }
        return;
    }
    auto block = [&](const permuted_dense *b) {
        for (int ii = 0; ii < b->m0; ++ii)
            for (int jj = 0; jj < b->n0; ++jj)
            {
                rows.push_back(b->row_perm[ii]);
                cols.push_back(b->col_perm[jj]);
            }
    };
    if (op->kind == MATRIX_PERMUTED_DENSE)
        block(as_pd(op));
    else
        for (int k = 0; k < as_spd(op)->n_blocks; ++k) block(as_spd(op)->blocks[k]);
}

// The values of an operand, in the order of its value array, into dst (device).
void stage_values(const matrix *op, double *dst, cudaStream_t s)
{
    if (op->nnz <= 0) return;
    if (op->kind == MATRIX_SPARSE)
    {
        const double *src = sparse_dev_values(as_sparse(op), s);
        SDL_CUDA(cudaMemcpyAsync(dst, src, (size_t)op->nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    else
        h2d(dst, op->x, (size_t)op->nnz, s);
}

// ------------------------------------------------------------------ sums
struct SumOp : BoundOp
{
    int n_ops = 0, m = 0, ncols = 0, total = 0;
    std::vector<Shape> shapes;
    std::vector<int> off; // first triplet of each operand (n_ops + 1)
    sdl_coalesce *plan = nullptr;
    DevBuf<int> rows, map;
    DevBuf<double> x, f, d1, d2;
    ~SumOp() override { sdl_coalesce_destroy(plan); }
};

std::unique_ptr<SumOp> build_sum(matrix *const *ops, int n, cudaStream_t s)
{
    if (n < 1 || !ops) fail(SDL_ERR_INVALID, "sum of matrices: needs at least one operand");
    auto op = std::make_unique<SumOp>();
    op->n_ops = n;
    for (int k = 0; k < n; ++k)
        if (!ops[k]) fail(SDL_ERR_INVALID, "sum of matrices: NULL operand");
    op->m = ops[0]->m;
    op->ncols = ops[0]->n;
    std::vector<int> rows, cols;
    long long total = 0;
    op->off.push_back(0);
    for (int k = 0; k < n; ++k)
    {
        if (ops[k]->m != op->m || ops[k]->n != op->ncols) fail(SDL_ERR_INVALID, "sum of matrices: operand shapes differ");
        op->shapes.push_back(shape_of(ops[k]));
        total += ops[k]->nnz;
        if (total > INT_MAX) fail(SDL_ERR_OVERFLOW, "sum of matrices: more than INT_MAX entries");
        triplets_of(ops[k], rows, cols);
        op->off.push_back((int)total);
    }
    if ((long long)rows.size() != total) fail(SDL_ERR_INTERNAL, "sum of matrices: operand entry count mismatch");
    op->total = (int)total;
    op->rows = upload(rows.data(), rows.size(), s);
    DevBuf<int> dcols = upload(cols.data(), cols.size(), s);
    sdl_status st = sdl_coalesce_create(op->rows.get(), dcols.get(), op->total, op->m, op->ncols, s, &op->plan);
    if (st != SDL_OK) fail(st, sdl_last_error());
    const int *Cp = nullptr, *Ci = nullptr;
    sdl_coalesce_info(op->plan, nullptr, &Cp, &Ci);
    op->map.reset((size_t)std::max(1, op->total));
    sum_positions(op->rows.get(), dcols.get(), op->total, Cp, Ci, op->map.get(), s);
    check_device_errors(s, "sum of matrices");
    op->x.reset((size_t)std::max(1, op->total));
    return op;
}

SumOp *sum_op_of(matrix *C, const char *what)
{
    if (!C || C->kind != MATRIX_SPARSE) fail(SDL_ERR_INVALID, std::string(what) + ": C must be a sparse matrix");
    auto *op = dynamic_cast<SumOp *>(as_sparse(C)->impl->bound.get());
    if (!op) fail(SDL_ERR_INVALID, std::string(what) + ": C was not produced by the matching alloc");
    return op;
}

void check_operands(const SumOp &op, matrix *const *ops, int n, const char *what)
{
    if (n != op.n_ops) fail(SDL_ERR_INVALID, std::string(what) + ": operand count differs from the alloc");
    for (int k = 0; k < n; ++k)
        if (!ops[k] || !(shape_of(ops[k]) == op.shapes[k]))
            fail(SDL_ERR_INVALID, std::string(what) + ": operands do not match the alloc");
}

void sum_fill(SumOp &op, matrix *const *ops, sdl_sparse *C, const double *f, cudaStream_t s)
{
    for (int k = 0; k < op.n_ops; ++k) stage_values(ops[k], op.x.get() + op.off[k], s);
    coalesce_fill_scaled(op.plan, op.x.get(), f, C->impl->vals.x.get(), s);
    publish_output(C, s);
}

sdl_sparse *sum_output(SumOp &op, cudaStream_t s)
{
    int nnz = 0;
    const int *Cp = nullptr, *Ci = nullptr;
    sdl_coalesce_info(op.plan, &nnz, &Cp, &Ci);
    return new_output(op.m, op.ncols, nnz, Cp, Ci, s);
}

// ------------------------------------------------------------------ vstack
struct VstackOp : BoundOp
{
    int n_ops = 0;
    std::vector<Shape> shapes;
    std::vector<int> nnz_off;
    std::vector<DevBuf<int>> pos; // stacked_pd operands: block-major value -> C position
    std::vector<uint64_t> seen;
    uint64_t C_seen = 0;
    DevBuf<double> scratch;
};

} // namespace
} // namespace sdl

using namespace sdl;

extern "C" void sum_matrices_alloc(matrix *A, matrix *B, matrix *C)
{
    guard_upstream_void("sum_matrices_alloc", [&]() {
        if (!A || !B || !C) fail(SDL_ERR_INVALID, "NULL operand");
        if (C->kind != MATRIX_SPARSE) fail(SDL_ERR_INVALID, "sum_matrices_alloc: C must be a sparse matrix");
        cudaStream_t s = S();
        matrix *ops[2] = {A, B};
        auto op = build_sum(ops, 2, s);
        sdl_sparse *Cs = as_sparse(C);
        CSR_matrix *csr = Cs->csr;
        int nnz = 0;
        const int *Cp = nullptr, *Ci = nullptr;
        sdl_coalesce_info(op->plan, &nnz, &Cp, &Ci);
        // upstream sum_csr_alloc writes the merged pattern into C's arrays, which the
        // caller sized for nnz(A) + nnz(B), then trims them
        if (csr->m != op->m || csr->n != op->ncols) fail(SDL_ERR_INVALID, "sum_matrices_alloc: C has another shape");
        if (csr->nnz < nnz) fail(SDL_ERR_INVALID, "sum_matrices_alloc: C has room for fewer entries than A + B");
        d2h(csr->p, Cp, (size_t)op->m + 1, s);
        d2h(csr->i, Ci, (size_t)nnz, s);
        SDL_CUDA(cudaStreamSynchronize(s));
        CSR_trim(csr);
        C->x = csr->x;
        C->nnz = csr->nnz;
        SparseImpl *im = Cs->impl;
        im->st.reset();
        im->csc.reset();
        im->vals = DevValues{};
        im->vals.x.reset((size_t)std::max(1, nnz));
        im->bound = std::move(op);
    });
}

extern "C" void sum_matrices_fill_values(matrix *A, matrix *B, matrix *C)
{
    guard_upstream_void("sum_matrices_fill_values", [&]() {
        SumOp *op = sum_op_of(C, "sum_matrices_fill_values");
        matrix *ops[2] = {A, B};
        check_operands(*op, ops, 2, "sum_matrices_fill_values");
        sum_fill(*op, ops, as_sparse(C), nullptr, S());
    });
}

extern "C" void sum_scaled_matrices_fill_values(matrix *A, matrix *B, matrix *C, const double *d1,
                                                const double *d2)
{
    guard_upstream_void("sum_scaled_matrices_fill_values", [&]() {
        SumOp *op = sum_op_of(C, "sum_scaled_matrices_fill_values");
        matrix *ops[2] = {A, B};
        check_operands(*op, ops, 2, "sum_scaled_matrices_fill_values");
        if (op->m > 0 && (!d1 || !d2)) fail(SDL_ERR_INVALID, "sum_scaled_matrices_fill_values: NULL scaling");
        cudaStream_t s = S();
        if (!op->f.get())
        {
            op->f.reset((size_t)std::max(1, op->total));
            op->d1.reset((size_t)std::max(1, op->m));
            op->d2.reset((size_t)std::max(1, op->m));
        }
        h2d(op->d1.get(), d1, (size_t)op->m, s);
        h2d(op->d2.get(), d2, (size_t)op->m, s);
        sum_factors(op->rows.get(), op->total, op->off[1], op->d1.get(), op->d2.get(), op->f.get(), s);
        sum_fill(*op, ops, as_sparse(C), op->f.get(), s);
    });
}

extern "C" matrix *sum_4_matrices_alloc(matrix *A, matrix *B, matrix *D, matrix *E)
{
    return guard_upstream<matrix *>("sum_4_matrices_alloc", nullptr, [&]() -> matrix * {
        matrix *ops[4] = {A, B, D, E};
        cudaStream_t s = S();
        auto op = build_sum(ops, 4, s);
        sdl_sparse *C = sum_output(*op, s);
        C->impl->bound = std::move(op);
        return &C->base;
    });
}

extern "C" void sum_4_matrices_fill_values(const matrix *A, const matrix *B, const matrix *D, const matrix *E,
                                           matrix *C)
{
    guard_upstream_void("sum_4_matrices_fill_values", [&]() {
        SumOp *op = sum_op_of(C, "sum_4_matrices_fill_values");
        matrix *ops[4] = {const_cast<matrix *>(A), const_cast<matrix *>(B), const_cast<matrix *>(D),
                          const_cast<matrix *>(E)};
        check_operands(*op, ops, 4, "sum_4_matrices_fill_values");
        sum_fill(*op, ops, as_sparse(C), nullptr, S());
    });
}

extern "C" matrix *sum_n_matrices_alloc(matrix *const *ops, int n)
{
    return guard_upstream<matrix *>("sum_n_matrices_alloc", nullptr, [&]() -> matrix * {
        cudaStream_t s = S();
        auto op = build_sum(ops, n, s);
        sdl_sparse *C = sum_output(*op, s);
        C->impl->bound = std::move(op);
        return &C->base;
    });
}

extern "C" void sum_n_matrices_fill_values(matrix *const *ops, int n, matrix *C)
{
    guard_upstream_void("sum_n_matrices_fill_values", [&]() {
        SumOp *op = sum_op_of(C, "sum_n_matrices_fill_values");
        if (!ops) fail(SDL_ERR_INVALID, "NULL operand list");
        check_operands(*op, ops, n, "sum_n_matrices_fill_values");
        sum_fill(*op, ops, as_sparse(C), nullptr, S());
    });
}

extern "C" void sum_n_matrices_fill_zero(matrix *C)
{
    guard_upstream_void("sum_n_matrices_fill_zero", [&]() {
        sum_op_of(C, "sum_n_matrices_fill_zero");
        sdl_sparse *Cs = as_sparse(C);
        cudaStream_t s = S();
        if (Cs->csr->nnz)
            SDL_CUDA(cudaMemsetAsync(Cs->impl->vals.x.get(), 0, (size_t)Cs->csr->nnz * sizeof(double), s));
        publish_output(Cs, s);
    });
}

extern "C" void sum_n_matrices_fill_add(const matrix *opm, int k, matrix *C)
{
    guard_upstream_void("sum_n_matrices_fill_add", [&]() {
        SumOp *op = sum_op_of(C, "sum_n_matrices_fill_add");
        if (!opm || k < 0 || k >= op->n_ops || !(shape_of(opm) == op->shapes[k]))
            fail(SDL_ERR_INVALID, "sum_n_matrices_fill_add: operand does not match the alloc");
        sdl_sparse *Cs = as_sparse(C);
        cudaStream_t s = S();
        DevValues &cv = Cs->impl->vals;
        // C->x is the running sum; bring the device copy up to it if it was written
        if (!cv.valid || cv.seen != C->values_version) h2d(cv.x.get(), Cs->csr->x, (size_t)Cs->csr->nnz, s);
        double *xk = op->x.get() + op->off[k];
        stage_values(opm, xk, s);
        scatter_add(op->map.get() + op->off[k], xk, opm->nnz, cv.x.get(), s);
        publish_output(Cs, s);
    });
}

extern "C" matrix *vstack_matrices_alloc(matrix *const *ops, int n)
{
    return guard_upstream<matrix *>("vstack_matrices_alloc", nullptr, [&]() -> matrix * {
        if (n < 1 || !ops) fail(SDL_ERR_INVALID, "vstack_matrices_alloc: needs at least one operand");
        auto op = std::make_unique<VstackOp>();
        op->n_ops = n;
        long long m_total = 0, nnz_total = 0;
        for (int k = 0; k < n; ++k)
        {
            if (!ops[k]) fail(SDL_ERR_INVALID, "vstack_matrices_alloc: NULL operand");
            if (ops[k]->n != ops[0]->n) fail(SDL_ERR_INVALID, "vstack_matrices_alloc: operands differ in columns");
            m_total += ops[k]->m;
            nnz_total += ops[k]->nnz;
        }
        if (m_total > INT_MAX || nnz_total > INT_MAX) fail(SDL_ERR_OVERFLOW, "vstack_matrices_alloc: result too large");
        CSR_matrix *csr = new_CSR_matrix((int)m_total, ops[0]->n, (int)nnz_total);
        if (!csr) fail(SDL_ERR_INTERNAL, "vstack_matrices_alloc: allocation failed");
        cudaStream_t s = S();
        int row_off = 0, nnz_off = 0, max_spd = 0;
        csr->p[0] = 0;
        for (int k = 0; k < n; ++k)
        {
            matrix *A = ops[k];
            const CSR_matrix *v = A->to_csr(A); // the operand's CSR view (pattern of its blocks)
            for (int r = 1; r <= A->m; ++r) csr->p[row_off + r] = nnz_off + v->p[r];
            if (A->nnz) std::memcpy(csr->i + nnz_off, v->i, (size_t)A->nnz * sizeof(int));
            op->shapes.push_back(shape_of(A));
            op->nnz_off.push_back(nnz_off);
            op->pos.emplace_back();
            if (A->kind == MATRIX_STACKED_PD && A->nnz)
            {
                // block-major value -> its CSR position in C (a block row is its
                // block's col_perm, in order)
                const sdl_stacked *spd = as_spd(A);
                std::vector<int> pos;
                pos.reserve(A->nnz);
                for (int b = 0; b < spd->n_blocks; ++b)
                {
                    const permuted_dense *blk = spd->blocks[b];
                    for (int ii = 0; ii < blk->m0; ++ii)
                        for (int jj = 0; jj < blk->n0; ++jj) pos.push_back(nnz_off + v->p[blk->row_perm[ii]] + jj);
                }
                op->pos.back() = upload(pos.data(), pos.size(), s);
                max_spd = std::max(max_spd, A->nnz);
            }
            row_off += A->m;
            nnz_off += A->nnz;
        }
        op->scratch.reset((size_t)std::max(1, max_spd));
        op->seen.assign(n, 0);
        SDL_CUDA(cudaStreamSynchronize(s));
        sdl_sparse *C = as_sparse(sparse_wrap(csr));
        C->impl->vals.x.reset((size_t)std::max<long long>(1, nnz_total));
        op->C_seen = C->base.values_version - 1; // the first fill copies every operand
        C->impl->bound = std::move(op);
        return &C->base;
    });
}

extern "C" void vstack_matrices_fill_values(matrix *const *ops, int n, matrix *C)
{
    guard_upstream_void("vstack_matrices_fill_values", [&]() {
        if (!C || C->kind != MATRIX_SPARSE || !ops) fail(SDL_ERR_INVALID, "vstack_matrices_fill_values: bad arguments");
        sdl_sparse *Cs = as_sparse(C);
        auto *op = dynamic_cast<VstackOp *>(Cs->impl->bound.get());
        if (!op) fail(SDL_ERR_INVALID, "vstack_matrices_fill_values: C was not produced by vstack_matrices_alloc");
        if (n != op->n_ops) fail(SDL_ERR_INVALID, "vstack_matrices_fill_values: operand count differs from the alloc");
        for (int k = 0; k < n; ++k)
            if (!ops[k] || !(shape_of(ops[k]) == op->shapes[k]))
                fail(SDL_ERR_INVALID, "vstack_matrices_fill_values: operands do not match the alloc");
        cudaStream_t s = S();
        double *Cx = Cs->impl->vals.x.get();
        const bool copy_all = op->C_seen != C->values_version;
        bool changed = false;
        for (int k = 0; k < n; ++k)
        {
            matrix *A = ops[k];
            if ((copy_all || op->seen[k] != A->values_version) && A->nnz > 0)
            {
                const int off = op->nnz_off[k];
                if (A->kind == MATRIX_STACKED_PD)
                {
                    stage_values(A, op->scratch.get(), s);
                    scatter_copy(op->pos[k].get(), op->scratch.get(), A->nnz, Cx, s);
                }
                else
                    stage_values(A, Cx + off, s);
                d2h(Cs->csr->x + off, Cx + off, (size_t)A->nnz, s);
                changed = true;
            }
            op->seen[k] = A->values_version;
        }
        SDL_CUDA(cudaStreamSynchronize(s));
        if (changed) matrix_values_changed(C);
        op->C_seen = C->values_version;
        Cs->impl->vals.seen = C->values_version;
        Cs->impl->vals.valid = true;
    });
}
