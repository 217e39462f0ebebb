// Kronecker products (upstream include/sparsediff_linalg/matmul_kron.h,
// src/matmul_kron_dispatchers.c):
//   y = kron(I_p, A) x                  BA_kron_vec_matrices
//   C = kron(I_p, A) J                  BA_kron_matrices_*   (p == 1: BA_matrices_*)
//   C = kron(A, I_m) J                  BA_dense_kron_I_matrices_*
// A sparse: C is the Gustavson product with L = A's rows repeated over p diagonal
// blocks (the `blocks` form of the product path), J read by its CSR (a dense-block
// J through its CSR view). A a full permuted_dense: blockwise dense-block fill
// programs (capi_dense_ops.cpp), C a stacked_pd.
#include <climits>

#include "capi_common.h"
#include "dense_impl.h"
#include "sparsediff_linalg/matmul.h"
#include "sparsediff_linalg/matmul_kron.h"
#include "sparsediff_linalg/matrix.h"

namespace sdl {

void kron_vec_csr(const int *Ap, const int *Ai, const double *Ax, int m, int n, int p, const double *x, double *y,
                  cudaStream_t s);
void kron_vec_dense(const double *A, int m, int n, int p, const double *x, double *y, cudaStream_t s);

namespace {

cudaStream_t S() { return runtime().stream; }

// J's CSR structure on the device and, for a stacked_pd J, the value index of
// each CSR position (its own values are block-major).
struct KronRight
{
    std::shared_ptr<DevStruct> st;
    DevBuf<int> perm;
    DevBuf<double> stage, csr_x;
    int kind = 0, m = 0, n = 0, nnz = 0;
};

void bind_right(KronRight &R, matrix *J, cudaStream_t s)
{
    R.kind = J->kind;
    R.m = J->m;
    R.n = J->n;
    R.nnz = J->nnz;
    if (J->kind == MATRIX_SPARSE)
    {
        sparse_dev_struct(as_sparse(J), s);
        R.st = as_sparse(J)->impl->st;
        return;
    }
    const CSR_matrix *v = J->to_csr(J); // the dense blocks' CSR pattern
    auto st = std::make_shared<DevStruct>();
    st->rows = v->m;
    st->cols = v->n;
    st->nnz = v->nnz;
    st->p = upload(v->p, (size_t)v->m + 1, s);
    st->i = upload(v->i, (size_t)v->nnz, s);
    R.st = std::move(st);
    R.csr_x.reset((size_t)std::max(1, J->nnz));
    if (J->kind == MATRIX_STACKED_PD)
    {
        const sdl_stacked *spd = as_spd(J);
        std::vector<int> perm((size_t)std::max(1, J->nnz));
        int vi = 0;
        for (int b = 0; b < spd->n_blocks; ++b)
        {
            const permuted_dense *blk = spd->blocks[b];
            for (int ii = 0; ii < blk->m0; ++ii)
                for (int jj = 0; jj < blk->n0; ++jj) perm[v->p[blk->row_perm[ii]] + jj] = vi++;
        }
        R.perm = upload(perm.data(), perm.size(), s);
        R.stage.reset((size_t)std::max(1, J->nnz));
    }
}

// J's values in CSR order, on the device.
const double *right_values(KronRight &R, const matrix *J, cudaStream_t s)
{
    if (R.kind == MATRIX_SPARSE) return sparse_dev_values(as_sparse(J), s);
    if (J->nnz == 0) return R.csr_x.get();
    if (R.kind == MATRIX_PERMUTED_DENSE)
    {
        h2d(R.csr_x.get(), J->x, (size_t)J->nnz, s);
        return R.csr_x.get();
    }
    h2d(R.stage.get(), J->x, (size_t)J->nnz, s);
    gather_values(R.perm.get(), R.stage.get(), R.csr_x.get(), J->nnz, s);
    return R.csr_x.get();
}

struct SparseKronOp : BoundOp
{
    std::shared_ptr<DevStruct> L;
    KronRight R;
    Product P;
    int p = 0, A_m = 0, A_n = 0, A_nnz = 0;
};

bool is_full_pd(const matrix *A)
{
    if (A->kind != MATRIX_PERMUTED_DENSE) return false;
    const permuted_dense *pd = as_pd(A);
    return pd->m0 == A->m && pd->n0 == A->n;
}

matrix *sparse_kron_alloc(matrix *Am, int p, matrix *J)
{
    sdl_sparse *A = as_sparse(Am);
    if ((long long)p * A->csr->n != J->m) fail(SDL_ERR_INVALID, "BA_kron_matrices_alloc: J must have p * A->n rows");
    if ((long long)p * A->csr->m > INT_MAX) fail(SDL_ERR_OVERFLOW, "BA_kron_matrices_alloc: p * A->m exceeds INT_MAX");
    cudaStream_t s = S();
    auto op = std::make_unique<SparseKronOp>();
    sparse_dev_struct(A, s);
    op->L = A->impl->st;
    bind_right(op->R, J, s);
    ProductDesc d;
    d.Lp = op->L->p.get();
    d.Li = op->L->i.get();
    d.L_m = A->csr->m;
    d.L_nnz = A->csr->nnz;
    d.blocks = p;
    d.Ap = op->R.st->p.get();
    d.Ai = op->R.st->i.get();
    d.A_m = J->m;
    d.A_n = J->n;
    d.A_nnz = J->nnz;
    product_symbolic(d, TuneConfig{}, op->P, s);
    op->p = p;
    op->A_m = A->csr->m;
    op->A_n = A->csr->n;
    op->A_nnz = A->csr->nnz;
    sdl_sparse *C = new_output(op->P.m_out, op->P.n, op->P.nnz, op->P.Cp.get(), op->P.Ci.get(), s);
    C->impl->bound = std::move(op);
    return &C->base;
}

void sparse_kron_fill(const matrix *Am, int p, const matrix *J, matrix *Cm)
{
    if (Cm->kind != MATRIX_SPARSE) fail(SDL_ERR_INVALID, "BA_kron_matrices_fill_values: C must be sparse here");
    sdl_sparse *C = as_sparse(Cm);
    auto *op = dynamic_cast<SparseKronOp *>(C->impl->bound.get());
    if (!op) fail(SDL_ERR_INVALID, "BA_kron_matrices_fill_values: C was not produced by BA_kron_matrices_alloc");
    sdl_sparse *A = as_sparse(Am);
    if (op->p != p || op->A_m != A->csr->m || op->A_n != A->csr->n || op->A_nnz != A->csr->nnz ||
        op->R.kind != (int)J->kind || op->R.m != J->m || op->R.n != J->n || op->R.nnz != J->nnz)
        fail(SDL_ERR_INVALID, "BA_kron_matrices_fill_values: operands do not match the alloc");
    cudaStream_t s = S();
    const double *Lx = sparse_dev_values(A, s);
    const double *Jx = right_values(op->R, J, s);
    product_numeric(op->P, Lx, nullptr, Jx, C->impl->vals.x.get(), s);
    publish_output(C, s);
}

} // namespace
} // namespace sdl

using namespace sdl;

extern "C" void BA_kron_vec_matrices(const matrix *A, const double *x, double *y, int p)
{
    guard_upstream_void("BA_kron_vec_matrices", [&]() {
        if (!A || p < 0 || (p > 0 && ((A->n > 0 && !x) || (A->m > 0 && !y))))
            fail(SDL_ERR_INVALID, "BA_kron_vec_matrices: bad arguments");
        if (A->kind == MATRIX_STACKED_PD) fail(SDL_ERR_INVALID, "BA_kron_vec_matrices: A must not be stacked_pd");
        if (A->kind == MATRIX_PERMUTED_DENSE && !is_full_pd(A))
            fail(SDL_ERR_INVALID, "BA_kron_vec_matrices: a permuted_dense A must cover its whole shape");
        const long long nx = (long long)p * A->n, ny = (long long)p * A->m;
        if (ny == 0) return;
        cudaStream_t s = S();
        DevBuf<double> dx((size_t)std::max<long long>(1, nx)), dy((size_t)ny);
        if (nx) h2d(dx.get(), x, (size_t)nx, s);
        if (A->kind == MATRIX_SPARSE)
        {
            sdl_sparse *a = as_sparse(A);
            const DevStruct &st = sparse_dev_struct(a, s);
            kron_vec_csr(st.p.get(), st.i.get(), sparse_dev_values(a, s), A->m, A->n, p, dx.get(), dy.get(), s);
        }
        else
        {
            DevBuf<double> dA((size_t)std::max(1, A->nnz));
            if (A->nnz) h2d(dA.get(), as_pd(A)->X, (size_t)A->nnz, s);
            kron_vec_dense(dA.get(), A->m, A->n, p, dx.get(), dy.get(), s);
            d2h(y, dy.get(), (size_t)ny, s);
            SDL_CUDA(cudaStreamSynchronize(s));
            return;
        }
        d2h(y, dy.get(), (size_t)ny, s);
        SDL_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" matrix *BA_kron_matrices_alloc(const matrix *A, int p, matrix *J)
{
    return guard_upstream<matrix *>("BA_kron_matrices_alloc", nullptr, [&]() -> matrix * {
        if (!A || !J || p < 0) fail(SDL_ERR_INVALID, "BA_kron_matrices_alloc: bad arguments");
        if (p == 1) return BA_matrices_alloc(A, J);
        if (A->kind == MATRIX_PERMUTED_DENSE) return prog_dense_kron_alloc(A, p, J, false);
        if (A->kind != MATRIX_SPARSE) fail(SDL_ERR_INVALID, "BA_kron_matrices_alloc: A must not be stacked_pd");
        return sparse_kron_alloc(const_cast<matrix *>(A), p, J);
    });
}

extern "C" void BA_kron_matrices_fill_values(const matrix *A, int p, matrix *J, matrix *C)
{
    guard_upstream_void("BA_kron_matrices_fill_values", [&]() {
        if (!A || !J || !C) fail(SDL_ERR_INVALID, "BA_kron_matrices_fill_values: NULL operand");
        if (p == 1)
        {
            BA_matrices_fill_values(A, J, C);
            return;
        }
        if (A->kind == MATRIX_PERMUTED_DENSE)
            prog_dense_kron_fill(A, p, J, C);
        else if (A->kind == MATRIX_SPARSE)
            sparse_kron_fill(A, p, J, C);
        else
            fail(SDL_ERR_INVALID, "BA_kron_matrices_fill_values: A must not be stacked_pd");
    });
}

extern "C" matrix *BA_dense_kron_I_matrices_alloc(const matrix *A, int m, matrix *J)
{
    return guard_upstream<matrix *>("BA_dense_kron_I_matrices_alloc", nullptr, [&]() -> matrix * {
        if (!A || !J) fail(SDL_ERR_INVALID, "BA_dense_kron_I_matrices_alloc: NULL operand");
        return prog_dense_kron_alloc(A, m, J, true);
    });
}

extern "C" void BA_dense_kron_I_matrices_fill_values(const matrix *A, int m, const matrix *J, matrix *C)
{
    guard_upstream_void("BA_dense_kron_I_matrices_fill_values", [&]() {
        if (!A || !J || !C) fail(SDL_ERR_INVALID, "BA_dense_kron_I_matrices_fill_values: NULL operand");
        prog_dense_kron_fill(A, m, J, C);
    });
}
