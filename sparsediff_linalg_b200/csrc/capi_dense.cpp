// permuted_dense and stacked_pd kinds (upstream src/permuted_dense/permuted_dense.c,
// src/stacked_pd/stacked_pd.c): constructors, destructors, CSR views and the
// product dispatch for operand pairs that involve a dense-block kind.
#include <climits>
#include <cstring>

#include "capi_common.h"
#include "dense_impl.h"
#include "sparsediff_linalg/matrix.h"
#include "sparsediff_linalg/tracked_alloc.h"

namespace sdl {

const double *sparse_dev_values(sdl_sparse *A, cudaStream_t s);

namespace {

// CSR pattern of row-disjoint dense blocks (upstream permuted_dense.c:344-385):
// each dense row contributes a copy of its block's col_perm.
void blocks_csr_pattern(permuted_dense *const *blocks, int n_blocks, int m, int *Cp, int *Ci)
{
    std::memset(Cp, 0, ((size_t)m + 1) * sizeof(int));
    for (int k = 0; k < n_blocks; ++k)
        for (int ii = 0; ii < blocks[k]->m0; ++ii) Cp[blocks[k]->row_perm[ii] + 1] = blocks[k]->n0;
    for (int r = 0; r < m; ++r) Cp[r + 1] += Cp[r];
    for (int k = 0; k < n_blocks; ++k)
        for (int ii = 0; ii < blocks[k]->m0; ++ii)
            if (blocks[k]->n0)
                std::memcpy(Ci + Cp[blocks[k]->row_perm[ii]], blocks[k]->col_perm,
                            (size_t)blocks[k]->n0 * sizeof(int));
}

CSR_matrix *pd_to_csr(matrix *self)
{
    permuted_dense *pd = as_pd(self);
    if (!pd->csr_cache)
    {
        CSR_matrix *C = new_CSR_matrix(pd->base.m, pd->base.n, pd->m0 * pd->n0);
        sp_free(C->x);
        C->x = pd->X; // values alias the block (upstream permuted_dense.c:314-330)
        permuted_dense *one = pd;
        blocks_csr_pattern(&one, 1, pd->base.m, C->p, C->i);
        pd->csr_cache = C;
    }
    return pd->csr_cache;
}

void wire_pd(permuted_dense *pd)
{
    pd->base.kind = MATRIX_PERMUTED_DENSE;
    pd->base.to_csr = pd_to_csr;
    pd->base.row_gather_alloc = pd_row_gather_alloc;
    pd->base.row_gather_fill_values = dense_rows_fill;
    pd->base.row_reduce_alloc = pd_row_reduce_alloc;
    pd->base.row_reduce_fill_values = dense_rows_fill;
}

CSR_matrix *spd_to_csr(matrix *self)
{
    sdl_stacked *spd = as_spd(self);
    if (!spd->csr_cache)
    {
        CSR_matrix *C = new_CSR_matrix(spd->base.m, spd->base.n, spd->base.nnz);
        blocks_csr_pattern(spd->blocks, spd->n_blocks, spd->base.m, C->p, C->i);
        spd->csr_cache = C;
    }
    // values: scatter the blocks' rows (upstream stacked_pd.c:65-86 refreshes iff
    // the version moved; the copy is cheap and always current here)
    CSR_matrix *C = spd->csr_cache;
    for (int k = 0; k < spd->n_blocks; ++k)
    {
        permuted_dense *b = spd->blocks[k];
        for (int ii = 0; ii < b->m0; ++ii)
            if (b->n0)
                std::memcpy(C->x + C->p[b->row_perm[ii]], b->X + (size_t)ii * b->n0,
                            (size_t)b->n0 * sizeof(double));
    }
    return C;
}

void wire_spd(sdl_stacked *spd)
{
    spd->base.kind = MATRIX_STACKED_PD;
    spd->base.to_csr = spd_to_csr;
    spd->base.row_gather_alloc = spd_row_gather_alloc;
    spd->base.row_gather_fill_values = dense_rows_fill;
    spd->base.row_reduce_alloc = spd_row_reduce_alloc;
    spd->base.row_reduce_fill_values = dense_rows_fill;
}

[[noreturn]] void unsupported(const char *what)
{
    fail(SDL_ERR_UNSUPPORTED, std::string(what) +
                                  ": this operand-kind combination is not provided by the B200 build");
}

} // namespace

void pd_free(permuted_dense *pd)
{
    sp_free(pd->row_perm);
    sp_free(pd->col_perm);
    sp_free(pd->row_inv);
    sp_free(pd->col_inv);
    if (pd->csr_cache)
    {
        pd->csr_cache->x = nullptr;
        free_CSR_matrix(pd->csr_cache);
    }
    if (pd->owns_X) sp_free(pd->X);
    delete pd->impl;
    sp_free(pd);
}

void spd_free(sdl_stacked *spd)
{
    for (int k = 0; k < spd->n_blocks; ++k) free_matrix(&spd->blocks[k]->base);
    sp_free(spd->blocks);
    sp_free(spd->src_block_idx_p);
    sp_free(spd->src_block_idx);
    free_CSR_matrix(spd->csr_cache);
    sp_free(spd->values);
    delete spd->impl;
    sp_free(spd);
}

matrix *pd_copy_sparsity(const permuted_dense *A)
{
    return new_permuted_dense(A->base.m, A->base.n, A->m0, A->n0, A->row_perm, A->col_perm, nullptr);
}

matrix *spd_copy_sparsity(const sdl_stacked *A)
{
    permuted_dense **blocks = (permuted_dense **)sp_malloc(sizeof(permuted_dense *) * std::max(1, A->n_blocks));
    for (int k = 0; k < A->n_blocks; ++k) blocks[k] = as_pd(pd_copy_sparsity(A->blocks[k]));
    // identity source map (upstream stacked_pd_linalg.c:34-47 passes NULL)
    matrix *C = new_stacked_pd(A->base.m, A->base.n, A->n_blocks, blocks, nullptr, nullptr);
    sp_free(blocks);
    return C;
}

// BTA with B sparse and A permuted_dense / stacked_pd (upstream matmul_dispatchers.c:
// 335-375 -> BTA_csc_pd_* / BTA_csc_spd_*): C = B^T diag(d) A, each block's partial
// bit-identical to upstream's, coalesced as upstream's stacked_pd.
namespace {
struct BlockView
{
    std::vector<int> m0, n0;
    std::vector<const int *> rp, cp;
    int m = 0, n = 0;
    const double *host_x = nullptr; // the blocks' values, block-major
};
BlockView blocks_of(const matrix *Am)
{
    BlockView v;
    if (Am->kind == MATRIX_PERMUTED_DENSE)
    {
        const permuted_dense *A = as_pd(Am);
        v.m0 = {A->m0};
        v.n0 = {A->n0};
        v.rp = {A->row_perm};
        v.cp = {A->col_perm};
        v.host_x = A->X;
    }
    else
    {
        const sdl_stacked *A = as_spd(Am);
        for (int k = 0; k < A->n_blocks; ++k)
        {
            v.m0.push_back(A->blocks[k]->m0);
            v.n0.push_back(A->blocks[k]->n0);
            v.rp.push_back(A->blocks[k]->row_perm);
            v.cp.push_back(A->blocks[k]->col_perm);
        }
        v.host_x = A->values;
    }
    v.m = Am->m;
    v.n = Am->n;
    return v;
}
} // namespace

matrix *dense_BTA_alloc(matrix *Am, matrix *Bm)
{
    if (Bm->kind != MATRIX_SPARSE) return prog_BTA_alloc(Am, Bm);
    if (Am->kind != MATRIX_PERMUTED_DENSE && Am->kind != MATRIX_STACKED_PD) unsupported("BTA_matrices_alloc");
    sdl_sparse *B = as_sparse(Bm);
    if (B->csr->m != Am->m) fail(SDL_ERR_INVALID, "BTA_matrices_alloc: B and A have different row counts");
    cudaStream_t s = runtime().stream;
    BlockView v = blocks_of(Am);
    const int nb = (int)v.m0.size();
    auto plan = blocks_btda_build(nb, v.m0.data(), v.n0.data(), v.rp.data(), v.cp.data(), v.m, v.n, B->csr->p,
                                  B->csr->i, B->csr->n, s);
    sparse_dev_values(B, s); // the device mirror of B's values exists before any fill
    matrix *Cm = nullptr;
    if (Am->kind == MATRIX_PERMUTED_DENSE)
    {
        // one block: rows = the columns of B that reach A's rows (upstream permuted_dense_linalg.c:646-672)
        const std::vector<int> &act = plan->act[0];
        const permuted_dense *A = as_pd(Am);
        Cm = new_permuted_dense(B->csr->n, A->base.n, (int)act.size(), A->n0, act.empty() ? nullptr : act.data(),
                                A->col_perm, nullptr);
        if (!Cm) fail(SDL_ERR_INTERNAL, "BTA_matrices_alloc: output allocation failed");
        permuted_dense *C = as_pd(Cm);
        C->impl->bvals.reset((size_t)std::max<long long>(1, plan->x_total));
        C->impl->cvals.reset((size_t)std::max<long long>(1, plan->c_total));
        C->impl->dvec.reset((size_t)std::max(1, v.m));
        C->impl->ata = std::move(plan);
        SDL_CUDA(cudaStreamSynchronize(s));
        return Cm;
    }
    const int no = plan->n_out;
    permuted_dense **blocks = (permuted_dense **)sp_malloc(sizeof(permuted_dense *) * std::max(1, no));
    std::vector<int> sp_p(1, 0), sp_i;
    for (int o = 0; o < no; ++o)
    {
        const std::vector<int> &r = plan->out_rows[o], &c = plan->out_cols[o];
        blocks[o] = as_pd(new_permuted_dense(B->csr->n, v.n, (int)r.size(), (int)c.size(), r.data(), c.data(), nullptr));
        if (!blocks[o]) fail(SDL_ERR_INTERNAL, "BTA_matrices_alloc: output allocation failed");
        sp_i.insert(sp_i.end(), plan->out_srcs[o].begin(), plan->out_srcs[o].end());
        sp_p.push_back((int)sp_i.size());
    }
    if (sp_i.empty()) sp_i.push_back(0);
    Cm = new_stacked_pd(B->csr->n, v.n, no, blocks, sp_p.data(), sp_i.data());
    sp_free(blocks);
    if (!Cm) fail(SDL_ERR_INTERNAL, "BTA_matrices_alloc: output allocation failed");
    sdl_stacked *C = as_spd(Cm);
    C->impl->xvals.reset((size_t)std::max<long long>(1, plan->x_total));
    C->impl->cvals.reset((size_t)std::max<long long>(1, plan->c_total));
    C->impl->dvec.reset((size_t)std::max(1, v.m));
    C->impl->ata = std::move(plan);
    SDL_CUDA(cudaStreamSynchronize(s));
    return Cm;
}

void dense_BTDA_fill(matrix *Am, const double *d, matrix *Bm, matrix *Cm)
{
    if (ProgState *ps = prog_state(Cm); ps && ps->op == DP_OP_BTA)
    {
        prog_product_fill(Bm, d, Am, Cm, DP_OP_BTA);
        return;
    }
    if (Bm->kind != MATRIX_SPARSE || Am->kind != Cm->kind ||
        (Am->kind != MATRIX_PERMUTED_DENSE && Am->kind != MATRIX_STACKED_PD))
        unsupported("BTDA_matrices_fill_values");
    cudaStream_t s = runtime().stream;
    const BlocksAtaPlan *P = nullptr;
    DevBuf<double> *xv = nullptr, *cv = nullptr, *dv = nullptr;
    double *hc = nullptr;
    if (Cm->kind == MATRIX_PERMUTED_DENSE)
    {
        permuted_dense *C = as_pd(Cm);
        P = C->impl ? C->impl->ata.get() : nullptr;
        if (P)
        {
            xv = &C->impl->bvals;
            cv = &C->impl->cvals;
            dv = &C->impl->dvec;
            hc = C->X;
        }
    }
    else
    {
        sdl_stacked *C = as_spd(Cm);
        P = C->impl ? C->impl->ata.get() : nullptr;
        if (P)
        {
            xv = &C->impl->xvals;
            cv = &C->impl->cvals;
            dv = &C->impl->dvec;
            hc = C->values;
        }
    }
    if (!P || !P->btda) fail(SDL_ERR_INVALID, "BTDA_matrices_fill_values: C was not produced by BTA_matrices_alloc");
    BlockView v = blocks_of(Am);
    if (P->x_total != (long long)[&]() { long long t = 0; for (size_t k = 0; k < v.m0.size(); ++k) t += (long long)v.m0[k] * v.n0[k]; return t; }())
        fail(SDL_ERR_INVALID, "BTDA_matrices_fill_values: A does not match the alloc");
    h2d(xv->get(), v.host_x, (size_t)P->x_total, s);
    if (d) h2d(dv->get(), d, (size_t)P->m, s);
    const double *Bx = sparse_dev_values(as_sparse(Bm), s);
    blocks_btda_fill(*P, xv->get(), d ? dv->get() : nullptr, Bx, cv->get(), s);
    d2h(hc, cv->get(), (size_t)P->c_total, s);
    SDL_CUDA(cudaStreamSynchronize(s));
    matrix_values_changed(Cm);
}
// BA with B permuted_dense and A sparse (upstream matmul_dispatchers.c:197-223 ->
// permuted_dense_linalg.c:313-430 BA_pd_csr_*): C is permuted_dense with B's
// row_perm and the columns of S = A's CSR that B's col_perm rows reach.
matrix *dense_BA_alloc(const matrix *Bm, matrix *Am)
{
    if (Bm->kind != MATRIX_PERMUTED_DENSE || Am->kind != MATRIX_SPARSE) return prog_BA_alloc(Bm, Am);
    const permuted_dense *B = as_pd(Bm);
    sdl_sparse *A = as_sparse(Am);
    cudaStream_t s = runtime().stream;
    const int *cperm = B->col_perm;
    auto plan = blocks_csr_build(1, &B->m0, &B->n0, &cperm, A->csr->p, A->csr->i, A->csr->m, A->csr->n,
                                 true, s);
    const std::vector<int> &cpC = plan->col_perm[0];
    matrix *Cm = new_permuted_dense(B->base.m, A->csr->n, B->m0, (int)cpC.size(), B->row_perm,
                                    cpC.empty() ? nullptr : cpC.data(), nullptr);
    if (!Cm) fail(SDL_ERR_INTERNAL, "BA_matrices_alloc: output allocation failed");
    permuted_dense *C = as_pd(Cm);
    C->impl->bvals.reset((size_t)std::max<long long>(1, plan->b_total));
    C->impl->cvals.reset((size_t)std::max<long long>(1, plan->c_total));
    C->impl->ba = std::move(plan);
    sparse_dev_values(A, s); // the device mirror of A's values exists before any fill
    SDL_CUDA(cudaStreamSynchronize(s));
    return Cm;
}

void dense_BA_fill(const matrix *Bm, const matrix *Am, matrix *Cm)
{
    if (ProgState *ps = prog_state(Cm); ps && ps->op == DP_OP_BA)
    {
        prog_product_fill(Bm, nullptr, Am, Cm, DP_OP_BA);
        return;
    }
    if (Bm->kind != MATRIX_PERMUTED_DENSE || Am->kind != MATRIX_SPARSE || Cm->kind != MATRIX_PERMUTED_DENSE)
        unsupported("BA_matrices_fill_values");
    const permuted_dense *B = as_pd(Bm);
    permuted_dense *C = as_pd(Cm);
    PdImpl *im = C->impl;
    if (!im || !im->ba) fail(SDL_ERR_INVALID, "BA_matrices_fill_values: C was not produced by BA_matrices_alloc");
    const BlocksCsrPlan &P = *im->ba;
    if (P.b_total != (long long)B->m0 * B->n0 || P.S_nnz != as_sparse(Am)->csr->nnz)
        fail(SDL_ERR_INVALID, "BA_matrices_fill_values: operands do not match the alloc");
    cudaStream_t s = runtime().stream;
    h2d(im->bvals.get(), B->X, (size_t)P.b_total, s);
    const double *Sx = sparse_dev_values(as_sparse(Am), s);
    blocks_csr_fill(P, im->bvals.get(), Sx, im->cvals.get(), s);
    d2h(C->X, im->cvals.get(), (size_t)P.c_total, s);
    SDL_CUDA(cudaStreamSynchronize(s));
    matrix_values_changed(Cm);
}
// ATA with A permuted_dense or stacked_pd (upstream matmul_dispatchers.c:490-527 ->
// ATA_pd_* / ATA_spd_*): the partials on the FP64 tensor cores, coalesced as upstream.
matrix *dense_ATA_alloc(matrix *Am)
{
    cudaStream_t s = runtime().stream;
    if (Am->kind == MATRIX_PERMUTED_DENSE)
    {
        const permuted_dense *A = as_pd(Am);
        const int *rp = A->row_perm, *cp = A->col_perm;
        auto plan = blocks_ata_build(1, &A->m0, &A->n0, &rp, &cp, A->base.m, A->base.n, s);
        // one block: C = n0 x n0 at col_perm x col_perm (upstream permuted_dense_linalg.c:87-99)
        matrix *Cm = new_permuted_dense(A->base.n, A->base.n, A->n0, A->n0, A->col_perm, A->col_perm, nullptr);
        if (!Cm) fail(SDL_ERR_INTERNAL, "ATA_matrices_alloc: output allocation failed");
        permuted_dense *C = as_pd(Cm);
        C->impl->bvals.reset((size_t)std::max<long long>(1, plan->x_total));
        C->impl->cvals.reset((size_t)std::max<long long>(1, plan->c_total));
        C->impl->dvec.reset((size_t)std::max(1, A->base.m));
        C->impl->ata = std::move(plan);
        return Cm;
    }
    if (Am->kind != MATRIX_STACKED_PD) unsupported("ATA_matrices_alloc");
    const sdl_stacked *A = as_spd(Am);
    std::vector<int> m0(std::max(1, A->n_blocks)), n0(std::max(1, A->n_blocks));
    std::vector<const int *> rp(std::max(1, A->n_blocks)), cp(std::max(1, A->n_blocks));
    for (int k = 0; k < A->n_blocks; ++k)
    {
        m0[k] = A->blocks[k]->m0;
        n0[k] = A->blocks[k]->n0;
        rp[k] = A->blocks[k]->row_perm;
        cp[k] = A->blocks[k]->col_perm;
    }
    auto plan = blocks_ata_build(A->n_blocks, m0.data(), n0.data(), rp.data(), cp.data(), A->base.m, A->base.n, s);
    const int nb = plan->n_out;
    permuted_dense **blocks = (permuted_dense **)sp_malloc(sizeof(permuted_dense *) * std::max(1, nb));
    std::vector<int> sp_p(1, 0), sp_i;
    for (int o = 0; o < nb; ++o)
    {
        const std::vector<int> &r = plan->out_rows[o], &c = plan->out_cols[o];
        blocks[o] = as_pd(new_permuted_dense(A->base.n, A->base.n, (int)r.size(), (int)c.size(), r.data(),
                                             c.data(), nullptr));
        if (!blocks[o]) fail(SDL_ERR_INTERNAL, "ATA_matrices_alloc: output allocation failed");
        sp_i.insert(sp_i.end(), plan->out_srcs[o].begin(), plan->out_srcs[o].end());
        sp_p.push_back((int)sp_i.size());
    }
    if (sp_i.empty()) sp_i.push_back(0);
    matrix *Cm = new_stacked_pd(A->base.n, A->base.n, nb, blocks, sp_p.data(), sp_i.data());
    sp_free(blocks);
    if (!Cm) fail(SDL_ERR_INTERNAL, "ATA_matrices_alloc: output allocation failed");
    sdl_stacked *C = as_spd(Cm);
    C->impl->xvals.reset((size_t)std::max<long long>(1, plan->x_total));
    C->impl->cvals.reset((size_t)std::max<long long>(1, plan->c_total));
    C->impl->dvec.reset((size_t)std::max(1, A->base.m));
    C->impl->ata = std::move(plan);
    return Cm;
}

void dense_ATDA_fill(const matrix *Am, const double *d, matrix *Cm)
{
    cudaStream_t s = runtime().stream;
    const BlocksAtaPlan *P = nullptr;
    DevBuf<double> *xv = nullptr, *cv = nullptr, *dv = nullptr;
    const double *hx = nullptr;
    double *hc = nullptr;
    if (Am->kind == MATRIX_PERMUTED_DENSE && Cm->kind == MATRIX_PERMUTED_DENSE)
    {
        permuted_dense *C = as_pd(Cm);
        if (!C->impl || !C->impl->ata || C->impl->ata->btda)
            fail(SDL_ERR_INVALID, "ATDA_matrices_fill_values: C was not produced by ATA_matrices_alloc");
        P = C->impl->ata.get();
        xv = &C->impl->bvals;
        cv = &C->impl->cvals;
        dv = &C->impl->dvec;
        hx = as_pd(Am)->X;
        hc = C->X;
    }
    else if (Am->kind == MATRIX_STACKED_PD && Cm->kind == MATRIX_STACKED_PD)
    {
        sdl_stacked *C = as_spd(Cm);
        if (!C->impl || !C->impl->ata || C->impl->ata->btda)
            fail(SDL_ERR_INVALID, "ATDA_matrices_fill_values: C was not produced by ATA_matrices_alloc");
        P = C->impl->ata.get();
        xv = &C->impl->xvals;
        cv = &C->impl->cvals;
        dv = &C->impl->dvec;
        hx = as_spd(Am)->values;
        hc = C->values;
    }
    else
        unsupported("ATDA_matrices_fill_values");
    h2d(xv->get(), hx, (size_t)P->x_total, s);
    if (d) h2d(dv->get(), d, (size_t)P->m, s);
    blocks_ata_fill(*P, xv->get(), d ? dv->get() : nullptr, cv->get(), s);
    d2h(hc, cv->get(), (size_t)P->c_total, s);
    SDL_CUDA(cudaStreamSynchronize(s));
    matrix_values_changed(Cm);
}
void dense_DA_fill(const double *d, const matrix *A, matrix *C) { prog_DA_fill(d, A, C); }
matrix *dense_transpose_alloc(const matrix *A) { return prog_transpose_alloc(A); }
void dense_transpose_fill(const matrix *A, matrix *AT) { prog_transpose_fill(A, AT); }

} // namespace sdl

using namespace sdl;

extern "C" matrix *new_permuted_dense(int m, int n, int m0, int n0, const int *row_perm,
                                      const int *col_perm, const double *X_data)
{
    return guard_upstream<matrix *>("new_permuted_dense", nullptr, [&]() -> matrix * {
        if (m < 0 || n < 0 || m0 < 0 || n0 < 0 || m0 > m || n0 > n)
            fail(SDL_ERR_INVALID, "bad block shape");
        for (int ii = 1; ii < m0; ++ii)
            if (row_perm[ii] <= row_perm[ii - 1]) fail(SDL_ERR_INVALID, "row_perm must be strictly increasing");
        for (int jj = 1; jj < n0; ++jj)
            if (col_perm[jj] <= col_perm[jj - 1]) fail(SDL_ERR_INVALID, "col_perm must be strictly increasing");
        if (m0 > 0 && (row_perm[0] < 0 || row_perm[m0 - 1] >= m)) fail(SDL_ERR_INVALID, "row_perm out of range");
        if (n0 > 0 && (col_perm[0] < 0 || col_perm[n0 - 1] >= n)) fail(SDL_ERR_INVALID, "col_perm out of range");
        if (m0 > 0 && n0 > INT_MAX / m0)
            fail(SDL_ERR_OVERFLOW, "dense block m0 * n0 exceeds INT_MAX"); // upstream permuted_dense.c:258-262
        permuted_dense *pd = (permuted_dense *)sp_calloc(1, sizeof(permuted_dense));
        pd->base.m = m;
        pd->base.n = n;
        pd->base.nnz = m0 * n0;
        pd->m0 = m0;
        pd->n0 = n0;
        pd->row_perm = (int *)sp_malloc(sizeof(int) * std::max(1, m0));
        pd->col_perm = (int *)sp_malloc(sizeof(int) * std::max(1, n0));
        pd->row_inv = (int *)sp_malloc(sizeof(int) * std::max(1, m));
        pd->col_inv = (int *)sp_malloc(sizeof(int) * std::max(1, n));
        pd->X = (double *)sp_malloc(sizeof(double) * std::max(1, m0 * n0));
        pd->owns_X = true;
        pd->base.x = pd->X;
        if (m0) std::memcpy(pd->row_perm, row_perm, sizeof(int) * m0);
        if (n0) std::memcpy(pd->col_perm, col_perm, sizeof(int) * n0);
        for (int i = 0; i < m; ++i) pd->row_inv[i] = -1;
        for (int j = 0; j < n; ++j) pd->col_inv[j] = -1;
        for (int ii = 0; ii < m0; ++ii) pd->row_inv[row_perm[ii]] = ii;
        for (int jj = 0; jj < n0; ++jj) pd->col_inv[col_perm[jj]] = jj;
        if (X_data && m0 * n0) std::memcpy(pd->X, X_data, sizeof(double) * m0 * n0);
        pd->impl = new PdImpl();
        wire_pd(pd);
        return &pd->base;
    });
}

extern "C" matrix *new_permuted_dense_full(int m, int n, const double *data)
{
    std::vector<int> rp(std::max(1, m)), cp(std::max(1, n));
    for (int i = 0; i < m; ++i) rp[i] = i;
    for (int j = 0; j < n; ++j) cp[j] = j;
    return new_permuted_dense(m, n, m, n, rp.data(), cp.data(), data);
}

extern "C" matrix *new_stacked_pd(int m, int n, int n_blocks, permuted_dense **blocks,
                                  const int *src_block_idx_p, const int *src_block_idx)
{
    return guard_upstream<matrix *>("new_stacked_pd", nullptr, [&]() -> matrix * {
        if ((src_block_idx_p == nullptr) != (src_block_idx == nullptr))
            fail(SDL_ERR_INVALID, "src_block_idx_p and src_block_idx must both be set or both NULL");
        sdl_stacked *spd = (sdl_stacked *)sp_calloc(1, sizeof(sdl_stacked));
        spd->base.m = m;
        spd->base.n = n;
        long long nnz = 0;
        for (int k = 0; k < n_blocks; ++k) nnz += blocks[k]->base.nnz;
        if (nnz > INT_MAX) fail(SDL_ERR_OVERFLOW, "stacked_pd nnz exceeds INT_MAX");
        spd->base.nnz = (int)nnz;
        spd->n_blocks = n_blocks;
        spd->blocks = (permuted_dense **)sp_malloc(sizeof(permuted_dense *) * std::max(1, n_blocks));
        if (n_blocks) std::memcpy(spd->blocks, blocks, sizeof(permuted_dense *) * n_blocks);
        spd->src_block_idx_p = (int *)sp_malloc(sizeof(int) * (n_blocks + 1));
        spd->src_block_idx_p[0] = 0;
        if (!src_block_idx_p)
        {
            spd->src_block_idx = (int *)sp_malloc(sizeof(int) * std::max(1, n_blocks));
            for (int k = 0; k < n_blocks; ++k)
            {
                spd->src_block_idx_p[k + 1] = k + 1;
                spd->src_block_idx[k] = k;
            }
        }
        else
        {
            int total = src_block_idx_p[n_blocks];
            std::memcpy(spd->src_block_idx_p, src_block_idx_p, sizeof(int) * (n_blocks + 1));
            spd->src_block_idx = (int *)sp_malloc(sizeof(int) * std::max(1, total));
            if (total) std::memcpy(spd->src_block_idx, src_block_idx, sizeof(int) * total);
        }
        // one shared block-major value buffer (upstream stacked_pd.c:303-319)
        spd->values = (double *)sp_malloc(sizeof(double) * std::max<long long>(1, nnz));
        spd->base.x = spd->values;
        long long off = 0;
        for (int k = 0; k < n_blocks; ++k)
        {
            permuted_dense *b = spd->blocks[k];
            int bn = b->base.nnz;
            if (bn == 0) continue;
            std::memcpy(spd->values + off, b->X, sizeof(double) * bn);
            if (b->owns_X) sp_free(b->X);
            b->X = spd->values + off;
            b->base.x = b->X;
            b->owns_X = false;
            off += bn;
        }
        spd->impl = new SpdImpl();
        wire_spd(spd);
        return &spd->base;
    });
}

// ------------------------------------------------------------------ device API
struct sdl_blocks_csr
{
    std::unique_ptr<sdl::BlocksCsrPlan> P;
};

extern "C" sdl_status sdl_blocks_csr_create(int n_blocks, const int *m0, const int *n0,
                                            const int *const *col_perm, const int *Sp, const int *Si,
                                            int S_m, int S_n, int keep_empty, void *stream,
                                            sdl_blocks_csr **out)
{
    return guard_status("sdl_blocks_csr_create", [&]() {
        if (!out || (n_blocks > 0 && (!m0 || !n0 || !col_perm)) || (S_m > 0 && (!Sp || !Si)))
            fail(SDL_ERR_INVALID, "NULL argument");
        *out = nullptr;
        auto h = std::make_unique<sdl_blocks_csr>();
        h->P = blocks_csr_build(n_blocks, m0, n0, col_perm, Sp, Si, S_m, S_n, keep_empty != 0,
                                pick_stream(stream));
        *out = h.release();
    });
}

extern "C" sdl_status sdl_blocks_csr_info(const sdl_blocks_csr *P, int *out_blocks, long long *c_values,
                                          long long *b_values)
{
    return guard_status("sdl_blocks_csr_info", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL plan");
        if (out_blocks) *out_blocks = (int)P->P->src.size();
        if (c_values) *c_values = P->P->c_total;
        if (b_values) *b_values = P->P->b_total;
    });
}

extern "C" sdl_status sdl_blocks_csr_block(const sdl_blocks_csr *P, int k, int *src_block, int *m0,
                                           int *n0_C, const int **col_perm)
{
    return guard_status("sdl_blocks_csr_block", [&]() {
        if (!P || k < 0 || k >= (int)P->P->src.size()) fail(SDL_ERR_INVALID, "bad output block");
        if (src_block) *src_block = P->P->src[k];
        if (m0) *m0 = P->P->m0[k];
        if (n0_C) *n0_C = P->P->n0_C[k];
        if (col_perm) *col_perm = P->P->col_perm[k].data();
    });
}

extern "C" sdl_status sdl_blocks_csr_fill(const sdl_blocks_csr *P, const double *B_vals, const double *S_x,
                                          double *C_vals, void *stream)
{
    return guard_status("sdl_blocks_csr_fill", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL plan");
        if (P->P->c_total > 0 && (!B_vals || !S_x || !C_vals)) fail(SDL_ERR_INVALID, "NULL value pointer");
        blocks_csr_fill(*P->P, B_vals, S_x, C_vals, pick_stream(stream));
    });
}

extern "C" void sdl_blocks_csr_destroy(sdl_blocks_csr *P) { delete P; }

struct sdl_blocks_ata
{
    std::unique_ptr<sdl::BlocksAtaPlan> P;
};

extern "C" sdl_status sdl_blocks_ata_create(int n_blocks, const int *m0, const int *n0,
                                            const int *const *row_perm, const int *const *col_perm, int m,
                                            int n, void *stream, sdl_blocks_ata **out)
{
    return guard_status("sdl_blocks_ata_create", [&]() {
        if (!out || (n_blocks > 0 && (!m0 || !n0 || !row_perm || !col_perm))) fail(SDL_ERR_INVALID, "NULL argument");
        *out = nullptr;
        auto h = std::make_unique<sdl_blocks_ata>();
        h->P = blocks_ata_build(n_blocks, m0, n0, row_perm, col_perm, m, n, pick_stream(stream));
        *out = h.release();
    });
}

extern "C" sdl_status sdl_blocks_ata_info(const sdl_blocks_ata *P, int *out_blocks, long long *c_values,
                                          long long *x_values)
{
    return guard_status("sdl_blocks_ata_info", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL plan");
        if (out_blocks) *out_blocks = P->P->n_out;
        if (c_values) *c_values = P->P->c_total;
        if (x_values) *x_values = P->P->x_total;
    });
}

extern "C" sdl_status sdl_blocks_ata_block(const sdl_blocks_ata *P, int k, int *m0, int *n0, const int **rows,
                                           const int **cols)
{
    return guard_status("sdl_blocks_ata_block", [&]() {
        if (!P || k < 0 || k >= P->P->n_out) fail(SDL_ERR_INVALID, "bad output block");
        if (m0) *m0 = (int)P->P->out_rows[k].size();
        if (n0) *n0 = (int)P->P->out_cols[k].size();
        if (rows) *rows = P->P->out_rows[k].data();
        if (cols) *cols = P->P->out_cols[k].data();
    });
}

extern "C" sdl_status sdl_blocks_ata_fill(const sdl_blocks_ata *P, const double *X_vals, const double *d,
                                          double *C_vals, void *stream)
{
    return guard_status("sdl_blocks_ata_fill", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL plan");
        if (P->P->c_total > 0 && (!X_vals || !C_vals)) fail(SDL_ERR_INVALID, "NULL value pointer");
        blocks_ata_fill(*P->P, X_vals, d, C_vals, pick_stream(stream));
    });
}

extern "C" void sdl_blocks_ata_destroy(sdl_blocks_ata *P) { delete P; }
