// The permuted_dense / stacked_pd operations whose fills run a DenseProg
// (dense_prog.h): B^T diag(d) A and B A for the dense-block operand pairs not
// served by a dedicated plan, DA, transpose, row_gather and row_reduce. Each alloc
// reproduces upstream's output structure exactly and compiles the fill program;
// each fill uploads the operands' values, runs the program and reads C back.
//
// Upstream structure followed (src/ paths of the upstream project):
//   BTA_pd_pd_*      permuted_dense/permuted_dense_linalg.c:118-247
//   BA_pd_pd_*       permuted_dense_linalg.c:458-540
//   BTA_pd_csc_*     permuted_dense_linalg.c:542-641   (B pd, A sparse)
//   BTA_csc_pd_*     permuted_dense_linalg.c:646-741   (BA with B sparse, A pd)
//   BTA_pd_spd_*     stacked_pd/stacked_pd_linalg.c:250-428, BA_pd_spd_* :627-650
//   BTA_spd_{pd,csc,spd}_*, BTA_csc_spd_*  stacked_pd_linalg.c:431-620 (blockwise
//                    partials + stacked_pd_coalesce.c accumulate)
//   DA / transpose   permuted_dense_linalg.c:30-85, stacked_pd_linalg.c:34-115
//   row_gather / row_reduce  permuted_dense/permuted_dense.c:72-222,
//                    stacked_pd/stacked_pd.c:88-200, stacked_pd_linalg.c:160-195
// Values: row copies, scalings, transposes and sparse x dense sums are
// bit-identical to upstream (same products, same order, from +0.0); the dense x
// dense products run on the FP64 tensor cores where upstream calls cblas_dgemm,
// whose order is unspecified, so those agree within rounding.
#include <algorithm>
#include <climits>
#include <cstring>

#include "capi_common.h"
#include "dense_impl.h"
#include "sparsediff_linalg/matrix.h"
#include "sparsediff_linalg/tracked_alloc.h"

namespace sdl {

const double *sparse_dev_values(sdl_sparse *A, cudaStream_t s);

namespace {

// One dense block with the offset of its values in its kind's value array.
struct Blk
{
    int m0, n0;
    const int *rp, *cp, *row_inv;
    long long off;
};

// The dense blocks of a permuted_dense (one block) or a stacked_pd.
struct Blocks
{
    int m = 0, n = 0;
    long long nnz = 0;
    std::vector<Blk> b;
    const double *host = nullptr; // value array (X / values)
};

Blocks view(const matrix *M)
{
    Blocks v;
    v.m = M->m;
    v.n = M->n;
    if (M->kind == MATRIX_PERMUTED_DENSE)
    {
        const permuted_dense *A = as_pd(M);
        v.b.push_back(Blk{A->m0, A->n0, A->row_perm, A->col_perm, A->row_inv, 0});
        v.nnz = (long long)A->m0 * A->n0;
        v.host = A->X;
        return v;
    }
    const sdl_stacked *A = as_spd(M);
    for (int k = 0; k < A->n_blocks; ++k)
    {
        const permuted_dense *p = A->blocks[k];
        v.b.push_back(Blk{p->m0, p->n0, p->row_perm, p->col_perm, p->row_inv, v.nnz});
        v.nnz += (long long)p->m0 * p->n0;
    }
    v.host = A->values;
    return v;
}

bool dense_kind(const matrix *M) { return M->kind == MATRIX_PERMUTED_DENSE || M->kind == MATRIX_STACKED_PD; }

// Positions of the common values of two ascending arrays (upstream
// sorted_intersect_indices, src/support/utils.c:57-84).
int intersect(const int *a, int na, const int *b, int nb, std::vector<int> &ia, std::vector<int> &ib)
{
    ia.clear();
    ib.clear();
    int i = 0, j = 0;
    while (i < na && j < nb)
    {
        if (a[i] < b[j])
            ++i;
        else if (a[i] > b[j])
            ++j;
        else
        {
            ia.push_back(i++);
            ib.push_back(j++);
        }
    }
    return (int)ia.size();
}

std::vector<int> sorted_union(const std::vector<const Blk *> &blks)
{
    std::vector<int> u;
    for (const Blk *k : blks) u.insert(u.end(), k->cp, k->cp + k->n0);
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    return u;
}

// CSC of a CSR structure with each entry's CSR position (rows ascending within a
// column, as upstream's counting-sort conversion leaves them).
struct Csc
{
    std::vector<int> p, row, pos;
};
Csc csc_of(const CSR_matrix *A)
{
    Csc c;
    c.p.assign((size_t)A->n + 1, 0);
    for (int q = 0; q < A->nnz; ++q) c.p[A->i[q] + 1]++;
    for (int j = 0; j < A->n; ++j) c.p[j + 1] += c.p[j];
    c.row.resize(std::max(1, A->nnz));
    c.pos.resize(std::max(1, A->nnz));
    std::vector<int> nx(c.p.begin(), c.p.end() - 1);
    for (int r = 0; r < A->m; ++r)
        for (int q = A->p[r]; q < A->p[r + 1]; ++q)
        {
            const int e = nx[A->i[q]]++;
            c.row[e] = r;
            c.pos[e] = q;
        }
    return c;
}

matrix *make_pd(int m, int n, const std::vector<int> &rows, const std::vector<int> &cols)
{
    matrix *C = new_permuted_dense(m, n, (int)rows.size(), (int)cols.size(), rows.empty() ? nullptr : rows.data(),
                                   cols.empty() ? nullptr : cols.data(), nullptr);
    if (!C) fail(SDL_ERR_INTERNAL, "dense-block output allocation failed");
    return C;
}

// A stacked_pd with the given blocks and source map (src_p / src_i, or the
// identity when src_p is empty).
matrix *make_spd(int m, int n, const std::vector<std::vector<int>> &rows, const std::vector<std::vector<int>> &cols,
                 const std::vector<int> &src_p, const std::vector<int> &src_i)
{
    const int nb = (int)rows.size();
    permuted_dense **blocks = (permuted_dense **)sp_malloc(sizeof(permuted_dense *) * std::max(1, nb));
    for (int o = 0; o < nb; ++o) blocks[o] = as_pd(make_pd(m, n, rows[o], cols[o]));
    std::vector<int> si = src_i;
    if (si.empty()) si.push_back(0);
    matrix *C = new_stacked_pd(m, n, nb, blocks, src_p.empty() ? nullptr : src_p.data(),
                               src_p.empty() ? nullptr : si.data());
    sp_free(blocks);
    if (!C) fail(SDL_ERR_INTERNAL, "dense-block output allocation failed");
    return C;
}

// The coalesced output of a program (upstream: signatures as the source map).
matrix *spd_of(int m, int n, const DenseProg &P)
{
    std::vector<int> sp(1, 0), si;
    for (const auto &s : P.out_srcs)
    {
        si.insert(si.end(), s.begin(), s.end());
        sp.push_back((int)si.size());
    }
    return make_spd(m, n, P.out_rows, P.out_cols, sp, si);
}

double *host_values(matrix *C) { return C->kind == MATRIX_PERMUTED_DENSE ? as_pd(C)->X : as_spd(C)->values; }
long long value_count(const matrix *C)
{
    return C->kind == MATRIX_PERMUTED_DENSE ? (long long)as_pd(C)->m0 * as_pd(C)->n0 : (long long)C->nnz;
}

void bind(matrix *C, int op, std::unique_ptr<DenseProg> prog)
{
    ProgState *ps = prog_state(C);
    if (!ps) fail(SDL_ERR_INTERNAL, "dense-block output without device state");
    if (prog->c_total != value_count(C)) fail(SDL_ERR_INTERNAL, "dense-block program does not match its output");
    ps->op = op;
    ps->xl.reset((size_t)std::max<long long>(1, prog->nl));
    ps->xr.reset((size_t)std::max<long long>(1, prog->nr));
    ps->dv.reset((size_t)std::max(1, prog->d_len));
    ps->cv.reset((size_t)std::max<long long>(1, prog->c_total));
    ps->prog = std::move(prog);
}

// Run the program bound to C; XL / XR host values (or null), Sx device values.
void run(matrix *C, int op, const double *hXL, long long nl, const double *hXR, long long nr, const double *Sx,
         int ns, const double *d, const char *what)
{
    ProgState *ps = prog_state(C);
    if (!ps || ps->op != op || !ps->prog) fail(SDL_ERR_INVALID, std::string(what) + ": C was not allocated for this operation");
    DenseProg &P = *ps->prog;
    if (nl != P.nl || nr != P.nr || ns != P.ns) fail(SDL_ERR_INVALID, std::string(what) + ": operands do not match the alloc");
    if (d && P.d_len == 0) d = nullptr; // a product over zero rows reads no d
    cudaStream_t s = runtime().stream;
    if (nl) h2d(ps->xl.get(), hXL, (size_t)nl, s);
    if (nr) h2d(ps->xr.get(), hXR, (size_t)nr, s);
    if (d) h2d(ps->dv.get(), d, (size_t)P.d_len, s);
    dp_fill(P, ps->xl.get(), ps->xr.get(), Sx, d ? ps->dv.get() : nullptr, ps->cv.get(), s);
    if (P.c_total) d2h(host_values(C), ps->cv.get(), (size_t)P.c_total, s);
    SDL_CUDA(cudaStreamSynchronize(s));
    matrix_values_changed(C);
}

// ------------------------------------------------------------------ products
enum AKind
{
    A_PD,
    A_SPD,
    A_SPARSE
};

int kind_of(const matrix *M)
{
    return M->kind == MATRIX_PERMUTED_DENSE ? A_PD : M->kind == MATRIX_STACKED_PD ? A_SPD : A_SPARSE;
}

std::vector<int> rows_at(const int *rp, const std::vector<int> &idx)
{
    std::vector<int> r(idx.size());
    for (size_t t = 0; t < idx.size(); ++t) r[t] = rp[idx[t]];
    return r;
}

// Entries of a sparse operand grouped by the dense block that owns their dense
// index: per block, (outer, dense-block row, position in the CSR values, global
// row) in traversal order.
using EntLists = std::vector<std::vector<int4>>;

// Row -> owning block (a stacked_pd's blocks own disjoint rows).
std::vector<int> row_blocks(const Blocks &V, int m)
{
    std::vector<int> rb(std::max(1, m), -1);
    for (size_t k = 0; k < V.b.size(); ++k)
        for (int ii = 0; ii < V.b[k].m0; ++ii)
        {
            const int r = V.b[k].rp[ii];
            if (r < 0 || r >= m) fail(SDL_ERR_INVALID, "dense block row outside the matrix");
            if (rb[r] >= 0) fail(SDL_ERR_INVALID, "stacked_pd blocks share a row");
            rb[r] = (int)k;
        }
    return rb;
}

// A sparse A read by columns (its CSC), for B^T A with B dense: outer = column of A.
EntLists entries_by_csc(const Blocks &B, const CSR_matrix *A)
{
    const std::vector<int> rb = row_blocks(B, A->m);
    const Csc c = csc_of(A);
    EntLists L(B.b.size());
    for (int j = 0; j < A->n; ++j)
        for (int e = c.p[j]; e < c.p[j + 1]; ++e)
        {
            const int k = rb[c.row[e]];
            if (k >= 0) L[k].push_back(make_int4(j, B.b[k].row_inv[c.row[e]], c.pos[e], c.row[e]));
        }
    return L;
}

// A sparse B read by rows (the CSC of B^T), for B A with A dense: outer = row of B.
EntLists entries_by_csr(const CSR_matrix *B, const Blocks &A)
{
    const std::vector<int> rb = row_blocks(A, B->n);
    EntLists L(A.b.size());
    for (int i = 0; i < B->m; ++i)
        for (int q = B->p[i]; q < B->p[i + 1]; ++q)
        {
            const int col = B->i[q];
            if (col < 0 || col >= B->n) fail(SDL_ERR_INVALID, "column index outside the matrix");
            const int k = rb[col];
            if (k >= 0) L[k].push_back(make_int4(i, A.b[k].row_inv[col], q, col));
        }
    return L;
}

// One vector task per distinct outer index of a block's entry list; returns the
// outer indices. Vector a of the partial at p: p + a * astride, elements t * stride.
std::vector<int> sparse_vectors(DpBuilder &b, const std::vector<int4> &ent, long long p, long long astride,
                                int nvec, int stride, const Blk &X, bool dense_right, int mode)
{
    std::vector<int> outer, kk, pos, row;
    size_t e = 0;
    while (e < ent.size())
    {
        const int o = ent[e].x;
        kk.clear();
        pos.clear();
        row.clear();
        for (; e < ent.size() && ent[e].x == o; ++e)
        {
            kk.push_back(ent[e].y);
            pos.push_back(ent[e].z);
            row.push_back(ent[e].w);
        }
        b.spvec(p + (long long)outer.size() * astride, nvec, stride, X.off, X.n0, dense_right, mode, kk, pos, row);
        outer.push_back(o);
    }
    return outer;
}

int distinct_outer(const std::vector<int4> &ent)
{
    int n = 0;
    for (size_t e = 0; e < ent.size(); ++e)
        if (e == 0 || ent[e].x != ent[e - 1].x) ++n;
    return n;
}

// Partial of Bk^T diag(d) A for one dense block Bk of the left operand (upstream
// BTA_pd_pd_alloc, BTA_pd_spd_alloc, BTA_pd_csc_alloc). An upstream 0 x 0 partial
// (BTA_pd_pd without common rows) has no rows here.
DpPart bta_partial(DpBuilder &b, const Blk &Bk, int akind, const Blocks *A, const std::vector<int4> *ent)
{
    DpPart part;
    std::vector<int> ib, ia;
    if (akind == A_PD)
    {
        const Blk &Ak = A->b[0];
        if (!intersect(Bk.rp, Bk.m0, Ak.rp, Ak.m0, ib, ia)) return part;
        part.rows.assign(Bk.cp, Bk.cp + Bk.n0);
        part.cols.assign(Ak.cp, Ak.cp + Ak.n0);
        const long long p = b.alloc((long long)Bk.n0 * Ak.n0);
        b.gemm(p, Bk.n0, Ak.n0, Bk.off, Bk.n0, true, ib, Ak.off, Ak.n0, ia, rows_at(Ak.rp, ia));
        part.vals.push_back(DpPart::Val{part.cols, p, Ak.n0, 1});
        return part;
    }
    part.rows.assign(Bk.cp, Bk.cp + Bk.n0);
    if (akind == A_SPD)
    {
        std::vector<const Blk *> contrib;
        for (const Blk &Ak : A->b)
            if (intersect(Bk.rp, Bk.m0, Ak.rp, Ak.m0, ib, ia)) contrib.push_back(&Ak);
        part.cols = sorted_union(contrib);
        for (const Blk *Ak : contrib)
        {
            intersect(Bk.rp, Bk.m0, Ak->rp, Ak->m0, ib, ia);
            const long long p = b.alloc((long long)Bk.n0 * Ak->n0);
            b.gemm(p, Bk.n0, Ak->n0, Bk.off, Bk.n0, true, ib, Ak->off, Ak->n0, ia, rows_at(Ak->rp, ia));
            part.vals.push_back(DpPart::Val{std::vector<int>(Ak->cp, Ak->cp + Ak->n0), p, Ak->n0, 1});
        }
        return part;
    }
    // A sparse: column j of C is sum over A's column j of (d[k] A[k, j]) * row kk of Bk
    const int nact = distinct_outer(*ent);
    const long long p = b.alloc((long long)Bk.n0 * nact);
    part.cols = sparse_vectors(b, *ent, p, 1, Bk.n0, nact, Bk, false, DP_SP_D_SPARSE);
    if (nact) part.vals.push_back(DpPart::Val{part.cols, p, nact, 1});
    return part;
}

// Partial of B Ak for B sparse and one dense block Ak of A (upstream
// BTA_csc_pd_alloc on the CSC view of B^T): rows = rows of B reaching Ak's rows.
DpPart ba_sparse_partial(DpBuilder &b, const Blk &Ak, const std::vector<int4> &ent)
{
    DpPart part;
    const int nact = distinct_outer(ent);
    const long long p = b.alloc((long long)nact * Ak.n0);
    part.rows = sparse_vectors(b, ent, p, Ak.n0, Ak.n0, 1, Ak, true, DP_SP_D_DENSE);
    part.cols.assign(Ak.cp, Ak.cp + Ak.n0);
    if (nact) part.vals.push_back(DpPart::Val{part.cols, p, Ak.n0, 1});
    return part;
}

// True when the part is one value source laid out as the output itself.
bool is_direct(const DpBuilder &b, const DpPart &part)
{
    if (part.vals.empty()) return b.p_total == 0;
    const DpPart::Val &v = part.vals[0];
    return part.vals.size() == 1 && v.p == 0 && v.cs == 1 && v.rs == (int)part.cols.size() &&
           v.cols == part.cols && b.p_total == (long long)part.rows.size() * part.cols.size();
}

long long nnz_of(const matrix *M) { return M->kind == MATRIX_SPARSE ? as_sparse(M)->csr->nnz : view(M).nnz; }

} // namespace

matrix *prog_BTA_alloc(matrix *Am, matrix *Bm)
{
    if (!dense_kind(Bm)) fail(SDL_ERR_INTERNAL, "prog_BTA_alloc: B must be a dense-block kind");
    if (Am->m != Bm->m) fail(SDL_ERR_INVALID, "BTA_matrices_alloc: B and A have different row counts");
    cudaStream_t s = runtime().stream;
    const Blocks B = view(Bm);
    const int akind = kind_of(Am);
    Blocks A;
    EntLists ent;
    if (akind == A_SPARSE)
        ent = entries_by_csc(B, as_sparse(Am)->csr);
    else
        A = view(Am);
    DpBuilder b;
    std::unique_ptr<DenseProg> prog;
    matrix *C = nullptr;
    if (Bm->kind == MATRIX_PERMUTED_DENSE)
    {
        // upstream BTA_pd_pd / BTA_pd_spd / BTA_pd_csc: one permuted_dense
        DpPart part = bta_partial(b, B.b[0], akind, &A, akind == A_SPARSE ? &ent[0] : nullptr);
        prog = (akind != A_SPD && is_direct(b, part))
                   ? dp_direct(b, (long long)part.rows.size() * part.cols.size(), s)
                   : dp_single(b, part.rows, part.cols, {part}, s);
        C = make_pd(Bm->n, Am->n, part.rows, part.cols);
    }
    else
    {
        // upstream BTA_spd_*: blockwise partials, coalesced with accumulation
        std::vector<DpPart> parts;
        for (size_t k = 0; k < B.b.size(); ++k)
            parts.push_back(bta_partial(b, B.b[k], akind, &A, akind == A_SPARSE ? &ent[k] : nullptr));
        prog = dp_coalesced(b, parts, Bm->n, Am->n, true, s);
        C = spd_of(Bm->n, Am->n, *prog);
    }
    try
    {
        dp_finish(*prog, b, B.nnz, akind == A_SPARSE ? 0 : A.nnz, akind == A_SPARSE ? as_sparse(Am)->csr->nnz : 0,
                  Am->m, s);
        bind(C, DP_OP_BTA, std::move(prog));
    }
    catch (...)
    {
        free_matrix(C);
        throw;
    }
    return C;
}

matrix *prog_BA_alloc(const matrix *Bm, matrix *Am)
{
    if (Bm->kind == MATRIX_STACKED_PD || !dense_kind(Am))
        fail(SDL_ERR_INTERNAL, "prog_BA_alloc: unsupported operand kinds");
    if (Bm->n != Am->m) fail(SDL_ERR_INVALID, "BA_matrices_alloc: inner dimensions differ");
    cudaStream_t s = runtime().stream;
    const Blocks A = view(Am);
    DpBuilder b;
    std::unique_ptr<DenseProg> prog;
    matrix *C = nullptr;
    long long nl = 0;
    int ns = 0;
    if (Bm->kind == MATRIX_PERMUTED_DENSE)
    {
        const Blocks B = view(Bm);
        const Blk &Bk = B.b[0];
        nl = B.nnz;
        std::vector<int> ib, ia;
        if (Am->kind == MATRIX_PERMUTED_DENSE)
        {
            // upstream BA_pd_pd: B[:, common] A[common, :]
            const Blk &Ak = A.b[0];
            if (!intersect(Bk.cp, Bk.n0, Ak.rp, Ak.m0, ib, ia))
                C = make_pd(Bm->m, Am->n, {}, {});
            else
            {
                C = make_pd(Bm->m, Am->n, std::vector<int>(Bk.rp, Bk.rp + Bk.m0),
                            std::vector<int>(Ak.cp, Ak.cp + Ak.n0));
                const long long p = b.alloc((long long)Bk.m0 * Ak.n0);
                b.gemm(p, Bk.m0, Ak.n0, Bk.off, Bk.n0, false, ib, Ak.off, Ak.n0, ia, rows_at(Ak.rp, ia));
            }
            prog = dp_direct(b, b.p_total, s);
        }
        else
        {
            // upstream BA_pd_spd = BTA_pd_spd(B^T, A)
            DpPart part;
            part.rows.assign(Bk.rp, Bk.rp + Bk.m0);
            std::vector<const Blk *> contrib;
            for (const Blk &Ak : A.b)
                if (intersect(Bk.cp, Bk.n0, Ak.rp, Ak.m0, ib, ia)) contrib.push_back(&Ak);
            part.cols = sorted_union(contrib);
            for (const Blk *Ak : contrib)
            {
                intersect(Bk.cp, Bk.n0, Ak->rp, Ak->m0, ib, ia);
                const long long p = b.alloc((long long)Bk.m0 * Ak->n0);
                b.gemm(p, Bk.m0, Ak->n0, Bk.off, Bk.n0, false, ib, Ak->off, Ak->n0, ia, rows_at(Ak->rp, ia));
                part.vals.push_back(DpPart::Val{std::vector<int>(Ak->cp, Ak->cp + Ak->n0), p, Ak->n0, 1});
            }
            prog = dp_single(b, part.rows, part.cols, {part}, s);
            C = make_pd(Bm->m, Am->n, part.rows, part.cols);
        }
    }
    else
    {
        // B sparse: upstream BTA_csc_pd / BTA_csc_spd on the CSC view of B^T
        const CSR_matrix *Bc = as_sparse(Bm)->csr;
        ns = Bc->nnz;
        const EntLists ent = entries_by_csr(Bc, A);
        if (Am->kind == MATRIX_PERMUTED_DENSE)
        {
            DpPart part = ba_sparse_partial(b, A.b[0], ent[0]);
            prog = dp_direct(b, (long long)part.rows.size() * part.cols.size(), s);
            C = make_pd(Bm->m, Am->n, part.rows, part.cols);
        }
        else
        {
            std::vector<DpPart> parts;
            for (size_t k = 0; k < A.b.size(); ++k) parts.push_back(ba_sparse_partial(b, A.b[k], ent[k]));
            prog = dp_coalesced(b, parts, Bm->m, Am->n, true, s);
            C = spd_of(Bm->m, Am->n, *prog);
        }
    }
    try
    {
        dp_finish(*prog, b, nl, A.nnz, ns, 0, s);
        bind(C, DP_OP_BA, std::move(prog));
    }
    catch (...)
    {
        free_matrix(C);
        throw;
    }
    return C;
}

void prog_product_fill(const matrix *Bm, const double *d, const matrix *Am, matrix *Cm, int op)
{
    const char *what = op == DP_OP_BTA ? (d ? "BTDA_matrices_fill_values" : "BTA_matrices_fill_values")
                                       : "BA_matrices_fill_values";
    cudaStream_t s = runtime().stream;
    const double *hl = nullptr, *hr = nullptr, *Sx = nullptr;
    long long nl = 0, nr = 0;
    int ns = 0;
    if (dense_kind(Bm))
    {
        hl = host_values(const_cast<matrix *>(Bm));
        nl = value_count(Bm);
    }
    else
    {
        Sx = sparse_dev_values(as_sparse(Bm), s);
        ns = as_sparse(Bm)->csr->nnz;
    }
    if (dense_kind(Am))
    {
        hr = host_values(const_cast<matrix *>(Am));
        nr = value_count(Am);
    }
    else
    {
        Sx = sparse_dev_values(as_sparse(Am), s);
        ns = as_sparse(Am)->csr->nnz;
    }
    run(Cm, op, hl, nl, hr, nr, Sx, ns, d, what);
}


// ------------------------------------------------------------- DA, transpose
// C = diag(d) A into C = copy_sparsity(A) (upstream DA_pd_fill_values,
// permuted_dense_linalg.c:76-85: each row of the block times d[row_perm[ii]];
// DA_spd_fill_values blockwise). The program is compiled on the first fill.
void prog_DA_fill(const double *d, const matrix *Am, matrix *Cm)
{
    if (!dense_kind(Am) || Cm->kind != Am->kind) fail(SDL_ERR_INVALID, "DA_matrices_fill_values: C must have A's kind");
    const Blocks A = view(Am);
    if (value_count(Cm) != A.nnz || Cm->m != Am->m)
        fail(SDL_ERR_INVALID, "DA_matrices_fill_values: C must come from copy_sparsity_matrices_alloc(A)");
    ProgState *ps = prog_state(Cm);
    if (ps->op != DP_OP_DA || !ps->prog || ps->prog->nl != A.nnz)
    {
        cudaStream_t s = runtime().stream;
        DpBuilder b;
        b.alloc(A.nnz);
        for (const Blk &k : A.b)
            for (int ii = 0; ii < k.m0; ++ii)
                b.row_copy(k.off + (long long)ii * k.n0, k.off + (long long)ii * k.n0, k.n0, DP_ROW_SCALE, k.rp[ii]);
        auto prog = dp_direct(b, A.nnz, s);
        dp_finish(*prog, b, A.nnz, 0, 0, Am->m, s);
        bind(Cm, DP_OP_DA, std::move(prog));
    }
    run(Cm, DP_OP_DA, A.host, A.nnz, nullptr, 0, nullptr, 0, d, "DA_matrices_fill_values");
}

// C = A^T (upstream transpose_pd_*: swapped shape and perms; transpose_spd_*:
// blockwise transposes coalesced by plain scatter, stacked_pd_linalg.c:66-115).
matrix *prog_transpose_alloc(const matrix *Am)
{
    if (!dense_kind(Am)) fail(SDL_ERR_INTERNAL, "prog_transpose_alloc: dense-block kind expected");
    cudaStream_t s = runtime().stream;
    const Blocks A = view(Am);
    DpBuilder b;
    std::unique_ptr<DenseProg> prog;
    matrix *C = nullptr;
    if (Am->kind == MATRIX_PERMUTED_DENSE)
    {
        const Blk &k = A.b[0];
        b.transpose(0, b.alloc(A.nnz), k.m0, k.n0);
        prog = dp_direct(b, A.nnz, s);
        C = make_pd(Am->n, Am->m, std::vector<int>(k.cp, k.cp + k.n0), std::vector<int>(k.rp, k.rp + k.m0));
    }
    else
    {
        std::vector<DpPart> parts;
        for (const Blk &k : A.b)
        {
            DpPart part;
            part.rows.assign(k.cp, k.cp + k.n0);
            part.cols.assign(k.rp, k.rp + k.m0);
            const long long p = b.alloc((long long)k.m0 * k.n0);
            b.transpose(k.off, p, k.m0, k.n0);
            if (k.m0 && k.n0) part.vals.push_back(DpPart::Val{part.cols, p, k.m0, 1});
            parts.push_back(std::move(part));
        }
        prog = dp_coalesced(b, parts, Am->n, Am->m, false, s);
        C = spd_of(Am->n, Am->m, *prog);
    }
    try
    {
        dp_finish(*prog, b, A.nnz, 0, 0, 0, s);
        bind(C, DP_OP_TRANSPOSE, std::move(prog));
    }
    catch (...)
    {
        free_matrix(C);
        throw;
    }
    return C;
}

void prog_transpose_fill(const matrix *Am, matrix *ATm)
{
    if (!dense_kind(Am)) fail(SDL_ERR_INVALID, "transpose_matrices_fill_values: dense-block kind expected");
    const Blocks A = view(Am);
    run(ATm, DP_OP_TRANSPOSE, A.host, A.nnz, nullptr, 0, nullptr, 0, nullptr, "transpose_matrices_fill_values");
}

// ------------------------------------------------------ row_gather / row_reduce
namespace {

void check_map(const int *map, int m_out, int m, const char *what)
{
    if (m_out < 0) fail(SDL_ERR_INVALID, std::string(what) + ": negative output size");
    if (m_out > 0 && !map) fail(SDL_ERR_INVALID, std::string(what) + ": NULL map");
    for (int i = 0; i < m_out; ++i)
        if (map[i] < 0 || map[i] >= m) fail(SDL_ERR_INVALID, std::string(what) + ": index outside the matrix");
}

matrix *finish_rows(matrix *C, std::unique_ptr<DenseProg> prog, DpBuilder &b, long long nl, int op)
{
    try
    {
        dp_finish(*prog, b, nl, 0, 0, 0, runtime().stream);
        bind(C, op, std::move(prog));
    }
    catch (...)
    {
        free_matrix(C);
        throw;
    }
    return C;
}

// Rows of block k kept by C = A[map, :] (upstream row_gather_pd_alloc,
// permuted_dense.c:72-102): output positions i whose source row is in the block,
// with the block row each copies.
void gathered_rows(const Blk &k, const int *map, int m_out, std::vector<int> &rows, std::vector<int> &src)
{
    rows.clear();
    src.clear();
    for (int i = 0; i < m_out; ++i)
    {
        const int ii = k.row_inv[map[i]];
        if (ii >= 0)
        {
            rows.push_back(i);
            src.push_back(ii);
        }
    }
}

// Groups hit by block k, ascending, and the output row of each block row
// (upstream row_reduce_pd_alloc, permuted_dense.c:152-192).
void reduced_rows(const Blk &k, const int *group, int m_out, std::vector<int> &rows, std::vector<int> &dst)
{
    std::vector<int> g2o(std::max(1, m_out), -1);
    for (int ii = 0; ii < k.m0; ++ii)
    {
        const int g = group[k.rp[ii]];
        if (g < 0 || g >= m_out) fail(SDL_ERR_INVALID, "row_reduce_alloc: group outside the output");
        g2o[g] = 0;
    }
    rows.clear();
    for (int g = 0; g < m_out; ++g)
        if (g2o[g] >= 0)
        {
            g2o[g] = (int)rows.size();
            rows.push_back(g);
        }
    dst.resize(k.m0);
    for (int ii = 0; ii < k.m0; ++ii) dst[ii] = g2o[group[k.rp[ii]]];
}

// One summing row task per output row of a reduced block at p (block rows in order).
void reduce_tasks(DpBuilder &b, const Blk &k, long long p, int nrows, const std::vector<int> &dst)
{
    std::vector<std::vector<long long>> src(nrows);
    for (int ii = 0; ii < k.m0; ++ii) src[dst[ii]].push_back(k.off + (long long)ii * k.n0);
    for (int r = 0; r < nrows; ++r) b.row_sum(p + (long long)r * k.n0, src[r], k.n0);
}

} // namespace

matrix *pd_row_gather_alloc(const matrix *self, const int *map, int m_out)
{
    return guard_upstream<matrix *>("row_gather_alloc", nullptr, [&]() -> matrix * {
        check_map(map, m_out, self->m, "row_gather_alloc");
        const Blocks A = view(self);
        const Blk &k = A.b[0];
        std::vector<int> rows, src;
        gathered_rows(k, map, m_out, rows, src);
        DpBuilder b;
        b.alloc((long long)rows.size() * k.n0);
        for (size_t r = 0; r < rows.size(); ++r) b.row_copy((long long)r * k.n0, (long long)src[r] * k.n0, k.n0);
        auto prog = dp_direct(b, b.p_total, runtime().stream);
        matrix *C = make_pd(m_out, self->n, rows, std::vector<int>(k.cp, k.cp + k.n0));
        return finish_rows(C, std::move(prog), b, A.nnz, DP_OP_GATHER);
    });
}

// upstream stacked_pd.c:167-198: per block row_gather_pd_alloc, blocks without
// values dropped (spd_map_filter_blocks), each output block's one source recorded.
matrix *spd_row_gather_alloc(const matrix *self, const int *map, int m_out)
{
    return guard_upstream<matrix *>("row_gather_alloc", nullptr, [&]() -> matrix * {
        check_map(map, m_out, self->m, "row_gather_alloc");
        const Blocks A = view(self);
        DpBuilder b;
        std::vector<std::vector<int>> orows, ocols;
        std::vector<int> sp(1, 0), si;
        std::vector<int> rows, src;
        for (size_t kk = 0; kk < A.b.size(); ++kk)
        {
            const Blk &k = A.b[kk];
            gathered_rows(k, map, m_out, rows, src);
            if ((long long)rows.size() * k.n0 == 0) continue;
            const long long p = b.alloc((long long)rows.size() * k.n0);
            for (size_t r = 0; r < rows.size(); ++r)
                b.row_copy(p + (long long)r * k.n0, k.off + (long long)src[r] * k.n0, k.n0);
            orows.push_back(rows);
            ocols.emplace_back(k.cp, k.cp + k.n0);
            si.push_back((int)kk);
            sp.push_back((int)si.size());
        }
        auto prog = dp_direct(b, b.p_total, runtime().stream);
        matrix *C = A.b.empty() ? make_spd(m_out, self->n, {}, {}, {}, {})
                                : make_spd(m_out, self->n, orows, ocols, sp, si);
        return finish_rows(C, std::move(prog), b, A.nnz, DP_OP_GATHER);
    });
}

matrix *pd_row_reduce_alloc(const matrix *self, const int *group, int m_out)
{
    return guard_upstream<matrix *>("row_reduce_alloc", nullptr, [&]() -> matrix * {
        if (m_out < 0 || (self->m > 0 && !group)) fail(SDL_ERR_INVALID, "row_reduce_alloc: bad arguments");
        const Blocks A = view(self);
        const Blk &k = A.b[0];
        std::vector<int> rows, dst;
        reduced_rows(k, group, m_out, rows, dst);
        DpBuilder b;
        const long long p = b.alloc((long long)rows.size() * k.n0);
        reduce_tasks(b, k, p, (int)rows.size(), dst);
        auto prog = dp_direct(b, b.p_total, runtime().stream);
        matrix *C = make_pd(m_out, self->n, rows, std::vector<int>(k.cp, k.cp + k.n0));
        return finish_rows(C, std::move(prog), b, A.nnz, DP_OP_REDUCE);
    });
}

// upstream stacked_pd_linalg.c:160-195: per block row_reduce_pd, then coalesced
// with accumulation.
matrix *spd_row_reduce_alloc(const matrix *self, const int *group, int m_out)
{
    return guard_upstream<matrix *>("row_reduce_alloc", nullptr, [&]() -> matrix * {
        if (m_out < 0 || (self->m > 0 && !group)) fail(SDL_ERR_INVALID, "row_reduce_alloc: bad arguments");
        const Blocks A = view(self);
        DpBuilder b;
        std::vector<DpPart> parts;
        std::vector<int> rows, dst;
        for (const Blk &k : A.b)
        {
            reduced_rows(k, group, m_out, rows, dst);
            DpPart part;
            part.rows = rows;
            part.cols.assign(k.cp, k.cp + k.n0);
            const long long p = b.alloc((long long)rows.size() * k.n0);
            reduce_tasks(b, k, p, (int)rows.size(), dst);
            if (!rows.empty() && k.n0) part.vals.push_back(DpPart::Val{part.cols, p, k.n0, 1});
            parts.push_back(std::move(part));
        }
        auto prog = dp_coalesced(b, parts, m_out, self->n, true, runtime().stream);
        matrix *C = spd_of(m_out, self->n, *prog);
        return finish_rows(C, std::move(prog), b, A.nnz, DP_OP_REDUCE);
    });
}

void dense_rows_fill(const matrix *self, matrix *out)
{
    guard_upstream_void("row_gather / row_reduce fill_values", [&]() {
        if (!self || !out) fail(SDL_ERR_INVALID, "NULL operand");
        ProgState *ps = prog_state(out);
        if (!ps || (ps->op != DP_OP_GATHER && ps->op != DP_OP_REDUCE))
            fail(SDL_ERR_INVALID, "output was not produced by row_gather_alloc / row_reduce_alloc");
        const Blocks A = view(self);
        run(out, ps->op, A.host, A.nnz, nullptr, 0, nullptr, 0, nullptr, "row fill_values");
    });
}

} // namespace sdl

namespace sdl {

// ------------------------------------------------------------------ dense kron
// C = kron(I_p, A) J or kron(A, I_p) J for a full permuted_dense A (m x n, identity
// perms) and J of any kind with J->m = p n (upstream src/stacked_pd/
// stacked_pd_kron_linalg.c:26-307, src/matmul_kron_dispatchers.c:28-123): diagonal
// block k of the Kronecker factor is A at rows k m + i, columns k n + j (or
// k + p i, k + p j); per block, upstream's BA_pd_pd (J pd), BA_pd_csr (J sparse)
// or BTA_pd_spd of its transpose (J spd); blocks without values are dropped and C's
// block q records its k.
matrix *prog_dense_kron_alloc(const matrix *Am, int p, matrix *Jm, bool a_i)
{
    if (Am->kind != MATRIX_PERMUTED_DENSE) fail(SDL_ERR_INVALID, "dense kron: A must be a full permuted_dense");
    const permuted_dense *A = as_pd(Am);
    const int m = A->m0, n = A->n0;
    if (m != Am->m || n != Am->n) fail(SDL_ERR_INVALID, "dense kron: A must be a full permuted_dense");
    for (int i = 0; i < m; ++i)
        if (A->row_perm[i] != i) fail(SDL_ERR_INVALID, "dense kron: A must be a full permuted_dense");
    for (int j = 0; j < n; ++j)
        if (A->col_perm[j] != j) fail(SDL_ERR_INVALID, "dense kron: A must be a full permuted_dense");
    if (p < 0) fail(SDL_ERR_INVALID, "dense kron: negative p");
    if ((long long)p * n != Jm->m) fail(SDL_ERR_INVALID, "dense kron: J must have p * A->n rows");
    if ((long long)p * m > INT_MAX) fail(SDL_ERR_OVERFLOW, "dense kron: p * A->m exceeds INT_MAX");
    cudaStream_t s = runtime().stream;
    const int jkind = kind_of(Jm);
    Blocks J;
    if (jkind != A_SPARSE) J = view(Jm);
    DpBuilder b;
    std::vector<DpPart> parts;
    std::vector<int> kept;
    std::vector<int> rows(m), cols(n), ib, ij;
    for (int k = 0; k < p; ++k)
    {
        for (int i = 0; i < m; ++i) rows[i] = a_i ? k + p * i : k * m + i;
        for (int j = 0; j < n; ++j) cols[j] = a_i ? k + p * j : k * n + j;
        DpPart part;
        part.rows = rows;
        if (jkind == A_PD)
        {
            const Blk &Jb = J.b[0];
            if (!m || !Jb.n0 || !intersect(cols.data(), n, Jb.rp, Jb.m0, ib, ij)) continue;
            part.cols.assign(Jb.cp, Jb.cp + Jb.n0);
            const long long q = b.alloc((long long)m * Jb.n0);
            b.gemm(q, m, Jb.n0, 0, n, false, ib, Jb.off, Jb.n0, ij, rows_at(Jb.rp, ij));
            part.vals.push_back(DpPart::Val{part.cols, q, Jb.n0, 1});
        }
        else if (jkind == A_SPD)
        {
            std::vector<const Blk *> contrib;
            for (const Blk &Jb : J.b)
                if (intersect(cols.data(), n, Jb.rp, Jb.m0, ib, ij)) contrib.push_back(&Jb);
            part.cols = sorted_union(contrib);
            if (!m || part.cols.empty()) continue;
            for (const Blk *Jb : contrib)
            {
                intersect(cols.data(), n, Jb->rp, Jb->m0, ib, ij);
                const long long q = b.alloc((long long)m * Jb->n0);
                b.gemm(q, m, Jb->n0, 0, n, false, ib, Jb->off, Jb->n0, ij, rows_at(Jb->rp, ij));
                part.vals.push_back(DpPart::Val{std::vector<int>(Jb->cp, Jb->cp + Jb->n0), q, Jb->n0, 1});
            }
        }
        else
        {
            // upstream BA_pd_csr: output columns = the union of J's rows cols[r];
            // column c sums B[i, r] * J.x over those rows in ascending r
            const CSR_matrix *S = as_sparse(Jm)->csr;
            std::vector<int4> ent; // (column, r, position, 0)
            for (int r = 0; r < n; ++r)
                for (int q = S->p[cols[r]]; q < S->p[cols[r] + 1]; ++q) ent.push_back(make_int4(S->i[q], r, q, 0));
            std::stable_sort(ent.begin(), ent.end(), [](const int4 &x, const int4 &y) { return x.x < y.x; });
            const int n0C = distinct_outer(ent);
            if (!m || !n0C) continue;
            const long long q = b.alloc((long long)m * n0C);
            Blk Ab{m, n, A->row_perm, A->col_perm, A->row_inv, 0};
            std::vector<int> kk, pos, zr;
            size_t e = 0;
            while (e < ent.size())
            {
                const int c = ent[e].x;
                kk.clear();
                pos.clear();
                zr.clear();
                for (; e < ent.size() && ent[e].x == c; ++e)
                {
                    kk.push_back(ent[e].y);
                    pos.push_back(ent[e].z);
                    zr.push_back(0);
                }
                b.spvec(q + (long long)part.cols.size(), m, n0C, Ab.off, n, false, DP_SP_D_DENSE, kk, pos, zr, true);
                part.cols.push_back(c);
            }
            part.vals.push_back(DpPart::Val{part.cols, q, n0C, 1});
        }
        parts.push_back(std::move(part));
        kept.push_back(k);
    }
    std::unique_ptr<DenseProg> prog =
        jkind == A_SPD ? dp_blocks(b, parts, s) : dp_direct(b, b.p_total, s);
    std::vector<std::vector<int>> orows, ocols;
    std::vector<int> sp(1, 0);
    for (const DpPart &pt : parts)
    {
        orows.push_back(pt.rows);
        ocols.push_back(pt.cols);
        sp.push_back((int)sp.size());
    }
    matrix *C = make_spd(p * m, Jm->n, orows, ocols, sp, kept);
    try
    {
        dp_finish(*prog, b, (long long)m * n, jkind == A_SPARSE ? 0 : J.nnz,
                  jkind == A_SPARSE ? as_sparse(Jm)->csr->nnz : 0, 0, s);
        bind(C, DP_OP_KRON, std::move(prog));
    }
    catch (...)
    {
        free_matrix(C);
        throw;
    }
    return C;
}

void prog_dense_kron_fill(const matrix *Am, int p, const matrix *Jm, matrix *Cm)
{
    (void)p;
    if (Am->kind != MATRIX_PERMUTED_DENSE) fail(SDL_ERR_INVALID, "dense kron: A must be a full permuted_dense");
    const double *hr = nullptr, *Sx = nullptr;
    long long nr = 0;
    int ns = 0;
    if (dense_kind(Jm))
    {
        hr = host_values(const_cast<matrix *>(Jm));
        nr = value_count(Jm);
    }
    else
    {
        Sx = sparse_dev_values(as_sparse(Jm), runtime().stream);
        ns = as_sparse(Jm)->csr->nnz;
    }
    run(Cm, DP_OP_KRON, as_pd(Am)->X, value_count(Am), hr, nr, Sx, ns, nullptr, "dense kron fill_values");
}

} // namespace sdl
