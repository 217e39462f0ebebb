/* CPU baseline timing harness (test / bench infrastructure only).
 *
 * Times upstream's own B^T D A and SpGEMM entry points (linked from
 * _ref/libsdl_ref.so, the upstream library compiled from its sources) on caller
 * arrays, so bench.py can report the reference CPU path beside the GPU numbers
 * without Python overhead inside the timed loop. Each call returns seconds per
 * repetition measured with CLOCK_MONOTONIC. */
#define _POSIX_C_SOURCE 199309L
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct
{
    int *p, *i;
    double *x;
    int m, n, nnz;
} mat_t; /* layout of upstream CSR_matrix / CSC_matrix */

typedef struct matrix matrix;
extern mat_t *new_CSR_matrix(int m, int n, int nnz);
extern void free_CSR_matrix(mat_t *);
extern void free_CSC_matrix(mat_t *);
extern mat_t *csr_to_csc_alloc(const mat_t *A, int *iwork);
extern void csr_to_csc_fill_values(const mat_t *A, mat_t *C, int *iwork);
extern mat_t *BTA_alloc(const mat_t *A, const mat_t *B);
extern void BTDA_fill_values(const mat_t *A, const mat_t *B, const double *d, double *acc, mat_t *C);
extern matrix *new_sparse_matrix(mat_t *A);
extern void free_matrix(matrix *);
extern matrix *BTA_matrices_alloc(matrix *A, matrix *B);
extern void BTDA_matrices_fill_values(matrix *A, const double *d, matrix *B, matrix *C);
extern matrix *BA_matrices_alloc(const matrix *B, matrix *A);
extern void BA_matrices_fill_values(const matrix *B, const matrix *A, matrix *C);

struct matrix_head
{
    int m, n, nnz;
    double *x;
    int kind;
    unsigned long long values_version;
};

static double now(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static mat_t *copy_csr(const int *p, const int *i, const double *x, int m, int n)
{
    int nnz = p[m];
    mat_t *A = new_CSR_matrix(m, n, nnz);
    memcpy(A->p, p, (size_t)(m + 1) * sizeof(int));
    memcpy(A->i, i, (size_t)nnz * sizeof(int));
    memcpy(A->x, x, (size_t)nnz * sizeof(double));
    return A;
}

/* B^T D A through upstream's matrix dispatchers, the path SparseDiffEngine
 * calls. out[0] = alloc seconds (CSC mirror + symbolic + plan), out[1] = seconds
 * per refill in which A, B and d all change (the fill refreshes B's CSC mirror),
 * out[2] = nnz(C). The refills alternate between two value sets. */
void ref_time_btda(const int *Ap, const int *Ai, const double *Ax, const double *Ax2, int m, int nA,
                   const int *Bp, const int *Bi, const double *Bx, const double *Bx2, int nB,
                   const double *d, const double *d2, int reps, double *out)
{
    mat_t *A = copy_csr(Ap, Ai, Ax, m, nA);
    mat_t *B = copy_csr(Bp, Bi, Bx, m, nB);
    matrix *Am = new_sparse_matrix(A);
    matrix *Bm = new_sparse_matrix(B);
    double t0 = now();
    matrix *Cm = BTA_matrices_alloc(Am, Bm);
    BTDA_matrices_fill_values(Am, d, Bm, Cm);
    out[0] = now() - t0;
    int nnzA = Ap[m], nnzB = Bp[m];
    t0 = now();
    for (int r = 0; r < reps; ++r)
    {
        const double *ax = (r & 1) ? Ax : Ax2, *bx = (r & 1) ? Bx : Bx2, *dd = (r & 1) ? d : d2;
        memcpy(A->x, ax, (size_t)nnzA * sizeof(double));
        memcpy(B->x, bx, (size_t)nnzB * sizeof(double));
        ((struct matrix_head *)Am)->values_version++;
        ((struct matrix_head *)Bm)->values_version++;
        BTDA_matrices_fill_values(Am, dd, Bm, Cm);
    }
    out[1] = (now() - t0) / (reps > 0 ? reps : 1);
    out[2] = ((struct matrix_head *)Cm)->nnz;
    free_matrix(Cm);
    free_matrix(Am);
    free_matrix(Bm);
}

/* C = A B (A's rows are the left operand, as upstream's BA_matrices with a sparse
 * left factor). out[0] = alloc seconds, out[1] = seconds per fill, out[2] = nnz. */
void ref_time_spgemm(const int *Ap, const int *Ai, const double *Ax, int mA, int nA,
                     const int *Bp, const int *Bi, const double *Bx, int nB, int reps, double *out)
{
    mat_t *A = copy_csr(Ap, Ai, Ax, mA, nA);
    mat_t *B = copy_csr(Bp, Bi, Bx, nA, nB);
    matrix *Am = new_sparse_matrix(A);
    matrix *Bm = new_sparse_matrix(B);
    double t0 = now();
    matrix *Cm = BA_matrices_alloc(Am, Bm);
    out[0] = now() - t0;
    t0 = now();
    for (int r = 0; r < reps; ++r)
    {
        ((struct matrix_head *)Am)->values_version++;
        BA_matrices_fill_values(Am, Bm, Cm);
    }
    out[1] = (now() - t0) / (reps > 0 ? reps : 1);
    out[2] = ((struct matrix_head *)Cm)->nnz;
    free_matrix(Cm);
    free_matrix(Am);
    free_matrix(Bm);
}

/* CSR -> CSC conversion through upstream's raw kernels (the CSC mirror refresh of
 * SparseDiffEngine). out[0] = alloc seconds (structure), out[1] = seconds per
 * value refill, out[2] = nnz. */
void ref_time_csr_to_csc(const int *Ap, const int *Ai, const double *Ax, int m, int n, int reps,
                         double *out)
{
    mat_t *A = copy_csr(Ap, Ai, Ax, m, n);
    int *iwork = (int *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    double t0 = now();
    mat_t *C = csr_to_csc_alloc(A, iwork);
    out[0] = now() - t0;
    t0 = now();
    for (int r = 0; r < reps; ++r) csr_to_csc_fill_values(A, C, iwork);
    out[1] = (now() - t0) / (reps > 0 ? reps : 1);
    out[2] = Ap[m];
    free(iwork);
    free_CSC_matrix(C);
    free_CSR_matrix(A);
}

/* stacked_pd x CSR through upstream's BA_spd_csr_alloc / BA_spd_csr_fill_values
 * (src/stacked_pd/stacked_pd_linalg.c:657-671): n_blocks dense blocks of m0 x n0
 * with row_perm rows[k * m0 ...] of an m-row stacked_pd and col_perm cperm (shared),
 * values X (block-major). out[0] = alloc seconds, out[1] = seconds per fill. */
extern matrix *new_permuted_dense(int m, int n, int m0, int n0, const int *row_perm,
                                  const int *col_perm, const double *X);
extern matrix *new_stacked_pd(int m, int n, int n_blocks, matrix **blocks,
                              const int *src_block_idx_p, const int *src_block_idx);
extern matrix *BA_spd_csr_alloc(const matrix *B, const mat_t *S);
extern void BA_spd_csr_fill_values(const matrix *B, const mat_t *S, matrix *C);

void ref_time_ba_spd_csr(int m, int n_blocks, int m0, int n0, const int *rows, const int *cperm,
                         const double *X, const int *Sp, const int *Si, const double *Sx, int S_m,
                         int S_n, int reps, double *out)
{
    matrix **blocks = (matrix **)malloc((size_t)n_blocks * sizeof(matrix *));
    for (int k = 0; k < n_blocks; ++k)
        blocks[k] = new_permuted_dense(m, S_m, m0, n0, rows + (size_t)k * m0, cperm,
                                       X + (size_t)k * m0 * n0);
    matrix *B = new_stacked_pd(m, S_m, n_blocks, blocks, NULL, NULL);
    free(blocks);
    mat_t *S = copy_csr(Sp, Si, Sx, S_m, S_n);
    double t0 = now();
    matrix *C = BA_spd_csr_alloc(B, S);
    out[0] = now() - t0;
    t0 = now();
    for (int r = 0; r < reps; ++r) BA_spd_csr_fill_values(B, S, C);
    out[1] = (now() - t0) / (reps > 0 ? reps : 1);
    free_matrix(C);
    free_matrix(B);
    free_CSR_matrix(S);
}

/* A^T diag(d) A of the same stacked_pd through upstream's ATA_matrices_alloc /
 * ATDA_matrices_fill_values (per-block cblas_dgemm, then coalescing).
 * out[0] = alloc seconds, out[1] = seconds per fill. */
extern matrix *ATA_matrices_alloc(matrix *A);
extern void ATDA_matrices_fill_values(const matrix *A, const double *d, matrix *C);

void ref_time_atda_spd(int m, int n, int n_blocks, int m0, int n0, const int *rows, const int *cperm,
                       const double *X, const double *d, int reps, double *out)
{
    matrix **blocks = (matrix **)malloc((size_t)n_blocks * sizeof(matrix *));
    for (int k = 0; k < n_blocks; ++k)
        blocks[k] = new_permuted_dense(m, n, m0, n0, rows + (size_t)k * m0, cperm, X + (size_t)k * m0 * n0);
    matrix *A = new_stacked_pd(m, n, n_blocks, blocks, NULL, NULL);
    free(blocks);
    double t0 = now();
    matrix *C = ATA_matrices_alloc(A);
    out[0] = now() - t0;
    t0 = now();
    for (int r = 0; r < reps; ++r) ATDA_matrices_fill_values(A, d, C);
    out[1] = (now() - t0) / (reps > 0 ? reps : 1);
    free_matrix(C);
    free_matrix(A);
}
