/* sparsediff_linalg drop-in (B200/CUDA build): compressed sparse row storage.
 *
 * Byte-identical layout and signatures to the upstream public header
 * include/sparsediff_linalg/CSR_matrix.h:31-55, so a consumer compiled against the
 * upstream headers links against this library unchanged. Arrays are host memory
 * (malloc/free, as upstream); the library mirrors them to the GPU itself. */
#ifndef SDL_CSR_MATRIX_H
#define SDL_CSR_MATRIX_H

#ifdef __cplusplus
extern "C" {
#endif

/* m x n matrix: p has m + 1 row offsets, i has nnz column indices, x has nnz
 * values; row r holds entries p[r] <= k < p[r + 1]. */
typedef struct CSR_matrix
{
    int *p;
    int *i;
    double *x;
    int m;
    int n;
    int nnz;
} CSR_matrix;

/* Allocate an m x n CSR with room for nnz entries; p is zeroed. */
CSR_matrix *new_CSR_matrix(int m, int n, int nnz);
/* Deep copy. */
CSR_matrix *new_csr(const CSR_matrix *A);
void free_CSR_matrix(CSR_matrix *matrix);
/* Copy A's shape, structure and values into the already-sized C. */
void copy_CSR_matrix(const CSR_matrix *A, CSR_matrix *C);

/* Shrink i and x to p[m] entries and set nnz (for capacity-built CSRs). */
void CSR_trim(CSR_matrix *A);

/* A^T as a CSR (column indices of each row of A^T ascending). iwork: A->n ints. */
CSR_matrix *transpose(const CSR_matrix *A, int *iwork);
/* Structure of A^T only; values left unset. */
CSR_matrix *AT_alloc(const CSR_matrix *A, int *iwork);
/* Values of A^T into an AT built by AT_alloc(A). */
void AT_fill_values(const CSR_matrix *A, CSR_matrix *AT, int *iwork);

#ifdef __cplusplus
}
#endif

#endif /* SDL_CSR_MATRIX_H */
