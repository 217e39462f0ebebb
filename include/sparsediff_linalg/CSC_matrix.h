/* sparsediff_linalg drop-in (B200/CUDA build): compressed sparse column storage
 * and the raw B^T D A product.
 *
 * Same layout and signatures as upstream include/sparsediff_linalg/CSC_matrix.h:33-61. */
#ifndef SDL_CSC_MATRIX_H
#define SDL_CSC_MATRIX_H

#include "sparsediff_linalg/CSR_matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

/* m x n matrix: p has n + 1 column offsets, i has nnz row indices, x has nnz values. */
typedef struct CSC_matrix
{
    int *p;
    int *i;
    double *x;
    int m;
    int n;
    int nnz;
} CSC_matrix;

/* Returns NULL if a host allocation fails. */
CSC_matrix *new_CSC_matrix(int m, int n, int nnz);
void free_CSC_matrix(CSC_matrix *matrix);

/* Exact structure of C = B^T D A (B is CSC, A is CSR, C is CSR with ascending,
 * unique column indices per row). Computed on the GPU. */
CSR_matrix *BTA_alloc(const CSR_matrix *A, const CSC_matrix *B);

/* Values of C = B^T diag(d) A into the C returned by BTA_alloc(A, B). d == NULL
 * means the identity. acc (A->n doubles) is accepted for ABI compatibility and is
 * not touched: the GPU keeps its accumulators on chip. Each entry is summed in the
 * same order and with the same roundings as the upstream CPU code. */
void BTDA_fill_values(const CSR_matrix *A, const CSC_matrix *B, const double *d,
                      double *acc, CSR_matrix *C);

/* CSR -> CSC (row indices ascending inside each column). iwork: A->n ints. */
CSC_matrix *csr_to_csc_alloc(const CSR_matrix *A, int *iwork);
void csr_to_csc_fill_values(const CSR_matrix *A, CSC_matrix *C, int *iwork);

/* CSC -> CSR (column indices ascending inside each row). iwork: A->m ints. */
CSR_matrix *csc_to_csr_alloc(const CSC_matrix *A, int *iwork);
void csc_to_csr_fill_values(const CSC_matrix *A, CSR_matrix *C, int *iwork);

#ifdef __cplusplus
}
#endif

#endif /* SDL_CSC_MATRIX_H */
