/* sparsediff_linalg drop-in (B200/CUDA build): polymorphic products.
 *
 * Same signatures and output-kind rules as upstream
 * include/sparsediff_linalg/matmul.h:38-69:
 *   B permuted_dense -> C permuted_dense; B stacked_pd -> C stacked_pd;
 *   B sparse -> C has A's kind.
 * Sparse operands are read by column through a device-resident CSC mirror that
 * the fills keep in step with the operand's values_version. Every fill bumps C's
 * values_version and leaves C's host values current. */
#ifndef SDL_MATMUL_H
#define SDL_MATMUL_H

#include "sparsediff_linalg/matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

/* C = B^T A and C = B^T diag(d) A (d: A->m values, NULL = identity). */
matrix *BTA_matrices_alloc(matrix *A, matrix *B);
void BTA_matrices_fill_values(matrix *A, matrix *B, matrix *C);
void BTDA_matrices_fill_values(matrix *A, const double *d, matrix *B, matrix *C);

/* C = diag(d) A into C = copy_sparsity_matrices_alloc(A); len(d) = A->m. */
void DA_matrices_fill_values(const double *d, const matrix *A, matrix *C);

/* C = A^T A and C = A^T diag(d) A; C has A's kind. */
matrix *ATA_matrices_alloc(matrix *A);
void ATDA_matrices_fill_values(const matrix *A, const double *d, matrix *C);

/* C = B A for a sparse or permuted_dense B (a stacked_pd B is rejected). */
matrix *BA_matrices_alloc(const matrix *B, matrix *A);
void BA_matrices_fill_values(const matrix *B, const matrix *A, matrix *C);

#ifdef __cplusplus
}
#endif

#endif /* SDL_MATMUL_H */
