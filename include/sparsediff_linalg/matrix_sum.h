/* sparsediff_linalg drop-in (B200/CUDA build): sums of matrices.
 *
 * Same signatures and semantics as upstream include/sparsediff_linalg/matrix_sum.h
 * (src/sparse/matrix_sum.c, src/sparse/CSR_sum.c): operands of any kind with equal
 * shapes; C is a sparse matrix whose pattern is the union of the operands'
 * patterns; every entry is the sum of the operands holding it, added from +0.0 in
 * operand order. Every fill bumps C's values_version and leaves C's host values
 * current. */
#ifndef SDL_MATRIX_SUM_H
#define SDL_MATRIX_SUM_H

#include "sparsediff_linalg/matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

/* C = A + B. C is a sparse matrix the caller allocated with room for
   nnz(A) + nnz(B) entries; the alloc writes the merged pattern and trims C. */
void sum_matrices_alloc(matrix *A, matrix *B, matrix *C);
void sum_matrices_fill_values(matrix *A, matrix *B, matrix *C);
/* C = diag(d1) A + diag(d2) B (len(d1) = len(d2) = A->m) into the C of
   sum_matrices_alloc. */
void sum_scaled_matrices_fill_values(matrix *A, matrix *B, matrix *C,
                                     const double *d1, const double *d2);

/* C = A + B + D + E; C is a new sparse matrix. */
matrix *sum_4_matrices_alloc(matrix *A, matrix *B, matrix *D, matrix *E);
void sum_4_matrices_fill_values(const matrix *A, const matrix *B, const matrix *D,
                                const matrix *E, matrix *C);

/* C = ops[0] + ... + ops[n-1] (n >= 1; an operand may appear more than once). */
matrix *sum_n_matrices_alloc(matrix *const *ops, int n);
/* ops must be the same operands, in the same order, as at the alloc. */
void sum_n_matrices_fill_values(matrix *const *ops, int n, matrix *C);
/* Incremental form: zero C, then add operand k (its alloc position) once its
   values are final; stays correct when a later operand's evaluation overwrites an
   earlier one's values. */
void sum_n_matrices_fill_zero(matrix *C);
void sum_n_matrices_fill_add(const matrix *op, int k, matrix *C);

#ifdef __cplusplus
}
#endif

#endif /* SDL_MATRIX_SUM_H */
