/* sparsediff_linalg drop-in (B200/CUDA build): coordinate storage.
 *
 * Same layout and signatures as upstream include/sparsediff_linalg/COO_matrix.h:35-57.
 * Duplicate coalescing (COO -> CSR with summed duplicates) has no upstream
 * counterpart; it is in sparsediff_linalg_cuda.h (sdl_coo_coalesce). */
#ifndef SDL_COO_MATRIX_H
#define SDL_COO_MATRIX_H

#include "sparsediff_linalg/CSR_matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

/* nnz triplets (rows[k], cols[k], x[k]); value_map[k] is the CSR position entry k
 * was taken from (lower-triangular form only, else NULL). */
typedef struct COO_matrix
{
    int *rows;
    int *cols;
    double *x;
    int *value_map;
    int m;
    int n;
    int nnz;
} COO_matrix;

COO_matrix *new_COO_matrix(const CSR_matrix *A);
/* Entries with col <= row of a symmetric CSR, with value_map filled. */
COO_matrix *new_COO_matrix_lower_triangular(const CSR_matrix *A);
/* coo->x[k] = vals[coo->value_map[k]]. */
void refresh_lower_triangular_coo(COO_matrix *coo, const double *vals);
void free_COO_matrix(COO_matrix *matrix);

#ifdef __cplusplus
}
#endif

#endif /* SDL_COO_MATRIX_H */
