/* sparsediff_linalg drop-in (B200/CUDA build): polymorphic matrix handle.
 *
 * Same struct layout, vtable slot order, enum values and constructor signatures
 * as upstream include/sparsediff_linalg/matrix.h:31-168. The kinds' private
 * layouts differ (they carry device mirrors); consumers only ever see the handle. */
#ifndef SDL_MATRIX_H
#define SDL_MATRIX_H

#include "sparsediff_linalg/CSC_matrix.h"
#include "sparsediff_linalg/CSR_matrix.h"
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct matrix matrix;

/* MATRIX_SPARSE is 0 so a zeroed handle is the sparse kind. */
typedef enum
{
    MATRIX_SPARSE = 0,     /* CSR-backed */
    MATRIX_PERMUTED_DENSE, /* one dense block at sorted row/col subsets */
    MATRIX_STACKED_PD      /* row-disjoint stack of permuted_dense blocks */
} matrix_kind;

typedef CSR_matrix *(*matrix_to_csr_fn)(matrix *A);
/* C = A[map, :]; C keeps map, so the fill takes none. */
typedef matrix *(*matrix_row_gather_alloc_fn)(const matrix *A, const int *map,
                                              int m_out);
typedef void (*matrix_row_gather_fill_values_fn)(const matrix *A, matrix *C);
/* C[g, :] = sum of rows i with group[i] == g, 0 <= group[i] < m_out. */
typedef matrix *(*matrix_row_reduce_alloc_fn)(const matrix *A, const int *group,
                                              int m_out);
typedef void (*matrix_row_reduce_fill_values_fn)(const matrix *A, matrix *C);

struct matrix
{
    int m, n, nnz;
    double *x; /* host value buffer, not owned by the handle */
    matrix_kind kind;

    /* Bumped whenever x changes. Every library fill bumps its output; code that
     * writes x directly calls matrix_values_changed on the owner. The GPU layer
     * re-uploads an operand's values iff this moved since its last upload. */
    uint64_t values_version;

    matrix_to_csr_fn to_csr;
    matrix_row_gather_alloc_fn row_gather_alloc;
    matrix_row_gather_fill_values_fn row_gather_fill_values;
    matrix_row_reduce_alloc_fn row_reduce_alloc;
    matrix_row_reduce_fill_values_fn row_reduce_fill_values;
};

static inline void matrix_values_changed(matrix *A)
{
    A->values_version++;
}

/* NULL is a no-op. */
void free_matrix(matrix *m);

/* Same kind and sparsity as A; values uninitialised. */
matrix *copy_sparsity_matrices_alloc(const matrix *A);

/* AT = A^T of A's kind (structure only), and its fill (bumps AT's version). */
matrix *transpose_matrices_alloc(const matrix *A);
void transpose_matrices_fill_values(const matrix *A, matrix *AT);

/* Sparse kind. Takes ownership of A (free_matrix frees it). */
matrix *new_sparse_matrix(CSR_matrix *A);
/* new_sparse_matrix(new_CSR_matrix(m, n, nnz)). */
matrix *new_sparse_matrix_alloc(int m, int n, int nnz);

/* permuted_dense: M[row_perm[ii], col_perm[jj]] = X[ii * n0 + jj], zero elsewhere;
 * row_perm / col_perm strictly increasing. X_data NULL leaves values unset,
 * otherwise m0 * n0 values are copied. */
typedef struct permuted_dense permuted_dense;
matrix *new_permuted_dense(int m, int n, int m0, int n0, const int *row_perm,
                           const int *col_perm, const double *X_data);
/* Identity perms, the block fills the whole m x n shape. */
matrix *new_permuted_dense_full(int m, int n, const double *data);

/* stacked_pd: vertical union of n_blocks permuted_dense blocks with disjoint
 * row_perms (column perms may overlap). Takes ownership of every block.
 * src_block_idx_p / src_block_idx (CSR-style, may be NULL for the identity) record
 * which source blocks fed each block. */
matrix *new_stacked_pd(int m, int n, int n_blocks, permuted_dense **blocks,
                       const int *src_block_idx_p, const int *src_block_idx);

#ifdef __cplusplus
}
#endif

#endif /* SDL_MATRIX_H */
