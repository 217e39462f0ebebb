/* sparsediff_linalg drop-in (B200/CUDA build): Kronecker products.
 *
 * Same signatures and output-kind rules as upstream
 * include/sparsediff_linalg/matmul_kron.h (src/matmul_kron_dispatchers.c). A "full"
 * permuted_dense is one whose dense block covers its whole (m, n) shape, as built
 * by new_permuted_dense_full. Every fill bumps C's values_version and leaves C's
 * host values current. */
#ifndef SDL_MATMUL_KRON_H
#define SDL_MATMUL_KRON_H

#include "sparsediff_linalg/matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

/* y = kron(I_p, A) x: x holds p blocks of length A->n, y p blocks of length
   A->m. A is a sparse_matrix or a full permuted_dense. */
void BA_kron_vec_matrices(const matrix *A, const double *x, double *y, int p);

/* C = kron(A, I_m) J for a full permuted_dense A and J of any kind with
   J->m == m * A->n; C is a stacked_pd with one block per i < m (blocks without
   values dropped). */
matrix *BA_dense_kron_I_matrices_alloc(const matrix *A, int m, matrix *J);
void BA_dense_kron_I_matrices_fill_values(const matrix *A, int m, const matrix *J,
                                          matrix *C);

/* C = kron(I_p, A) J for A a full permuted_dense or a sparse_matrix and J of any
   kind with J->m == p * A->n. p == 1: as BA_matrices_*; A full permuted_dense:
   C stacked_pd; A sparse: C sparse. */
matrix *BA_kron_matrices_alloc(const matrix *A, int p, matrix *J);
void BA_kron_matrices_fill_values(const matrix *A, int p, matrix *J, matrix *C);

#ifdef __cplusplus
}
#endif

#endif /* SDL_MATMUL_KRON_H */
