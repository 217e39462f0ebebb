/* sparsediff_linalg drop-in (B200/CUDA build): vertical stacking.
 *
 * Same signatures and semantics as upstream include/sparsediff_linalg/
 * matrix_vstack.h (src/sparse/matrix_vstack.c). */
#ifndef SDL_MATRIX_VSTACK_H
#define SDL_MATRIX_VSTACK_H

#include "sparsediff_linalg/matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

/* C = [ops[0]; ...; ops[n-1]] for n >= 1 operands of any kind with equal column
   counts; C is a sparse matrix whose rows are the operands' rows in order. */
matrix *vstack_matrices_alloc(matrix *const *ops, int n);
/* ops must be the same matrices, in the same order, as at the alloc. Copies the
   operands whose values_version moved since the previous fill (all of them after
   C itself was written and matrix_values_changed(C) called) and bumps C's
   values_version iff it copied something. */
void vstack_matrices_fill_values(matrix *const *ops, int n, matrix *C);

#ifdef __cplusplus
}
#endif

#endif /* SDL_MATRIX_VSTACK_H */
