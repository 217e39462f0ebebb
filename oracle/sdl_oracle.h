/* CPU oracle for the sparse-product path: a plain-C restatement of the upstream
 * algorithms, used only by the tests and by bench.py's CPU baseline as the
 * checker. Not part of the product library and never linked into it.
 *
 * All arrays are host arrays; every function mirrors the summation order and the
 * roundings of the upstream code it cites, so its results are bit-identical to
 * upstream's (pinned against upstream's own golden vectors and against the
 * upstream library built from source by oracle/Makefile). */
#ifndef SDL_ORACLE_H
#define SDL_ORACLE_H

#include <stdint.h>

/* C = kron(I_blocks, L) diag(d) A, rows sorted ascending.
 * Phase 1 writes Cp (L_m * blocks + 1 offsets) and returns nnz(C) (-1 if it does
 * not fit int32). Phase 2 writes Ci. Phase 3 writes Cx; Lx NULL means unit L
 * values, d NULL means identity. `work` needs A_n ints (phases 1, 2) or A_n doubles
 * (phase 3). */
long long orc_gustavson_count(const int *Lp, const int *Li, int L_m, int blocks,
                              const int *Ap, const int *Ai, int A_m, int A_n, int *Cp,
                              int *work);
void orc_gustavson_structure(const int *Lp, const int *Li, int L_m, int blocks,
                             const int *Ap, const int *Ai, int A_m, int A_n,
                             const int *Cp, int *Ci, int *work);
void orc_gustavson_values(const int *Lp, const int *Li, const double *Lx, int L_m,
                          int blocks, const double *d, const int *Ap, const int *Ai,
                          const double *Ax, int A_m, int A_n, const int *Cp,
                          const int *Ci, double *Cx, double *work);

/* Stable transpose (counting sort): rows x cols with nnz entries -> Tp (cols + 1),
 * Ti (source rows, ascending per output row), Tx (values; x may be NULL). */
void orc_transpose(const int *p, const int *idx, const double *x, int rows, int cols,
                   int *Tp, int *Ti, double *Tx, int *work);

/* Duplicate coalescing of nnz triplets into an m x n CSR: returns nnz_out and
 * writes Cp; the second call writes Ci, Cx (duplicates summed in ascending
 * triplet order from +0.0). */
long long orc_coalesce_count(const int *rows, const int *cols, int nnz, int m, int n,
                             int *Cp);
void orc_coalesce_fill(const int *rows, const int *cols, const double *x, int nnz, int m,
                       int n, const int *Cp, int *Ci, double *Cx);

/* Row gather C = A[map, :]: returns nnz(C) and writes Cp; then Ci / Cx. */
long long orc_row_gather_count(const int *Ap, const int *map, int m_out, int *Cp);
void orc_row_gather_fill(const int *Ap, const int *Ai, const double *Ax, const int *map,
                         int m_out, const int *Cp, int *Ci, double *Cx);

/* Row reduce C[g, :] = sum of rows i of A with group[i] == g. */
long long orc_row_reduce_count(const int *Ap, const int *Ai, int m, int n,
                               const int *group, int m_out, int *Cp);
void orc_row_reduce_fill(const int *Ap, const int *Ai, const double *Ax, int m, int n,
                         const int *group, int m_out, const int *Cp, int *Ci,
                         double *Cx);

/* Dense helpers for the block paths: C (rows x cols, row-major) =
 * sum_k A[k, r] * w[k] * B[k, c] summed over ascending k in double (w NULL = 1). */
void orc_dense_btdb(const double *A, const double *B, const double *w, int K, int rows,
                    int cols, double *C);

#endif /* SDL_ORACLE_H */
