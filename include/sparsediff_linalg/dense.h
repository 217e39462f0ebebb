/* sparsediff_linalg drop-in (B200/CUDA build): dense-vector helpers.
 *
 * Same signatures and results as upstream include/sparsediff_linalg/dense.h
 * (src/support/mini_numpy.c); host arrays in and out, computed on the device with
 * every sum in upstream's loop order. */
#ifndef SDL_DENSE_H
#define SDL_DENSE_H

#ifdef __cplusplus
extern "C" {
#endif

/* result[i * repeats + j] = a[i] */
void repeat(double *result, const double *a, int len, int repeats);
/* result[i * len + t] = a[t] for i < tiles */
void tile_double(double *result, const double *a, int len, int tiles);
/* result[i] = value */
void scaled_ones(double *result, int size, double value);
/* Row-major dense transpose: AT[j*m + i] = A[i*n + j] for an m x n A. */
void A_transpose(double *AT, const double *A, int m, int n);
/* v = (Y kron I_m) w for Y k x n (col-major), len(w) = m n, len(v) = m k. */
void Y_kron_I_vec(int m, int k, int n, const double *Y, const double *w, double *v);
/* v = (I_n kron X^T) w for X m x k (col-major), len(w) = m n, len(v) = k n. */
void I_kron_XT_vec(int m, int k, int n, const double *X, const double *w, double *v);

#ifdef __cplusplus
}
#endif

#endif /* SDL_DENSE_H */
