/* Minimal CBLAS prototypes (standard netlib CBLAS interface) so the reference
 * sources compile without a system cblas.h. Only the routines the reference's
 * dense-block kernels call are declared. The enum values are the standard
 * CBLAS ones, which every CBLAS implementation (OpenBLAS included) uses. */
#ifndef SDL_ORACLE_CBLAS_H
#define SDL_ORACLE_CBLAS_H
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;
void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc);
void cblas_dscal(int n, double alpha, double *x, int incx);
void cblas_dcopy(int n, const double *x, int incx, double *y, int incy);
double cblas_ddot(int n, const double *x, int incx, const double *y, int incy);
#endif
