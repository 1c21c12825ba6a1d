/* Minimal cblas.h for building the reference's EMIN C++ sources (emin_blas.h
 * calls cblas_dgemv) against scipy's bundled OpenBLAS, whose CBLAS exports
 * carry a scipy_ prefix.
 *
 * Oracle test infrastructure only: nothing in the chronoslab_b200 package
 * includes or links this header. */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

void scipy_cblas_dgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, int m, int n, double alpha,
                       const double *a, int lda, const double *x, int incx, double beta,
                       double *y, int incy);

#ifdef __cplusplus
}
#endif

#define cblas_dgemv scipy_cblas_dgemv
