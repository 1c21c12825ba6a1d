/* Minimal lapacke.h for building the reference's FSAI and BAMG C++ sources
 * against the LAPACKE symbols exported by scipy's bundled OpenBLAS
 * (scipy.libs/libscipy_openblas-*.so, LP64: lapack_int = int).
 *
 * Oracle test infrastructure only: nothing in the chronoslab_b200 package
 * includes or links this header.  It declares the LAPACKE entry points the
 * reference calls (dpotrf/dpotrs in cpt_afsai_coef.cpp:446,454, dgels_work in
 * BAMG.cpp:64,165 / Reduce_IntSet.cpp, and dgeqrf/dorgqr/dgesvd/dtrtrs in the
 * EMIN sources' emin_blas.h) and maps them onto the scipy_-prefixed exports. */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

lapack_int scipy_LAPACKE_dpotrf(int matrix_layout, char uplo, lapack_int n,
                                double *a, lapack_int lda);
lapack_int scipy_LAPACKE_dpotrs(int matrix_layout, char uplo, lapack_int n,
                                lapack_int nrhs, const double *a, lapack_int lda,
                                double *b, lapack_int ldb);
lapack_int scipy_LAPACKE_dgels_work(int matrix_layout, char trans, lapack_int m,
                                    lapack_int n, lapack_int nrhs, double *a,
                                    lapack_int lda, double *b, lapack_int ldb,
                                    double *work, lapack_int lwork);
lapack_int scipy_LAPACKE_dgeqrf_work(int matrix_layout, lapack_int m, lapack_int n, double *a,
                                     lapack_int lda, double *tau, double *work,
                                     lapack_int lwork);
lapack_int scipy_LAPACKE_dorgqr_work(int matrix_layout, lapack_int m, lapack_int n,
                                     lapack_int k, double *a, lapack_int lda,
                                     const double *tau, double *work, lapack_int lwork);
lapack_int scipy_LAPACKE_dgesvd_work(int matrix_layout, char jobu, char jobvt, lapack_int m,
                                     lapack_int n, double *a, lapack_int lda, double *s,
                                     double *u, lapack_int ldu, double *vt, lapack_int ldvt,
                                     double *work, lapack_int lwork);
lapack_int scipy_LAPACKE_dtrtrs(int matrix_layout, char uplo, char trans, char diag,
                                lapack_int n, lapack_int nrhs, const double *a, lapack_int lda,
                                double *b, lapack_int ldb);

#ifdef __cplusplus
}
#endif

#define LAPACKE_dpotrf scipy_LAPACKE_dpotrf
#define LAPACKE_dpotrs scipy_LAPACKE_dpotrs
#define LAPACKE_dgels_work scipy_LAPACKE_dgels_work
#define LAPACKE_dgeqrf_work scipy_LAPACKE_dgeqrf_work
#define LAPACKE_dorgqr_work scipy_LAPACKE_dorgqr_work
#define LAPACKE_dgesvd_work scipy_LAPACKE_dgesvd_work
#define LAPACKE_dtrtrs scipy_LAPACKE_dtrtrs
