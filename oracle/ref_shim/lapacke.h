/*
 * lapacke.h -- prototypes of the LAPACKE routines that the culip reference's
 * libs/la/dense_la_instances.cu wraps (host Cholesky helpers, not on the
 * block-iLDLt + SQMR path).  No LAPACK library is installed here:
 * ref_shim.cu defines them to abort.  TEST INFRASTRUCTURE ONLY.
 */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

lapack_int LAPACKE_spotrf(int layout, char uplo, lapack_int n, float* a, lapack_int lda);
lapack_int LAPACKE_dpotrf(int layout, char uplo, lapack_int n, double* a, lapack_int lda);
lapack_int LAPACKE_spotrs(int layout, char uplo, lapack_int n, lapack_int nrhs, const float* a, lapack_int lda,
                          float* b, lapack_int ldb);
lapack_int LAPACKE_dpotrs(int layout, char uplo, lapack_int n, lapack_int nrhs, const double* a, lapack_int lda,
                          double* b, lapack_int ldb);
lapack_int LAPACKE_sposv(int layout, char uplo, lapack_int n, lapack_int nrhs, float* a, lapack_int lda, float* b,
                         lapack_int ldb);
lapack_int LAPACKE_dposv(int layout, char uplo, lapack_int n, lapack_int nrhs, double* a, lapack_int lda, double* b,
                         lapack_int ldb);

#ifdef __cplusplus
}
#endif
