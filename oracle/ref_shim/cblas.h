/*
 * cblas.h -- prototypes of the CBLAS routines that the culip reference's
 * libs/la/dense_la_instances.cu wraps (host T_H_* helpers, not on the
 * block-iLDLt + SQMR path).  No BLAS library is installed here: ref_shim.cu
 * defines them to abort.  TEST INFRASTRUCTURE ONLY (reference build).
 */
#pragma once

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

void cblas_saxpy(const int n, const float alpha, const float* x, const int incx, float* y, const int incy);
void cblas_daxpy(const int n, const double alpha, const double* x, const int incx, double* y, const int incy);
void cblas_sgemv(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE trans, const int m, const int n,
                 const float alpha, const float* a, const int lda, const float* x, const int incx, const float beta,
                 float* y, const int incy);
void cblas_dgemv(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE trans, const int m, const int n,
                 const double alpha, const double* a, const int lda, const double* x, const int incx,
                 const double beta, double* y, const int incy);
void cblas_sgemm(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE ta, const enum CBLAS_TRANSPOSE tb,
                 const int m, const int n, const int k, const float alpha, const float* a, const int lda,
                 const float* b, const int ldb, const float beta, float* c, const int ldc);
void cblas_dgemm(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE ta, const enum CBLAS_TRANSPOSE tb,
                 const int m, const int n, const int k, const double alpha, const double* a, const int lda,
                 const double* b, const int ldb, const double beta, double* c, const int ldc);
