/*
 * culip_ref_shim.h -- force-included (nvcc -include) into every translation
 * unit of the culip reference when oracle/build_ref.py compiles it for
 * sm_100a with CUDA 12.9.
 *
 * TEST INFRASTRUCTURE ONLY: the reference build is the checker of the
 * culip_b200 factorization and solves, never part of the product.
 *
 * It supplies what the reference's sources assume from CUDA <= 10:
 *   - headers the reference uses without including them: Thrust
 *     algorithms (thrust::remove_if / count / sort / transform in
 *     libs/la/preconditioner/block_ildlt.impl.cuh) and <fstream>
 *     (std::ifstream in libs/test/test.impl.h);
 *   - the type cusparseSolveAnalysisInfo_t (removed in CUDA 11);
 *   - declarations of the legacy cuSPARSE routines that
 *     libs/la/sparse_la_instances.cu calls and CUDA 12 no longer ships.
 *     csrmv and csr2csc are defined in ref_shim.cu on the generic API
 *     (cusparseSpMV, cusparseCsr2cscEx2); the others are not on the
 *     block-iLDLt + SQMR path and report CUSPARSE_STATUS_NOT_SUPPORTED.
 */
#pragma once

#include <cuda_runtime.h>
#include <cusparse.h>

#ifdef __cplusplus
#include <fstream>
#include <thrust/count.h>
#include <thrust/execution_policy.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/remove.h>
#include <thrust/sort.h>
#include <thrust/transform.h>

typedef void* cusparseSolveAnalysisInfo_t;
typedef void* csrsv2Info_t;

/* y = alpha * op(A) x + beta * y, CSR (legacy cusparse<t>csrmv) */
cusparseStatus_t cusparseScsrmv(cusparseHandle_t h, cusparseOperation_t op, int m, int n, int nnz, const float* alpha,
                                const cusparseMatDescr_t descr, const float* val, const int* rowptr,
                                const int* colidx, const float* x, const float* beta, float* y);
cusparseStatus_t cusparseDcsrmv(cusparseHandle_t h, cusparseOperation_t op, int m, int n, int nnz,
                                const double* alpha, const cusparseMatDescr_t descr, const double* val,
                                const int* rowptr, const int* colidx, const double* x, const double* beta,
                                double* y);

/* CSR -> CSC (legacy cusparse<t>csr2csc) */
cusparseStatus_t cusparseScsr2csc(cusparseHandle_t h, int m, int n, int nnz, const float* val, const int* rowptr,
                                  const int* colidx, float* csc_val, int* csc_row, int* csc_colptr,
                                  cusparseAction_t action, cusparseIndexBase_t base);
cusparseStatus_t cusparseDcsr2csc(cusparseHandle_t h, int m, int n, int nnz, const double* val, const int* rowptr,
                                  const int* colidx, double* csc_val, int* csc_row, int* csc_colptr,
                                  cusparseAction_t action, cusparseIndexBase_t base);

/* legacy routines off the solve path: accepted for any arguments, never run */
#define CULIP_REF_UNSUPPORTED(name)                                       \
    template <class... Args>                                              \
    inline cusparseStatus_t name(Args&&...)                               \
    {                                                                     \
        return CUSPARSE_STATUS_NOT_SUPPORTED;                             \
    }
CULIP_REF_UNSUPPORTED(cusparseXcsrgeamNnz)
CULIP_REF_UNSUPPORTED(cusparseScsrgeam)
CULIP_REF_UNSUPPORTED(cusparseDcsrgeam)
CULIP_REF_UNSUPPORTED(cusparseXcsrgemmNnz)
CULIP_REF_UNSUPPORTED(cusparseScsrgemm)
CULIP_REF_UNSUPPORTED(cusparseDcsrgemm)
CULIP_REF_UNSUPPORTED(cusparseScsrsv_analysis)
CULIP_REF_UNSUPPORTED(cusparseDcsrsv_analysis)
CULIP_REF_UNSUPPORTED(cusparseScsrsv_solve)
CULIP_REF_UNSUPPORTED(cusparseDcsrsv_solve)
CULIP_REF_UNSUPPORTED(cusparseCreateCsrsv2Info)
CULIP_REF_UNSUPPORTED(cusparseDestroyCsrsv2Info)
CULIP_REF_UNSUPPORTED(cusparseScsrsv2_bufferSize)
CULIP_REF_UNSUPPORTED(cusparseDcsrsv2_bufferSize)
CULIP_REF_UNSUPPORTED(cusparseScsrsv2_analysis)
CULIP_REF_UNSUPPORTED(cusparseDcsrsv2_analysis)
CULIP_REF_UNSUPPORTED(cusparseScsrsv2_solve)
CULIP_REF_UNSUPPORTED(cusparseDcsrsv2_solve)
#undef CULIP_REF_UNSUPPORTED
#endif
