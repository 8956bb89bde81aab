/*
 * ref_shim.cu -- definitions behind culip_ref_shim.h, cblas.h and lapacke.h
 * for the reference build (oracle/build_ref.py).  TEST INFRASTRUCTURE ONLY.
 *
 * The reference's CSR product T_csrmv (libs/la/sparse_la_instances.cu:129-217)
 * calls the legacy cusparse<t>csrmv, removed in CUDA 11; here it runs on the
 * generic cusparseSpMV with the same arguments and the handle's pointer mode
 * and stream (CSR_ALG2, deterministic, for the non-transposed product).
 * T_transpose_csr's cusparse<t>csr2csc runs on cusparseCsr2cscEx2.
 * The BLAS/LAPACKE wrappers are host helpers off the solve path; calling one
 * aborts with a message.
 */
#include "culip_ref_shim.h"
extern "C" {
#include "cblas.h"
}
#include "lapacke.h"

#include <cstdio>
#include <cstdlib>

namespace {

// one growable work buffer per host thread (the reference runs one thread)
struct WorkBuffer {
    void* p = nullptr;
    size_t bytes = 0;
    void* get(size_t need)
    {
        if (need <= bytes) return p;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, need) != cudaSuccess) return nullptr;
        bytes = need;
        return p;
    }
};
thread_local WorkBuffer g_buf;

cusparseStatus_t spmv_csr(cusparseHandle_t h, cusparseOperation_t op, int m, int n, int nnz, const void* alpha,
                          const void* val, const int* rowptr, const int* colidx, const void* x, const void* beta,
                          void* y, cudaDataType vt)
{
    cusparseSpMatDescr_t A = nullptr;
    cusparseDnVecDescr_t X = nullptr, Y = nullptr;
    const bool nt = op == CUSPARSE_OPERATION_NON_TRANSPOSE;
    const cusparseSpMVAlg_t alg = nt ? CUSPARSE_SPMV_CSR_ALG2 : CUSPARSE_SPMV_ALG_DEFAULT;
    cusparseStatus_t st = cusparseCreateCsr(&A, m, n, nnz, const_cast<int*>(rowptr), const_cast<int*>(colidx),
                                            const_cast<void*>(val), CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                                            CUSPARSE_INDEX_BASE_ZERO, vt);
    if (st == CUSPARSE_STATUS_SUCCESS) st = cusparseCreateDnVec(&X, nt ? n : m, const_cast<void*>(x), vt);
    if (st == CUSPARSE_STATUS_SUCCESS) st = cusparseCreateDnVec(&Y, nt ? m : n, y, vt);
    size_t bytes = 0;
    if (st == CUSPARSE_STATUS_SUCCESS) st = cusparseSpMV_bufferSize(h, op, alpha, A, X, beta, Y, vt, alg, &bytes);
    void* buf = nullptr;
    if (st == CUSPARSE_STATUS_SUCCESS) {
        buf = g_buf.get(bytes ? bytes : 16);
        if (!buf) st = CUSPARSE_STATUS_ALLOC_FAILED;
    }
    if (st == CUSPARSE_STATUS_SUCCESS) st = cusparseSpMV(h, op, alpha, A, X, beta, Y, vt, alg, buf);
    if (Y) cusparseDestroyDnVec(Y);
    if (X) cusparseDestroyDnVec(X);
    if (A) cusparseDestroySpMat(A);
    return st;
}

cusparseStatus_t csr2csc(cusparseHandle_t h, int m, int n, int nnz, const void* val, const int* rowptr,
                         const int* colidx, void* csc_val, int* csc_row, int* csc_colptr, cusparseAction_t action,
                         cusparseIndexBase_t base, cudaDataType vt)
{
    size_t bytes = 0;
    cusparseStatus_t st = cusparseCsr2cscEx2_bufferSize(h, m, n, nnz, val, rowptr, colidx, csc_val, csc_colptr,
                                                        csc_row, vt, action, base, CUSPARSE_CSR2CSC_ALG1, &bytes);
    if (st != CUSPARSE_STATUS_SUCCESS) return st;
    void* buf = g_buf.get(bytes ? bytes : 16);
    if (!buf) return CUSPARSE_STATUS_ALLOC_FAILED;
    return cusparseCsr2cscEx2(h, m, n, nnz, val, rowptr, colidx, csc_val, csc_colptr, csc_row, vt, action, base,
                              CUSPARSE_CSR2CSC_ALG1, buf);
}

[[noreturn]] void off_path(const char* name)
{
    std::fprintf(stderr, "reference build: %s is not available (no BLAS/LAPACK here; not on the solve path)\n", name);
    std::abort();
}

}  // namespace

cusparseStatus_t cusparseScsrmv(cusparseHandle_t h, cusparseOperation_t op, int m, int n, int nnz, const float* alpha,
                                const cusparseMatDescr_t, const float* val, const int* rowptr, const int* colidx,
                                const float* x, const float* beta, float* y)
{
    return spmv_csr(h, op, m, n, nnz, alpha, val, rowptr, colidx, x, beta, y, CUDA_R_32F);
}

cusparseStatus_t cusparseDcsrmv(cusparseHandle_t h, cusparseOperation_t op, int m, int n, int nnz,
                                const double* alpha, const cusparseMatDescr_t, const double* val, const int* rowptr,
                                const int* colidx, const double* x, const double* beta, double* y)
{
    return spmv_csr(h, op, m, n, nnz, alpha, val, rowptr, colidx, x, beta, y, CUDA_R_64F);
}

cusparseStatus_t cusparseScsr2csc(cusparseHandle_t h, int m, int n, int nnz, const float* val, const int* rowptr,
                                  const int* colidx, float* csc_val, int* csc_row, int* csc_colptr,
                                  cusparseAction_t action, cusparseIndexBase_t base)
{
    return csr2csc(h, m, n, nnz, val, rowptr, colidx, csc_val, csc_row, csc_colptr, action, base, CUDA_R_32F);
}

cusparseStatus_t cusparseDcsr2csc(cusparseHandle_t h, int m, int n, int nnz, const double* val, const int* rowptr,
                                  const int* colidx, double* csc_val, int* csc_row, int* csc_colptr,
                                  cusparseAction_t action, cusparseIndexBase_t base)
{
    return csr2csc(h, m, n, nnz, val, rowptr, colidx, csc_val, csc_row, csc_colptr, action, base, CUDA_R_64F);
}

extern "C" {
void cblas_saxpy(const int, const float, const float*, const int, float*, const int) { off_path("cblas_saxpy"); }
void cblas_daxpy(const int, const double, const double*, const int, double*, const int) { off_path("cblas_daxpy"); }
void cblas_sgemv(const enum CBLAS_ORDER, const enum CBLAS_TRANSPOSE, const int, const int, const float, const float*,
                 const int, const float*, const int, const float, float*, const int)
{
    off_path("cblas_sgemv");
}
void cblas_dgemv(const enum CBLAS_ORDER, const enum CBLAS_TRANSPOSE, const int, const int, const double,
                 const double*, const int, const double*, const int, const double, double*, const int)
{
    off_path("cblas_dgemv");
}
void cblas_sgemm(const enum CBLAS_ORDER, const enum CBLAS_TRANSPOSE, const enum CBLAS_TRANSPOSE, const int, const int,
                 const int, const float, const float*, const int, const float*, const int, const float, float*,
                 const int)
{
    off_path("cblas_sgemm");
}
void cblas_dgemm(const enum CBLAS_ORDER, const enum CBLAS_TRANSPOSE, const enum CBLAS_TRANSPOSE, const int, const int,
                 const int, const double, const double*, const int, const double*, const int, const double, double*,
                 const int)
{
    off_path("cblas_dgemm");
}
lapack_int LAPACKE_spotrf(int, char, lapack_int, float*, lapack_int) { off_path("LAPACKE_spotrf"); }
lapack_int LAPACKE_dpotrf(int, char, lapack_int, double*, lapack_int) { off_path("LAPACKE_dpotrf"); }
lapack_int LAPACKE_spotrs(int, char, lapack_int, lapack_int, const float*, lapack_int, float*, lapack_int)
{
    off_path("LAPACKE_spotrs");
}
lapack_int LAPACKE_dpotrs(int, char, lapack_int, lapack_int, const double*, lapack_int, double*, lapack_int)
{
    off_path("LAPACKE_dpotrs");
}
lapack_int LAPACKE_sposv(int, char, lapack_int, lapack_int, float*, lapack_int, float*, lapack_int)
{
    off_path("LAPACKE_sposv");
}
lapack_int LAPACKE_dposv(int, char, lapack_int, lapack_int, double*, lapack_int, double*, lapack_int)
{
    off_path("LAPACKE_dposv");
}
}
