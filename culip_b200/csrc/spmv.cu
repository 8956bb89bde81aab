// CSR sparse matrix-vector product, y = alpha op(A) x + beta y.
//
// Replaces CSRMatrixSPMV<T>::multiply -> T_csrmv -> legacy cusparse{S,D}csrmv
// (libs/la/spmv.impl.cuh:78-113, libs/la/sparse_la_instances.cu:129-217).
//
// Short rows (average up to 16 nonzeros, the KKT case): a thread owns a
// row and sums it in column order (acc = fma(v, x, acc) from 0, the order of
// a serial CSR loop, so the result is bit-identical to it), loading its
// entries in batches of 8 with all 8 x gathers in flight before the fmas.
// Rows of more than 64 nonzeros are summed by their whole warp instead
// (lane-strided partial sums, fixed shfl_xor tree).  Measured on B200 this
// beats shared-memory staging of the rows' range (warp-wide or through TMA
// bulk copies): the kernel is bound by the L1TEX pipe, not by DRAM.
// Longer rows: a group of L lanes (L = 16 or 32) owns a row and reduces with a fixed
// shfl_xor tree (bit-reproducible run to run).  The transpose
// product uses an explicit transposed copy, as CSRMatrixSPMV does when
// explicit_At is set (spmv.impl.cuh:34-41).
#include "spmv.h"
#include "kernels_common.cuh"

#include <algorithm>
#include <vector>

namespace culipx {

namespace {

template <class T, int L>
__global__ void __launch_bounds__(256) k_csr_spmv(int m, const int* __restrict__ rowptr,
                                                  const int* __restrict__ colidx, const T* __restrict__ val,
                                                  const T* __restrict__ x, T* __restrict__ y, T alpha, T beta)
{
    constexpr int kRowsPerWarp = 32 / L;
    const int lane = lane_id();
    const int sub = lane % L;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * kRowsPerWarp; base < m; base += nwarps * kRowsPerWarp) {
        const long long row = base + lane / L;
        T acc = T(0);
        if (row < m) {
            const int e = __ldg(rowptr + row + 1);
            for (int k = __ldg(rowptr + row) + sub; k < e; k += L)
                acc = fma_rn(__ldg(val + k), __ldg(x + __ldg(colidx + k)), acc);
        }
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (row < m && sub == 0) y[row] = (beta == T(0)) ? alpha * acc : fma_rn(alpha, acc, beta * y[row]);
    }
}

// rows up to kLongRow nonzeros: one thread, entries in batches of 8 (all 8
// x gathers issued before the 8 fmas); longer rows: the whole warp
constexpr int kLongRow = 64;
constexpr int kGatherBatch = 8;

template <class T>
__global__ void __launch_bounds__(256) k_csr_spmv_rows(int m, const int* __restrict__ rowptr,
                                                       const int* __restrict__ colidx, const T* __restrict__ val,
                                                       const T* __restrict__ x, T* __restrict__ y, T alpha, T beta)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = lane_id();
    int rs = 0, re = 0;
    if (row < m) {
        rs = __ldg(rowptr + row);
        re = __ldg(rowptr + row + 1);
    }
    const bool lng = re - rs > kLongRow;
    T acc = T(0);
    if (!lng) {
        for (int kb = rs; kb < re; kb += kGatherBatch) {
            T v[kGatherBatch], xv[kGatherBatch];
            int c[kGatherBatch];
#pragma unroll
            for (int j = 0; j < kGatherBatch; ++j) {
                const bool ok = kb + j < re;
                c[j] = ok ? __ldg(colidx + kb + j) : -1;
                v[j] = ok ? __ldg(val + kb + j) : T(0);
            }
#pragma unroll
            for (int j = 0; j < kGatherBatch; ++j) xv[j] = (c[j] >= 0) ? __ldg(x + c[j]) : T(0);
#pragma unroll
            for (int j = 0; j < kGatherBatch; ++j)
                if (c[j] >= 0) acc = fma_rn(v[j], xv[j], acc);
        }
    }
    // long rows of this warp, one at a time with all lanes (fixed shfl_xor tree)
    unsigned todo = __ballot_sync(0xffffffffu, lng);
    while (todo) {
        const int src = __ffs(todo) - 1;
        todo &= todo - 1;
        const int a = __shfl_sync(0xffffffffu, rs, src), e = __shfl_sync(0xffffffffu, re, src);
        T part = T(0);
        for (int k = a + lane; k < e; k += 32) part = fma_rn(__ldg(val + k), __ldg(x + __ldg(colidx + k)), part);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == src) acc = part;
    }
    if (row < m) y[row] = (beta == T(0)) ? alpha * acc : fma_rn(alpha, acc, beta * y[row]);
}

template <class T>
int launch(const int* rowptr, const int* colidx, const void* val, int m, double avg, const void* x, void* y,
           double alpha, double beta, cudaStream_t s)
{
    const T* v = static_cast<const T*>(val);
    const T* xx = static_cast<const T*>(x);
    T* yy = static_cast<T*>(y);
    if (avg <= 16.0) {
        k_csr_spmv_rows<T><<<(m + 255) / 256, 256, 0, s>>>(m, rowptr, colidx, v, xx, yy, (T)alpha, (T)beta);
    } else {
        // 8 warps per block, 32 / L rows per warp
        auto grid = [&](int L) {
            const long long blocks = ((long long)m * L + 255) / 256;
            return (int)std::min<long long>(blocks, 148LL * 16);
        };
        if (avg <= 24.0)
            k_csr_spmv<T, 16><<<grid(16), 256, 0, s>>>(m, rowptr, colidx, v, xx, yy, (T)alpha, (T)beta);
        else
            k_csr_spmv<T, 32><<<grid(32), 256, 0, s>>>(m, rowptr, colidx, v, xx, yy, (T)alpha, (T)beta);
    }
    return launch_check("k_csr_spmv");
}

}  // namespace

int csr_build_transpose(Csr* A)
{
    // one-time host transpose of the borrowed device arrays
    const size_t vb = (A->precision == CULIPX_F64) ? 8 : 4;
    std::vector<int> rp(A->m + 1), ci(A->nnz);
    std::vector<unsigned char> vv(A->nnz * vb);
    CULIPX_CUDA(cudaMemcpy(rp.data(), A->rowptr, (A->m + 1) * sizeof(int), cudaMemcpyDeviceToHost));
    CULIPX_CUDA(cudaMemcpy(ci.data(), A->colidx, A->nnz * sizeof(int), cudaMemcpyDeviceToHost));
    CULIPX_CUDA(cudaMemcpy(vv.data(), A->val, A->nnz * vb, cudaMemcpyDeviceToHost));
    std::vector<int> trp(A->n + 1, 0), tci(A->nnz);
    std::vector<unsigned char> tvv(A->nnz * vb);
    for (long long k = 0; k < A->nnz; ++k) trp[ci[k] + 1]++;
    for (int c = 0; c < A->n; ++c) trp[c + 1] += trp[c];
    std::vector<int> pos(trp.begin(), trp.end() - 1);
    for (int r = 0; r < A->m; ++r)
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            const int d = pos[ci[k]]++;
            tci[d] = r;
            std::copy(&vv[k * vb], &vv[k * vb] + vb, &tvv[d * vb]);
        }
    CULIPX_TRY(A->t_rowptr.upload(A->h, trp.data(), trp.size() * sizeof(int)));
    CULIPX_TRY(A->t_colidx.upload(A->h, tci.data(), tci.size() * sizeof(int)));
    CULIPX_TRY(A->t_val.upload(A->h, tvv.data(), tvv.size()));
    A->has_t = true;
    return CULIPX_OK;
}

int csr_spmv(Csr* A, const void* x, void* y, double alpha, double beta, int transpose, cudaStream_t s)
{
    if (!A || !x || !y) return fail(CULIPX_INVALID_ARG, "culipx_spmv: null argument");
    const int* rp = A->rowptr;
    const int* ci = A->colidx;
    const void* v = A->val;
    int m = A->m;
    if (transpose) {
        if (!A->has_t) CULIPX_TRY(csr_build_transpose(A));
        rp = A->t_rowptr.as<int>();
        ci = A->t_colidx.as<int>();
        v = A->t_val.get();
        m = A->n;
    }
    if (m == 0) return CULIPX_OK;
    const double avg = (double)A->nnz / (double)std::max(m, 1);
    A->h->launches += 1;
    if (A->precision == CULIPX_F64) return launch<double>(rp, ci, v, m, avg, x, y, alpha, beta, s);
    return launch<float>(rp, ci, v, m, avg, x, y, alpha, beta, s);
}

}  // namespace culipx
