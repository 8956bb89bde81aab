// Matrix-free KKT operators over the constraint matrix A (m x n CSR, FP64):
//
//   augmented  y = alpha [D x1 + A' x2 ; A x1 + (delta I)(ix) x2] + beta y
//              (x = [x1; x2], x1 of n, x2 of m)
//   normal     y = alpha (A D^-1 A' x + (delta I)(ix) x) + beta y   (m x m)
//
// They replace AugmentedMatrixSPMV<T> / NormalMatrixSPMV<T>
// (libs/la/spmv.cuh:75-149, spmv.impl.cuh:122-430) for FP64.  Two points
// differ from that code on purpose, both where it does not compute the
// operator its comments define: its augmented product adds A' x1 where A' x2
// belongs (spmv.impl.cuh:416-420), and its (delta I)(ix) term adds
// delta * x[i] at row ix[i] (k_add_app, helper_kernels.impl.cuh:361-374)
// where the shift of row ix[i] multiplies x[ix[i]]; here the shift is a
// dense per-row vector (delta at the rows listed in ix, 0 elsewhere) built
// once, so both products apply delta * x[ix[i]] at row ix[i].
//
// B200 layout: A and an explicit transpose A' (built once on the host, like
// the reference's explicit_At) as CSR; one fused launch for the augmented
// product (the n rows of D x1 + A' x2 and the m rows of A x1 + shift x2 in
// one grid, thread per row, gathers batched as in the standalone SpMV), two
// for the normal product (t = D^-1 A' x, then A t + shift x).
#include "operators.h"
#include "kernels_common.cuh"

#include <algorithm>
#include <vector>

namespace culipx {

namespace {

constexpr int kOpT = 256;
constexpr int kOpBatch = 8;

// sum_k val[k] x[col[k]] over [k0, k1), column order, from 0
__device__ __forceinline__ double row_dot(const int* __restrict__ col, const double* __restrict__ val, int k0, int k1,
                                          const double* __restrict__ x)
{
    double acc = 0.0;
    for (int kb = k0; kb < k1; kb += kOpBatch) {
        int c[kOpBatch];
        double v[kOpBatch], xv[kOpBatch];
#pragma unroll
        for (int j = 0; j < kOpBatch; ++j) {
            const bool ok = kb + j < k1;
            c[j] = ok ? __ldg(col + kb + j) : -1;
            v[j] = ok ? __ldg(val + kb + j) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < kOpBatch; ++j) xv[j] = (c[j] >= 0) ? __ldg(x + c[j]) : 0.0;
#pragma unroll
        for (int j = 0; j < kOpBatch; ++j)
            if (c[j] >= 0) acc = fma_rn(v[j], xv[j], acc);
    }
    return acc;
}

__device__ __forceinline__ void put(double* y, long long r, double v, double alpha, double beta)
{
    y[r] = (beta == 0.0) ? alpha * v : fma_rn(alpha, v, beta * y[r]);
}

__global__ void __launch_bounds__(kOpT) k_augmented(int m, int n, const int* __restrict__ rp,
                                                    const int* __restrict__ ci, const double* __restrict__ val,
                                                    const int* __restrict__ trp, const int* __restrict__ tci,
                                                    const double* __restrict__ tval, const double* __restrict__ d,
                                                    const double* __restrict__ shift, const double* __restrict__ x,
                                                    double* __restrict__ y, double alpha, double beta)
{
    const long long r = (long long)blockIdx.x * kOpT + threadIdx.x;
    if (r < n) {
        // D x1 + A' x2
        const double acc = row_dot(tci, tval, __ldg(trp + r), __ldg(trp + r + 1), x + n);
        put(y, r, fma_rn(__ldg(d + r), __ldg(x + r), acc), alpha, beta);
    } else if (r < (long long)n + m) {
        // A x1 + shift x2
        const long long i = r - n;
        const double acc = row_dot(ci, val, __ldg(rp + i), __ldg(rp + i + 1), x);
        put(y, r, fma_rn(__ldg(shift + i), __ldg(x + r), acc), alpha, beta);
    }
}

// t = D^-1 A' x (n rows of A')
__global__ void __launch_bounds__(kOpT) k_normal_t(int n, const int* __restrict__ trp, const int* __restrict__ tci,
                                                   const double* __restrict__ tval, const double* __restrict__ d,
                                                   const double* __restrict__ x, double* __restrict__ t)
{
    const long long j = (long long)blockIdx.x * kOpT + threadIdx.x;
    if (j < n) t[j] = row_dot(tci, tval, __ldg(trp + j), __ldg(trp + j + 1), x) / __ldg(d + j);
}

// y = alpha (A t + shift x) + beta y (m rows)
__global__ void __launch_bounds__(kOpT) k_normal_y(int m, const int* __restrict__ rp, const int* __restrict__ ci,
                                                   const double* __restrict__ val, const double* __restrict__ shift,
                                                   const double* __restrict__ t, const double* __restrict__ x,
                                                   double* __restrict__ y, double alpha, double beta)
{
    const long long i = (long long)blockIdx.x * kOpT + threadIdx.x;
    if (i < m) {
        const double acc = row_dot(ci, val, __ldg(rp + i), __ldg(rp + i + 1), t);
        put(y, i, fma_rn(__ldg(shift + i), __ldg(x + i), acc), alpha, beta);
    }
}

}  // namespace

int kkt_operator_create(culipx_handle_t* h, int kind, int m, int n, long long nnz, const int* d_rowptr,
                        const int* d_colidx, const double* d_val, const double* d_d, double delta, int num_ix,
                        const int* d_ix, KktOperator** out)
{
    if (!h || !out || (kind != 0 && kind != 1) || m < 0 || n < 0 || nnz < 0 || !d_rowptr ||
        (nnz > 0 && (!d_colidx || !d_val)) || (n > 0 && !d_d) || num_ix < 0 || (num_ix > 0 && !d_ix))
        return fail(CULIPX_INVALID_ARG, "culipx_kkt_operator_create: bad argument");
    KktOperator* op = new culipx_kkt_operator_t();
    op->h = h;
    op->kind = kind;
    op->m = m;
    op->n = n;
    op->nnz = nnz;
    op->rowptr = d_rowptr;
    op->colidx = d_colidx;
    op->val = d_val;
    op->d = d_d;
    // A' on the host, once (the reference's explicit_At)
    std::vector<int> rp(m + 1), ci(nnz);
    std::vector<double> vv(nnz);
    int st = CULIPX_OK;
    auto cp = [&](void* dst, const void* src, size_t bytes) {
        if (st == CULIPX_OK && bytes > 0 && cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
            st = fail(CULIPX_CUDA_ERROR, "culipx_kkt_operator_create: copy failed");
    };
    cp(rp.data(), d_rowptr, (size_t)(m + 1) * sizeof(int));
    cp(ci.data(), d_colidx, (size_t)nnz * sizeof(int));
    cp(vv.data(), d_val, (size_t)nnz * sizeof(double));
    std::vector<int> ix(num_ix);
    cp(ix.data(), d_ix, (size_t)num_ix * sizeof(int));
    if (st == CULIPX_OK && (rp[0] != 0 || rp[m] != nnz))
        st = fail(CULIPX_INVALID_ARG, "culipx_kkt_operator_create: rowptr does not span [0, nnz]");
    for (int r = 0; r < m && st == CULIPX_OK; ++r)
        if (rp[r + 1] < rp[r]) st = fail(CULIPX_INVALID_ARG, "culipx_kkt_operator_create: rowptr decreases");
    if (st == CULIPX_OK) {
        for (long long k = 0; k < nnz; ++k)
            if (ci[k] < 0 || ci[k] >= n) st = fail(CULIPX_INVALID_ARG, "culipx_kkt_operator_create: column out of range");
        for (int i = 0; i < num_ix && st == CULIPX_OK; ++i)
            if (ix[i] < 0 || ix[i] >= m) st = fail(CULIPX_INVALID_ARG, "culipx_kkt_operator_create: ix out of range");
    }
    if (st != CULIPX_OK) {
        delete static_cast<culipx_kkt_operator_t*>(op);
        return st;
    }
    std::vector<int> trp(n + 1, 0), tci(nnz);
    std::vector<double> tvv(nnz);
    for (long long k = 0; k < nnz; ++k) trp[ci[k] + 1]++;
    for (int c = 0; c < n; ++c) trp[c + 1] += trp[c];
    std::vector<int> pos(trp.begin(), trp.end() - 1);
    for (int r = 0; r < m; ++r)
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            const int q = pos[ci[k]]++;
            tci[q] = r;
            tvv[q] = vv[k];
        }
    std::vector<double> shift(std::max(m, 1), 0.0);
    for (int i = 0; i < num_ix; ++i) shift[ix[i]] = delta;
    st = op->t_rowptr.upload(h, trp.data(), trp.size() * sizeof(int));
    if (st == CULIPX_OK) st = op->t_colidx.upload(h, tci.data(), std::max<size_t>(tci.size(), 1) * sizeof(int));
    if (st == CULIPX_OK) st = op->t_val.upload(h, tvv.data(), std::max<size_t>(tvv.size(), 1) * sizeof(double));
    if (st == CULIPX_OK) st = op->shift.upload(h, shift.data(), shift.size() * sizeof(double));
    if (st == CULIPX_OK && kind == 1) st = op->tmp.alloc(h, (size_t)std::max(n, 1) * sizeof(double));
    if (st != CULIPX_OK) {
        delete static_cast<culipx_kkt_operator_t*>(op);
        return st;
    }
    *out = op;
    return CULIPX_OK;
}

int kkt_operator_multiply(KktOperator* op, const double* x, double* y, double alpha, double beta)
{
    if (!op || !x || !y) return fail(CULIPX_INVALID_ARG, "culipx_kkt_operator_multiply: null argument");
    cudaStream_t s = op->h->stream;
    if (op->kind == 0) {
        const long long rows = (long long)op->n + op->m;
        if (rows == 0) return CULIPX_OK;
        k_augmented<<<(unsigned)((rows + kOpT - 1) / kOpT), kOpT, 0, s>>>(
            op->m, op->n, op->rowptr, op->colidx, op->val, op->t_rowptr.as<int>(), op->t_colidx.as<int>(),
            op->t_val.as<double>(), op->d, op->shift.as<double>(), x, y, alpha, beta);
        op->h->launches += 1;
        return launch_check("k_augmented");
    }
    if (op->m == 0) return CULIPX_OK;
    if (op->n > 0) {
        k_normal_t<<<(op->n + kOpT - 1) / kOpT, kOpT, 0, s>>>(op->n, op->t_rowptr.as<int>(), op->t_colidx.as<int>(),
                                                             op->t_val.as<double>(), op->d, x, op->tmp.as<double>());
        op->h->launches += 1;
        CULIPX_TRY(launch_check("k_normal_t"));
    }
    k_normal_y<<<(op->m + kOpT - 1) / kOpT, kOpT, 0, s>>>(op->m, op->rowptr, op->colidx, op->val,
                                                         op->shift.as<double>(), op->tmp.as<double>(), x, y, alpha,
                                                         beta);
    op->h->launches += 1;
    return launch_check("k_normal_y");
}

}  // namespace culipx
