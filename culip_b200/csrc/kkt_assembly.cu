// KKT assembly for an interior-point iteration.
//
//   K = [[ diag(d) + delta I   A' ]
//        [ A             -gamma I ]],   d_j = s_j / x_j  (or d given),
//
// the augmented system of an LP interior-point step (the barrier Hessian
// X^-1 S, primal / dual regularization delta, gamma), as full symmetric CSR
// with sorted columns and an explicit diagonal: the matrix the block-iLDL'
// path factors and SQMR multiplies.  It is the explicit form of the operator
// AugmentedMatrixSPMV<T> applies (libs/la/spmv.cuh:104-149, K = [D A'; A
// (delta I)(ix)]) with the dual shift applied to every row.  In culip the IPM
// caller forms K on the host every iteration; here K's structure is planned
// once per pattern of A (host counting sort of A's columns, stable in row
// order, so A' rows come out sorted) and each iteration's values are one
// gather on the device:
//   row j < n:      (j, j) then (j, n + i) for A_ij != 0, i increasing
//   row n + i:      (n + i, j) for A_ij != 0, j increasing, then (n + i, n + i)
// src[e] is the entry of A that K's entry e copies, or -1 - r for the
// diagonal of row r.  The gather reads src and the A values once and writes K
// once: nnz_K (8 + 8) + 8 nnz_A + 16 n bytes (HBM-bound).
#include "kkt_assembly.h"
#include "kernels_common.cuh"

#include <algorithm>
#include <vector>

namespace culipx {

namespace {

template <class TO>
__global__ void k_kkt_values(long long nnz_k, int n, const long long* __restrict__ src,
                             const double* __restrict__ aval, const double* __restrict__ x,
                             const double* __restrict__ s, const double* __restrict__ d, double delta, double gamma,
                             TO* __restrict__ kval)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz_k; e += stride) {
        const long long q = __ldg(src + e);
        double v;
        if (q >= 0) {
            v = __ldg(aval + q);
        } else {
            const int r = (int)(-1 - q);
            if (r < n) v = (d ? __ldg(d + r) : __ldg(s + r) / __ldg(x + r)) + delta;
            else v = -gamma;
        }
        kval[e] = (TO)v;
    }
}

}  // namespace

int kkt_assembly_create(culipx_handle_t* h, int m, int n, long long nnz_a, const int* d_rowptr, const int* d_colidx,
                        KktAssembly** out)
{
    if (!h || !out || m < 0 || n < 0 || nnz_a < 0 || (nnz_a > 0 && (!d_rowptr || !d_colidx)) || (m > 0 && !d_rowptr))
        return fail(CULIPX_INVALID_ARG, "culipx_kkt_assembly_create: bad argument");
    if ((long long)n + m > 0x7fffffffLL || 2 * nnz_a + n + m > 0x7fffffffLL)
        return fail(CULIPX_NOT_SUPPORTED, "culipx_kkt_assembly_create: K beyond int32 indices");
    std::vector<int> rp(m + 1, 0), ci(nnz_a);
    if (m > 0)
        CULIPX_CUDA(cudaMemcpyAsync(rp.data(), d_rowptr, (m + 1) * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    if (nnz_a > 0)
        CULIPX_CUDA(cudaMemcpyAsync(ci.data(), d_colidx, nnz_a * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CULIPX_CUDA(cudaStreamSynchronize(h->stream));
    if (rp[0] != 0 || rp[m] != nnz_a)
        return fail(CULIPX_INVALID_ARG, "culipx_kkt_assembly_create: rowptr does not span nnz entries");
    std::vector<int> cnt(n + 1, 0);
    for (int i = 0; i < m; ++i) {
        if (rp[i + 1] < rp[i]) return fail(CULIPX_INVALID_ARG, "culipx_kkt_assembly_create: rowptr decreases at %d", i);
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            if (j < 0 || j >= n) return fail(CULIPX_INVALID_ARG, "culipx_kkt_assembly_create: column %d out of range", j);
            if (k > rp[i] && j <= ci[k - 1])
                return fail(CULIPX_INVALID_ARG, "culipx_kkt_assembly_create: row %d not sorted / has duplicates", i);
            ++cnt[j + 1];
        }
    }
    for (int j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
    // A' by a counting sort that keeps row order: column j's entries, rows increasing
    std::vector<int> t_row(nnz_a);
    std::vector<long long> t_src(nnz_a);
    {
        std::vector<int> pos(cnt.begin(), cnt.end() - 1);
        for (int i = 0; i < m; ++i)
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                const int p = pos[ci[k]]++;
                t_row[p] = i;
                t_src[p] = k;
            }
    }
    const int N = n + m;
    const long long nnz_k = 2 * nnz_a + N;
    std::vector<int> krp(N + 1), kci(nnz_k);
    std::vector<long long> ksrc(nnz_k);
    long long e = 0;
    for (int j = 0; j < n; ++j) {
        krp[j] = (int)e;
        kci[e] = j;
        ksrc[e++] = -1 - (long long)j;
        for (int p = cnt[j]; p < cnt[j + 1]; ++p) {
            kci[e] = n + t_row[p];
            ksrc[e++] = t_src[p];
        }
    }
    for (int i = 0; i < m; ++i) {
        krp[n + i] = (int)e;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            kci[e] = ci[k];
            ksrc[e++] = k;
        }
        kci[e] = n + i;
        ksrc[e++] = -1 - (long long)(n + i);
    }
    krp[N] = (int)e;
    auto* K = new KktAssembly();
    K->handle = h;
    K->m = m;
    K->n = n;
    K->nnz_a = nnz_a;
    K->nnz_k = nnz_k;
    int st = K->rowptr.upload(h, krp.data(), krp.size() * sizeof(int));
    if (st == CULIPX_OK) st = K->colidx.upload(h, kci.data(), std::max<size_t>(1, kci.size()) * sizeof(int));
    if (st == CULIPX_OK) st = K->src.upload(h, ksrc.data(), std::max<size_t>(1, ksrc.size()) * sizeof(long long));
    if (st != CULIPX_OK) {
        delete K;
        return st;
    }
    *out = K;
    return CULIPX_OK;
}

int kkt_assembly_values(KktAssembly* K, const double* d_aval, const double* d_x, const double* d_s,
                        const double* d_d, double delta, double gamma, int precision, void* d_kval)
{
    if (!K || !d_kval || (K->nnz_a > 0 && !d_aval) || (K->n > 0 && !d_d && (!d_x || !d_s)))
        return fail(CULIPX_INVALID_ARG, "culipx_kkt_assemble: null argument");
    if (precision != CULIPX_F64 && precision != CULIPX_F32)
        return fail(CULIPX_INVALID_ARG, "culipx_kkt_assemble: bad precision");
    cudaStream_t s = K->handle->stream;
    const long long blocks = std::min<long long>((K->nnz_k + 255) / 256, 148LL * 8);
    if (blocks <= 0) return CULIPX_OK;
    if (precision == CULIPX_F64)
        k_kkt_values<double><<<(unsigned)blocks, 256, 0, s>>>(K->nnz_k, K->n, K->src.as<long long>(), d_aval, d_x, d_s,
                                                              d_d, delta, gamma, static_cast<double*>(d_kval));
    else
        k_kkt_values<float><<<(unsigned)blocks, 256, 0, s>>>(K->nnz_k, K->n, K->src.as<long long>(), d_aval, d_x, d_s,
                                                             d_d, delta, gamma, static_cast<float*>(d_kval));
    K->handle->launches += 1;
    return launch_check("k_kkt_values");
}

}  // namespace culipx
