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
//
// With the SELL-32 format (culipx_csr_set_format) the rows of at most 64
// entries are read from a slice-major copy instead: the same serial sum per
// row, with the warp's index and value loads contiguous (see Sell in spmv.h).
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

// SELL-32 product: thread (slice s, lane) sums row rows[32 s + lane] over
// the slots slice_off[s] + lane + 32 j in column order (col < 0: padding
// after the row's last entry), in batches of 8: a batch's gathers of x are
// issued together with the next batch's index and value loads (software
// pipelined), and the slot stream is read with evict-first loads so that x
// keeps its place in the caches.  128-thread CTAs (measured on the mixed
// matrix: 0.594 of HBM against 0.551 for the unpipelined 256-thread kernel).
template <class T>
__global__ void __launch_bounds__(128) k_sell_spmv(int nslices, const int* __restrict__ rows,
                                                   const long long* __restrict__ slice_off,
                                                   const int* __restrict__ slice_len, const int* __restrict__ col,
                                                   const T* __restrict__ val, const T* __restrict__ x,
                                                   T* __restrict__ y, T alpha, T beta)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int sl = t >> 5;
    if (sl >= nslices) return;
    const int row = __ldg(rows + t);
    const int len = __ldg(slice_len + sl);
    const int* cp = col + __ldg(slice_off + sl) + (t & 31);
    const T* vp = val + __ldg(slice_off + sl) + (t & 31);
    T acc = T(0);
    constexpr int B = kGatherBatch;
    int c[B];
    T v[B];
#pragma unroll
    for (int j = 0; j < B; ++j) {
        const bool ok = j < len;
        c[j] = ok ? __ldcs(cp + 32 * j) : -1;
        v[j] = ok ? __ldcs(vp + 32 * j) : T(0);
    }
    for (int jb = 0; jb < len; jb += B) {
        T xv[B];
#pragma unroll
        for (int j = 0; j < B; ++j) xv[j] = (c[j] >= 0) ? __ldg(x + c[j]) : T(0);
        // the next batch's indices and values, in flight with this batch's gathers
        int cn[B];
        T vn[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            const bool ok = jb + B + j < len;
            cn[j] = ok ? __ldcs(cp + 32 * (jb + B + j)) : -1;
            vn[j] = ok ? __ldcs(vp + 32 * (jb + B + j)) : T(0);
        }
#pragma unroll
        for (int j = 0; j < B; ++j)
            if (c[j] >= 0) acc = fma_rn(v[j], xv[j], acc);
#pragma unroll
        for (int j = 0; j < B; ++j) {
            c[j] = cn[j];
            v[j] = vn[j];
        }
    }
    if (row >= 0) y[row] = (beta == T(0)) ? alpha * acc : fma_rn(alpha, acc, beta * y[row]);
}

// the rows left out of the slices: a warp each, lane-strided partial sums
// and a fixed shfl_xor tree (k_csr_spmv_rows' long-row arithmetic)
template <class T>
__global__ void __launch_bounds__(256) k_long_rows(int nlong, const int* __restrict__ list,
                                                   const long long* __restrict__ off, const int* __restrict__ col,
                                                   const T* __restrict__ val, const T* __restrict__ x,
                                                   T* __restrict__ y, T alpha, T beta)
{
    const int lane = lane_id();
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nlong; w += nw) {
        const int row = __ldg(list + w);
        const long long a = __ldg(off + w), e = __ldg(off + w + 1);
        T part = T(0);
        for (long long k = a + lane; k < e; k += 32) part = fma_rn(__ldg(val + k), __ldg(x + __ldg(col + k)), part);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) y[row] = (beta == T(0)) ? alpha * part : fma_rn(alpha, part, beta * y[row]);
    }
}

template <class T>
__global__ void k_sell_gather(long long slots, const long long* __restrict__ map, const T* __restrict__ src,
                              T* __restrict__ dst)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < slots; i += stride) {
        const long long m = __ldg(map + i);
        dst[i] = (m >= 0) ? __ldg(src + m) : T(0);
    }
}

template <class T>
int launch_sell(Csr* A, const void* x, void* y, double alpha, double beta, cudaStream_t s)
{
    const Sell& S = A->sell;
    const T* xx = static_cast<const T*>(x);
    T* yy = static_cast<T*>(y);
    if (S.nslices > 0) {
        const long long threads = 32LL * S.nslices;
        k_sell_spmv<T><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(
            S.nslices, S.rows.as<int>(), S.slice_off.as<long long>(), S.slice_len.as<int>(), S.col.as<int>(),
            S.val.as<T>(), xx, yy, (T)alpha, (T)beta);
        CULIPX_TRY(launch_check("k_sell_spmv"));
    }
    if (S.nlong > 0) {
        A->h->launches += 1;
        const int blocks = std::min((S.nlong + 7) / 8, 148 * 8);
        k_long_rows<T><<<blocks, 256, 0, s>>>(S.nlong, S.long_rows.as<int>(), S.long_off.as<long long>(),
                                              S.col.as<int>(), S.val.as<T>(), xx, yy, (T)alpha, (T)beta);
        CULIPX_TRY(launch_check("k_long_rows"));
    }
    return CULIPX_OK;
}

}  // namespace

int csr_refresh_sell(Csr* A, cudaStream_t s)
{
    Sell& S = A->sell;
    if (!S.built || S.slots == 0) return CULIPX_OK;
    const int blocks = (int)std::min<long long>((S.slots + 255) / 256, 148 * 8);
    if (A->precision == CULIPX_F64)
        k_sell_gather<double><<<blocks, 256, 0, s>>>(S.slots, S.map.as<long long>(),
                                                      static_cast<const double*>(A->val), S.val.as<double>());
    else
        k_sell_gather<float><<<blocks, 256, 0, s>>>(S.slots, S.map.as<long long>(),
                                                     static_cast<const float*>(A->val), S.val.as<float>());
    A->h->launches += 1;
    return launch_check("k_sell_gather");
}

int csr_build_sell(Csr* A)
{
    Sell& S = A->sell;
    const int m = A->m;
    std::vector<int> rp(m + 1), ci(A->nnz);
    CULIPX_CUDA(cudaMemcpy(rp.data(), A->rowptr, (m + 1) * sizeof(int), cudaMemcpyDeviceToHost));
    if (A->nnz) CULIPX_CUDA(cudaMemcpy(ci.data(), A->colidx, A->nnz * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> shortr, longr;
    for (int r = 0; r < m; ++r) (rp[r + 1] - rp[r] > kSellMaxRow ? longr : shortr).push_back(r);
    // decreasing length inside each window (stable: ties keep row order)
    for (size_t w0 = 0; w0 < shortr.size(); w0 += kSellWindow) {
        const size_t w1 = std::min(shortr.size(), w0 + kSellWindow);
        std::stable_sort(shortr.begin() + w0, shortr.begin() + w1,
                         [&](int a, int b) { return rp[a + 1] - rp[a] > rp[b + 1] - rp[b]; });
    }
    const int ns = (int)((shortr.size() + 31) / 32);
    std::vector<int> rows((size_t)ns * 32, -1), slen(ns, 0);
    std::vector<long long> soff(ns + 1, 0);
    for (size_t i = 0; i < shortr.size(); ++i) rows[i] = shortr[i];
    for (int s = 0; s < ns; ++s) {
        int mx = 0;
        for (int l = 0; l < 32; ++l) {
            const int r = rows[(size_t)s * 32 + l];
            if (r >= 0) mx = std::max(mx, rp[r + 1] - rp[r]);
        }
        slen[s] = mx;
        soff[s + 1] = soff[s] + 32LL * mx;
    }
    std::vector<long long> loff(longr.size() + 1, soff[ns]);
    for (size_t i = 0; i < longr.size(); ++i) loff[i + 1] = loff[i] + (rp[longr[i] + 1] - rp[longr[i]]);
    const long long slots = loff.back();
    std::vector<int> col((size_t)std::max<long long>(slots, 1), -1);
    std::vector<long long> map((size_t)std::max<long long>(slots, 1), -1);
    for (size_t i = 0; i < longr.size(); ++i)
        for (int k = rp[longr[i]]; k < rp[longr[i] + 1]; ++k) {
            col[loff[i] + (k - rp[longr[i]])] = ci[k];
            map[loff[i] + (k - rp[longr[i]])] = k;
        }
    for (int s = 0; s < ns; ++s)
        for (int l = 0; l < 32; ++l) {
            const int r = rows[(size_t)s * 32 + l];
            if (r < 0) continue;
            for (int j = 0; j < rp[r + 1] - rp[r]; ++j) {
                const long long slot = soff[s] + 32LL * j + l;
                col[slot] = ci[rp[r] + j];
                map[slot] = rp[r] + j;
            }
        }
    S = Sell();
    const size_t vb = (A->precision == CULIPX_F64) ? 8 : 4;
    // (an empty list still gets a buffer: upload of 0 bytes allocates)
    CULIPX_TRY(S.rows.upload(A->h, rows.data(), rows.size() * sizeof(int)));
    CULIPX_TRY(S.slice_off.upload(A->h, soff.data(), soff.size() * sizeof(long long)));
    CULIPX_TRY(S.slice_len.upload(A->h, slen.data(), slen.size() * sizeof(int)));
    CULIPX_TRY(S.col.upload(A->h, col.data(), col.size() * sizeof(int)));
    CULIPX_TRY(S.map.upload(A->h, map.data(), map.size() * sizeof(long long)));
    CULIPX_TRY(S.val.alloc(A->h, col.size() * vb));
    CULIPX_TRY(S.long_rows.upload(A->h, longr.data(), longr.size() * sizeof(int)));
    CULIPX_TRY(S.long_off.upload(A->h, loff.data(), loff.size() * sizeof(long long)));
    S.nslices = ns;
    S.nrows = (int)shortr.size();
    S.nlong = (int)longr.size();
    S.slots = slots;
    S.built = true;
    CULIPX_TRY(csr_refresh_sell(A, A->h->stream));
    CULIPX_CUDA(cudaStreamSynchronize(A->h->stream));
    return CULIPX_OK;
}

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
    if (!transpose && A->sell.built) {
        if (A->precision == CULIPX_F64) return launch_sell<double>(A, x, y, alpha, beta, s);
        return launch_sell<float>(A, x, y, alpha, beta, s);
    }
    if (A->precision == CULIPX_F64) return launch<double>(rp, ci, v, m, avg, x, y, alpha, beta, s);
    return launch<float>(rp, ci, v, m, avg, x, y, alpha, beta, s);
}

}  // namespace culipx
