// Symmetric / general permutation and scaling of a CSR matrix on the device:
// B = diag(1/r) P_r A P_c' diag(1/c) with rows and columns of B sorted, the
// operation the driver applies to K before the factorization
// (T_matrix_permute_scale, libs/la/sparse_la.impl.cuh:599-657, with
// k_inv_perm :586-595 and k_transform_coo :552-582; host_permute,
// apps/block_ildlt/block_ildlt_invariants.h:31-69).
//
// The reference converts to COO, rewrites every triplet and sorts all of
// them by (row, column) on each call.  Here the structure is computed once
// per pattern (a plan: B's row offsets and columns plus, for every entry of
// B, the entry of A it comes from); every call with new values is then one
// gather kernel.  B's row i is A's row p_r^-1(i) with its columns mapped by
// p_c and ranked within the row, so no global sort is needed; the result is
// the unique row/column-sorted CSR that the reference's sort produces.
#include "permute.h"
#include "kernels_common.cuh"

#include <algorithm>
#include <vector>

namespace culipx {

int exclusive_scan(int* d, int n, DeviceBuffer& tmp, culipx_handle_t* h, cudaStream_t s, int* launches);

namespace {

// new row i takes the length of old row inv_row[i]; row offsets outside
// [0, nnz] or decreasing set *bad and give the row no entries
__global__ void k_perm_lengths(int n, long long nnz, const int* __restrict__ rowptr, const int* __restrict__ inv_row,
                               int* __restrict__ len, int* __restrict__ bad)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        if (i == n) {
            len[n] = 0;
            continue;
        }
        const int o = inv_row[i];
        const int a = rowptr[o], b = rowptr[o + 1];
        const bool ok = a >= 0 && b >= a && b <= nnz;
        if (!ok) *bad = 1;
        len[i] = ok ? b - a : 0;
    }
}

// warp per new row: every entry's new column is ranked among its row's new
// columns (ties, i.e. duplicate entries, keep their order in A) and written
// to its sorted place together with its source position
__global__ void k_perm_fill(int n, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                            const int* __restrict__ inv_row, const int* __restrict__ col_perm,
                            const int* __restrict__ b_rowptr, int* __restrict__ b_col, int* __restrict__ src,
                            int* __restrict__ old_col_of, int* __restrict__ bad)
{
    const int lane = lane_id();
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const int o = inv_row[i];
        const int k0 = rowptr[o];
        const int len = b_rowptr[i + 1] - b_rowptr[i];  // 0 for a rejected row
        const int out0 = b_rowptr[i];
        // column indices outside [0, n) set *bad and map to column 0
        auto newcol = [&](int t) {
            const int c = colidx[k0 + t];
            if (c < 0 || c >= n) {
                *bad = 1;
                return col_perm[0];
            }
            return col_perm[c];
        };
        for (int j = lane; j < len; j += 32) {
            const int c = newcol(j);
            int rank = 0;
            for (int t = 0; t < len; ++t) {
                const int ct = newcol(t);
                rank += (ct < c) || (ct == c && t < j);
            }
            b_col[out0 + rank] = c;
            src[out0 + rank] = k0 + j;
            const int oc = colidx[k0 + j];
            old_col_of[out0 + rank] = (oc >= 0 && oc < n) ? oc : 0;
        }
    }
}

// B's values: val[src[k]] / (row scale * column scale), the scales taken at
// the old (row, column) when scale_before_match, else at the new ones
// (k_transform_coo); without scales the values are copied (v / 1 == v)
template <class T>
__global__ void k_perm_values(long long nnz, const int* __restrict__ src, const T* __restrict__ val,
                              const int* __restrict__ new_row_of, const int* __restrict__ new_col,
                              const int* __restrict__ old_row_of, const int* __restrict__ old_col_of,
                              const T* __restrict__ row_scale, const T* __restrict__ col_scale,
                              int scale_before_match, T* __restrict__ out)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz; k += stride) {
        const int s = src[k];
        const T v = val[s];
        if (!row_scale) {
            out[k] = v;
            continue;
        }
        const T sc = scale_before_match ? row_scale[old_row_of[k]] * col_scale[old_col_of[k]]
                                        : row_scale[new_row_of[k]] * col_scale[new_col[k]];
        out[k] = v / sc;
    }
}

__global__ void k_row_of(int n, const int* __restrict__ b_rowptr, const int* __restrict__ inv_row,
                         int* __restrict__ new_row_of, int* __restrict__ old_row_of)
{
    const int lane = lane_id();
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw)
        for (int k = b_rowptr[i] + lane; k < b_rowptr[i + 1]; k += 32) {
            new_row_of[k] = i;
            old_row_of[k] = inv_row[i];
        }
}

}  // namespace

int permute_plan_create(culipx_handle_t* h, int n, long long nnz, const int* d_rowptr, const int* d_colidx,
                        const int* h_row_perm, const int* h_col_perm, int perm_is_old_to_new, PermutePlan** out)
{
    if (n < 0 || nnz < 0 || nnz > 0x7fffffffLL || !d_rowptr || (nnz && !d_colidx) || !h_row_perm || !out)
        return fail(CULIPX_INVALID_ARG, "culipx_permute_plan_create: bad argument");
    if (!h_col_perm) h_col_perm = h_row_perm;
    // validate both permutations and build old -> new maps and their inverses on the host
    std::vector<int> rp(n), cp(n), inv_r(n, -1), inv_c(n, -1);  // old -> new, new -> old
    for (int pass = 0; pass < 2; ++pass) {
        const int* src = pass ? h_col_perm : h_row_perm;
        std::vector<int>& fwd = pass ? cp : rp;
        std::vector<int>& inv = pass ? inv_c : inv_r;
        std::vector<int> given(n);
        for (int i = 0; i < n; ++i) {
            if (src[i] < 0 || src[i] >= n) return fail(CULIPX_INVALID_ARG, "culipx_permute_plan_create: index out of range");
            given[i] = src[i];
        }
        if (perm_is_old_to_new) {
            fwd = given;
        } else {  // k_inv_perm: the given map is new -> old
            std::vector<int> seen(n, 0);
            for (int i = 0; i < n; ++i) {
                if (seen[given[i]]++) return fail(CULIPX_INVALID_ARG, "culipx_permute_plan_create: not a permutation");
                fwd[given[i]] = i;
            }
        }
        std::vector<int> seen(n, 0);
        for (int i = 0; i < n; ++i) {
            if (seen[fwd[i]]++) return fail(CULIPX_INVALID_ARG, "culipx_permute_plan_create: not a permutation");
            inv[fwd[i]] = i;
        }
    }
    auto* p = new PermutePlan();
    p->handle = h;
    p->n = n;
    p->nnz = nnz;
    int st = CULIPX_OK;
    auto up = [&](DeviceBuffer& b, const std::vector<int>& v) {
        if (st == CULIPX_OK) st = b.upload(h, v.data(), std::max<size_t>(v.size(), 1) * sizeof(int));
    };
    auto al = [&](DeviceBuffer& b, size_t bytes) {
        if (st == CULIPX_OK) st = b.alloc(h, bytes ? bytes : 16);
    };
    up(p->col_perm, cp);
    up(p->inv_row, inv_r);
    al(p->rowptr, (size_t)(n + 1) * sizeof(int));
    al(p->colidx, (size_t)nnz * sizeof(int));
    al(p->src, (size_t)nnz * sizeof(int));
    al(p->new_row_of, (size_t)nnz * sizeof(int));
    al(p->old_row_of, (size_t)nnz * sizeof(int));
    al(p->old_col_of, (size_t)nnz * sizeof(int));
    al(p->bad, sizeof(int));
    if (st != CULIPX_OK) {
        delete p;
        return st;
    }
    cudaStream_t s = h->stream;
    int launches = 0;
    const int grid = std::max(1, std::min((n + 256) / 256, 148 * 8));
    if (st == CULIPX_OK && cudaMemsetAsync(p->bad.get(), 0, sizeof(int), s) != cudaSuccess) st = launch_check("memset");
    k_perm_lengths<<<grid, 256, 0, s>>>(n, nnz, d_rowptr, p->inv_row.as<int>(), p->rowptr.as<int>(), p->bad.as<int>());
    st = launch_check("k_perm_lengths");
    if (st == CULIPX_OK) st = exclusive_scan(p->rowptr.as<int>(), n + 1, p->scan_tmp, h, s, &launches);
    if (st == CULIPX_OK && n > 0) {
        const int wgrid = std::max(1, std::min((n + 7) / 8, 148 * 16));
        k_perm_fill<<<wgrid, 256, 0, s>>>(n, d_rowptr, d_colidx, p->inv_row.as<int>(), p->col_perm.as<int>(),
                                          p->rowptr.as<int>(), p->colidx.as<int>(), p->src.as<int>(),
                                          p->old_col_of.as<int>(), p->bad.as<int>());
        k_row_of<<<wgrid, 256, 0, s>>>(n, p->rowptr.as<int>(), p->inv_row.as<int>(), p->new_row_of.as<int>(),
                                       p->old_row_of.as<int>());
        st = launch_check("k_perm_fill");
    }
    h->launches += launches + 3;
    int bad = 0, total = 0;
    if (st == CULIPX_OK && (cudaMemcpyAsync(&bad, p->bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                            cudaMemcpyAsync(&total, p->rowptr.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, s) !=
                                cudaSuccess ||
                            cudaStreamSynchronize(s) != cudaSuccess))
        st = launch_check("culipx_permute_create");
    if (st == CULIPX_OK && (bad || total != nnz))
        st = fail(CULIPX_INVALID_ARG, "culipx_permute_create: row offsets or column indices out of range");
    if (st != CULIPX_OK) {
        delete p;
        return st;
    }
    *out = p;
    return CULIPX_OK;
}

int permute_plan_apply(PermutePlan* p, int precision, const void* d_val, const void* d_row_scale,
                       const void* d_col_scale, int scale_before_match, void* d_out)
{
    if (!p || !d_val || !d_out) return fail(CULIPX_INVALID_ARG, "culipx_permute_apply: null argument");
    if ((d_row_scale == nullptr) != (d_col_scale == nullptr))
        return fail(CULIPX_INVALID_ARG, "culipx_permute_apply: give both scale vectors or neither");
    if (precision != CULIPX_F64 && precision != CULIPX_F32)
        return fail(CULIPX_INVALID_ARG, "culipx_permute_apply: bad precision");
    if (p->nnz == 0) return CULIPX_OK;
    cudaStream_t s = p->handle->stream;
    const int grid = (int)std::min<long long>((p->nnz + 255) / 256, 148 * 8);
    if (precision == CULIPX_F64)
        k_perm_values<double><<<grid, 256, 0, s>>>(
            p->nnz, p->src.as<int>(), static_cast<const double*>(d_val), p->new_row_of.as<int>(), p->colidx.as<int>(),
            p->old_row_of.as<int>(), p->old_col_of.as<int>(), static_cast<const double*>(d_row_scale), static_cast<const double*>(d_col_scale), scale_before_match,
            static_cast<double*>(d_out));
    else
        k_perm_values<float><<<grid, 256, 0, s>>>(
            p->nnz, p->src.as<int>(), static_cast<const float*>(d_val), p->new_row_of.as<int>(), p->colidx.as<int>(),
            p->old_row_of.as<int>(), p->old_col_of.as<int>(), static_cast<const float*>(d_row_scale), static_cast<const float*>(d_col_scale), scale_before_match,
            static_cast<float*>(d_out));
    p->handle->launches += 1;
    return launch_check("k_perm_values");
}

}  // namespace culipx
