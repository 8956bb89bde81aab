// Imported L D L' preconditioner (ImportLDUPreconditioner<T>,
// libs/la/preconditioner/import_ldu_preconditioner.impl.cuh; the reference's
// tests/la/test_sqmr.cc:192-293 run SQMR with it on exported factors):
//
//   solve_left   x = L^-1 P' (S .* b)      (forward substitution)
//   solve_middle x = D^-1 b                (1x1 / 2x2 pivots, tri / is_piv)
//   solve_right  x = S .* P (L'^-1 b)      (backward substitution)
//
// L is any lower-triangular CSR (its diagonal, 1 where absent, divides).
// Both substitutions are level-scheduled: the rows of one level depend only on
// earlier levels, one launch per level, a thread per row.  Each row sums its
// terms in the order of the CPU restatement's loops (forward: L's row order;
// backward: the columns of L from the last row up, i.e. L' rows in descending
// column order), so the applies match it bit for bit.
#include "ldu.h"
#include "kernels_common.cuh"

#include <algorithm>
#include <vector>

namespace culipx {

namespace {

constexpr int kLT = 256;

// t2[g] = b[perm[g]] * scale[perm[g]]
__global__ void k_ldu_left_in(int n, const int* __restrict__ perm, const double* __restrict__ scale,
                              const double* __restrict__ b, double* __restrict__ t2)
{
    const int g = blockIdx.x * kLT + threadIdx.x;
    if (g < n) {
        const int q = __ldg(perm + g);
        t2[g] = b[q] * __ldg(scale + q);
    }
}

// x[perm[g]] = t1[g] * scale[perm[g]]
__global__ void k_ldu_right_out(int n, const int* __restrict__ perm, const double* __restrict__ scale,
                                const double* __restrict__ t1, double* __restrict__ x)
{
    const int g = blockIdx.x * kLT + threadIdx.x;
    if (g < n) {
        const int q = __ldg(perm + g);
        x[q] = t1[g] * __ldg(scale + q);
    }
}

// one level of a substitution: x[i] = (rhs[i] - sum_k val[k] x[col[k]]) / diag[i]
// over the stored entries of row i (lower: entries on or right of the
// diagonal are skipped, as the restatement's forward sweep does)
__global__ void k_ldu_level(const int* __restrict__ rows, int r0, int r1, const int* __restrict__ rp,
                            const int* __restrict__ ci, const double* __restrict__ val,
                            const double* __restrict__ diag, const double* __restrict__ rhs, double* __restrict__ x,
                            int lower)
{
    const int t = r0 + blockIdx.x * kLT + threadIdx.x;
    if (t >= r1) return;
    const int i = __ldg(rows + t);
    double acc = rhs[i];
    for (int k = __ldg(rp + i); k < __ldg(rp + i + 1); ++k) {
        const int j = __ldg(ci + k);
        if (!lower || j < i) acc = fma_rn(-__ldg(val + k), x[j], acc);
    }
    x[i] = acc / __ldg(diag + i);
}

// D^-1 (k_solve_D, helper_kernels.impl.cuh:720-774) from b into x
__global__ void k_ldu_d(int n, const double* __restrict__ tri, const int* __restrict__ is_piv,
                        const double* __restrict__ b, double* __restrict__ x)
{
    const int g = blockIdx.x * kLT + threadIdx.x;
    if (g >= n) return;
    const int this_piv = __ldg(is_piv + g);
    const int next_piv = (g < n - 1) ? __ldg(is_piv + g + 1) : 1;
    const double p11 = __ldg(tri + 3 * g + 1), p12 = __ldg(tri + 3 * g + 2);
    const double p22 = !next_piv ? __ldg(tri + 3 * (g + 1) + 1) : 1.0;
    const double r1 = b[g], r2 = (g < n - 1) ? b[g + 1] : 0.0;
    const double gr = sqrt(fma_rn(p11, p11, p12 * p12));
    const double gc = p11 / gr, gs = p12 / gr;
    double g1 = fma_rn(gc, r1, gs * r2), g2 = fma_rn(gc, r2, -(gs * r1));
    const double tp12 = fma_rn(gc, p12, gs * p22), tp22 = fma_rn(gc, p22, -(gs * p12));
    g2 = g2 / tp22;
    g1 = fma_rn(-tp12, g2, g1) / gr;
    if (this_piv) x[g] = g1;
    if (!next_piv) x[g + 1] = g2;
    if (g == 0 && !this_piv) x[0] = r1;  // no pivot starts at row 0: the copy of b stands
}

// rows of each level, levels in order, from per-row levels
void level_lists(const std::vector<int>& lev, std::vector<int>& rows, std::vector<int>& off)
{
    const int nl = lev.empty() ? 0 : *std::max_element(lev.begin(), lev.end()) + 1;
    off.assign(nl + 1, 0);
    for (int l : lev) off[l + 1]++;
    for (int l = 0; l < nl; ++l) off[l + 1] += off[l];
    std::vector<int> pos(off.begin(), off.end() - 1);
    rows.assign(lev.size(), 0);
    for (size_t i = 0; i < lev.size(); ++i) rows[pos[lev[i]]++] = (int)i;
}

}  // namespace

int ldu_create(culipx_handle_t* h, int n, const int* d_rowptr, const int* d_colidx, const double* d_val,
               const double* d_tri, const int* d_is_piv, const int* d_perm, const double* d_scale, Ldu** out)
{
    if (!h || !out || n < 1 || !d_rowptr || !d_colidx || !d_val || !d_tri || !d_is_piv || !d_perm || !d_scale)
        return fail(CULIPX_INVALID_ARG, "culipx_ldu_create: bad argument");
    std::vector<int> rp(n + 1);
    CULIPX_CUDA(cudaMemcpy(rp.data(), d_rowptr, (size_t)(n + 1) * sizeof(int), cudaMemcpyDeviceToHost));
    if (rp[0] != 0) return fail(CULIPX_INVALID_ARG, "culipx_ldu_create: rowptr[0] != 0");
    for (int i = 0; i < n; ++i)
        if (rp[i + 1] < rp[i]) return fail(CULIPX_INVALID_ARG, "culipx_ldu_create: rowptr decreases");
    const long long nnz = rp[n];
    std::vector<int> ci(std::max(nnz, 1LL)), perm(n);
    std::vector<double> val(std::max(nnz, 1LL));
    CULIPX_CUDA(cudaMemcpy(ci.data(), d_colidx, (size_t)nnz * sizeof(int), cudaMemcpyDeviceToHost));
    CULIPX_CUDA(cudaMemcpy(val.data(), d_val, (size_t)nnz * sizeof(double), cudaMemcpyDeviceToHost));
    CULIPX_CUDA(cudaMemcpy(perm.data(), d_perm, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<char> seen(n, 0);
    for (int g = 0; g < n; ++g) {
        if (perm[g] < 0 || perm[g] >= n || seen[perm[g]])
            return fail(CULIPX_INVALID_ARG, "culipx_ldu_create: perm is not a permutation");
        seen[perm[g]] = 1;
    }
    std::vector<double> diag(n, 1.0);
    std::vector<int> lev_f(n, 0), cnt(n, 0);
    for (int i = 0; i < n; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            if (j < 0 || j > i) return fail(CULIPX_INVALID_ARG, "culipx_ldu_create: L is not lower triangular");
            if (j == i) {
                diag[i] = val[k];  // the last stored diagonal entry, as the restatement
            } else {
                lev_f[i] = std::max(lev_f[i], lev_f[j] + 1);
                cnt[j]++;
            }
        }
    // L' rows: row j lists (i, L_ij), i > j, in descending i
    std::vector<int> trp(n + 1, 0);
    for (int j = 0; j < n; ++j) trp[j + 1] = trp[j] + cnt[j];
    std::vector<int> tci(std::max(trp[n], 1)), pos(trp.begin(), trp.end() - 1);
    std::vector<double> tval(std::max(trp[n], 1));
    for (int i = n - 1; i >= 0; --i)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            if (j < i) {
                tci[pos[j]] = i;
                tval[pos[j]++] = val[k];
            }
        }
    std::vector<int> lev_b(n, 0);
    for (int j = n - 1; j >= 0; --j)
        for (int k = trp[j]; k < trp[j + 1]; ++k) lev_b[j] = std::max(lev_b[j], lev_b[tci[k]] + 1);
    auto* P = new culipx_ldu_t();
    P->h = h;
    P->n = n;
    level_lists(lev_f, P->fwd_rows_h, P->fwd_off);
    level_lists(lev_b, P->bwd_rows_h, P->bwd_off);
    int st = P->rp.upload(h, rp.data(), rp.size() * sizeof(int));
    if (st == CULIPX_OK) st = P->ci.upload(h, ci.data(), ci.size() * sizeof(int));
    if (st == CULIPX_OK) st = P->val.upload(h, val.data(), val.size() * sizeof(double));
    if (st == CULIPX_OK) st = P->diag.upload(h, diag.data(), diag.size() * sizeof(double));
    if (st == CULIPX_OK) st = P->trp.upload(h, trp.data(), trp.size() * sizeof(int));
    if (st == CULIPX_OK) st = P->tci.upload(h, tci.data(), tci.size() * sizeof(int));
    if (st == CULIPX_OK) st = P->tval.upload(h, tval.data(), tval.size() * sizeof(double));
    if (st == CULIPX_OK) st = P->fwd_rows.upload(h, P->fwd_rows_h.data(), P->fwd_rows_h.size() * sizeof(int));
    if (st == CULIPX_OK) st = P->bwd_rows.upload(h, P->bwd_rows_h.data(), P->bwd_rows_h.size() * sizeof(int));
    if (st == CULIPX_OK) st = P->tri.alloc(h, (size_t)3 * n * sizeof(double));
    if (st == CULIPX_OK) st = P->is_piv.alloc(h, (size_t)n * sizeof(int));
    if (st == CULIPX_OK) st = P->perm.alloc(h, (size_t)n * sizeof(int));
    if (st == CULIPX_OK) st = P->scale.alloc(h, (size_t)n * sizeof(double));
    if (st == CULIPX_OK) st = P->t1.alloc(h, (size_t)n * sizeof(double));
    if (st == CULIPX_OK) st = P->t2.alloc(h, (size_t)n * sizeof(double));
    if (st == CULIPX_OK) {
        const bool ok =
            cudaMemcpy(P->tri.get(), d_tri, (size_t)3 * n * sizeof(double), cudaMemcpyDeviceToDevice) == cudaSuccess &&
            cudaMemcpy(P->is_piv.get(), d_is_piv, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice) == cudaSuccess &&
            cudaMemcpy(P->perm.get(), d_perm, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice) == cudaSuccess &&
            cudaMemcpy(P->scale.get(), d_scale, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice) == cudaSuccess;
        if (!ok) st = fail(CULIPX_CUDA_ERROR, "culipx_ldu_create: copy failed");
    }
    if (st != CULIPX_OK) {
        delete P;
        return st;
    }
    *out = P;
    return CULIPX_OK;
}

int ldu_apply(Ldu* P, int stage, const double* b, double* x, cudaStream_t s)
{
    if (!P || !b || !x) return fail(CULIPX_INVALID_ARG, "culipx_ldu_apply: null argument");
    const int n = P->n;
    const int grid = (n + kLT - 1) / kLT;
    if (stage == CULIPX_MIDDLE) {
        k_ldu_d<<<grid, kLT, 0, s>>>(n, P->tri.as<double>(), P->is_piv.as<int>(), b, x);
        P->h->launches += 1;
        return launch_check("k_ldu_d");
    }
    if (stage == CULIPX_LEFT) {
        k_ldu_left_in<<<grid, kLT, 0, s>>>(n, P->perm.as<int>(), P->scale.as<double>(), b, P->t2.as<double>());
        P->h->launches += 1;
        for (size_t l = 0; l + 1 < P->fwd_off.size(); ++l) {
            const int r0 = P->fwd_off[l], r1 = P->fwd_off[l + 1];
            k_ldu_level<<<(r1 - r0 + kLT - 1) / kLT, kLT, 0, s>>>(P->fwd_rows.as<int>(), r0, r1, P->rp.as<int>(),
                                                                 P->ci.as<int>(), P->val.as<double>(),
                                                                 P->diag.as<double>(), P->t2.as<double>(), x, 1);
            P->h->launches += 1;
        }
        return launch_check("k_ldu_level (forward)");
    }
    if (stage == CULIPX_RIGHT) {
        for (size_t l = 0; l + 1 < P->bwd_off.size(); ++l) {
            const int r0 = P->bwd_off[l], r1 = P->bwd_off[l + 1];
            k_ldu_level<<<(r1 - r0 + kLT - 1) / kLT, kLT, 0, s>>>(P->bwd_rows.as<int>(), r0, r1, P->trp.as<int>(),
                                                                 P->tci.as<int>(), P->tval.as<double>(),
                                                                 P->diag.as<double>(), b, P->t1.as<double>(), 0);
            P->h->launches += 1;
        }
        k_ldu_right_out<<<grid, kLT, 0, s>>>(n, P->perm.as<int>(), P->scale.as<double>(), P->t1.as<double>(), x);
        P->h->launches += 1;
        return launch_check("k_ldu_level (backward)");
    }
    return fail(CULIPX_INVALID_ARG, "culipx_ldu_apply: bad stage %d", stage);
}

}  // namespace culipx
