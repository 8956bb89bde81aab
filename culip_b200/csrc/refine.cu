// FP64 iterative refinement around the preconditioned SQMR solve.
//
// No counterpart in the reference (its SQMR<T> solves once in the factor's
// precision T, libs/la/iterative_solvers/sqmr.impl.cuh:109-355).  With an
// FP32 factor the preconditioner applies run in single precision; the true
// residual r = b - K x, the correction update x += d and all of SQMR's
// scalars and vectors stay FP64:
//
//   x = 0, r = b
//   repeat: stop if ||r|| <= tol ||b|| or after max_refine corrections
//           d = SQMR(K, M, r, inner_tol, inner_max_it); x += d; r = b - K x
//           keep x as the best iterate if ||r|| is the smallest so far;
//           stop (CULIPX_STALLED) after kRefinePatience corrections in a row
//           that did not lower the smallest ||r||
//   return the best iterate and its residual
//
// When the inner solve does not converge (a poor FP32 factor, an inner cap
// too low for the system) a correction can raise the residual; an unguarded
// loop would then return a worse x than it had, or diverge.  A single
// non-improving correction is still followed (the next one often recovers),
// two in a row end the loop.  The step count counts corrections computed,
// the iterations every inner SQMR iteration.
//
// ||r|| is reduced in a fixed order (per-CTA partials summed on the host), so
// the step count is deterministic.
#include "sqmr.h"
#include "factor.h"
#include "kernels_common.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace culipx {

namespace {

constexpr int kRT = 256;
constexpr int kRGrid = 148 * 4;
constexpr int kRefinePatience = 2;  // non-improving corrections in a row that end the loop

__global__ void k_sumsq(const double* __restrict__ v, int n, double* __restrict__ part)
{
    __shared__ double sh[kRT / 32];
    double s = 0.0;
    for (int g = blockIdx.x * kRT + threadIdx.x; g < n; g += gridDim.x * kRT) s = fma_rn(v[g], v[g], s);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < kRT / 32; ++i) t += sh[i];
        part[blockIdx.x] = t;
    }
}

__global__ void k_add(double* __restrict__ x, const double* __restrict__ d, int n)
{
    for (int g = blockIdx.x * kRT + threadIdx.x; g < n; g += gridDim.x * kRT) x[g] += d[g];
}

int norm2(const double* v, int n, double* part_d, double* part_h, cudaStream_t s, culipx_handle_t* h, double* out)
{
    k_sumsq<<<kRGrid, kRT, 0, s>>>(v, n, part_d);
    h->launches += 1;
    CULIPX_TRY(launch_check("k_sumsq"));
    CULIPX_CUDA(cudaMemcpyAsync(part_h, part_d, kRGrid * sizeof(double), cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaStreamSynchronize(s));
    double t = 0.0;
    for (int i = 0; i < kRGrid; ++i) t += part_h[i];
    *out = std::sqrt(t);
    return CULIPX_OK;
}

// per system k: sum of squares of v over rows row_off[k] .. row_off[k+1]
// (one CTA per system, fixed order)
__global__ void k_seg_sumsq(const double* __restrict__ v, const int* __restrict__ row_off, int num,
                            double* __restrict__ out)
{
    __shared__ double sh[kRT / 32];
    for (int k = blockIdx.x; k < num; k += gridDim.x) {
        double s = 0.0;
        for (int g = row_off[k] + threadIdx.x; g < row_off[k + 1]; g += kRT) s = fma_rn(v[g], v[g], s);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int i = 0; i < kRT / 32; ++i) t += sh[i];
            out[k] = t;
        }
        __syncthreads();
    }
}

// rows of the systems with keep[k] == 0 set to zero
__global__ void k_seg_mask(double* __restrict__ v, const int* __restrict__ row_off, int num,
                           const int* __restrict__ keep)
{
    for (int k = blockIdx.x; k < num; k += gridDim.x)
        if (!keep[k])
            for (int g = row_off[k] + threadIdx.x; g < row_off[k + 1]; g += kRT) v[g] = 0.0;
}

// x = c on the rows of the systems with take[k] != 0
__global__ void k_seg_take(double* __restrict__ x, const double* __restrict__ c, const int* __restrict__ row_off,
                           int num, const int* __restrict__ take)
{
    for (int k = blockIdx.x; k < num; k += gridDim.x)
        if (take[k])
            for (int g = row_off[k] + threadIdx.x; g < row_off[k + 1]; g += kRT) x[g] = c[g];
}

int seg_norms(const double* v, Batch* bt, double* d_out, std::vector<double>& h_out, cudaStream_t s)
{
    k_seg_sumsq<<<std::min(bt->num, 148 * 8), kRT, 0, s>>>(v, bt->d_row_off.as<int>(), bt->num, d_out);
    bt->h->launches += 1;
    CULIPX_TRY(launch_check("k_seg_sumsq"));
    CULIPX_CUDA(cudaMemcpyAsync(h_out.data(), d_out, bt->num * sizeof(double), cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaStreamSynchronize(s));
    for (double& t : h_out) t = std::sqrt(t);
    return CULIPX_OK;
}

}  // namespace

// Batched refinement: the loop above per system, all systems' corrections in
// one batched SQMR launch per step; systems that reached tol, stalled or broke
// down get a zero right-hand side (their correction is zero) and stop
// counting steps.
int batch_sqmr_refine(Batch* bt, Csr* A, Factor* M, const double* b, double* x, double tol, double inner_tol,
                      int inner_max_it, int max_refine, double* h_relres, int* h_its, int* h_steps, int* h_status,
                      Sqmr* w)
{
    if (!bt || !A || !M || !b || !x || !w) return fail(CULIPX_INVALID_ARG, "culipx_batch_sqmr_refine: null argument");
    if (!(tol >= 0.0) || !(inner_tol >= 0.0) || inner_max_it < 0 || max_refine < 0)
        return fail(CULIPX_INVALID_ARG, "culipx_batch_sqmr_refine: bad tolerance or limit");
    culipx_handle_t* h = bt->h;
    const int n = A->m, num = bt->num;
    cudaStream_t s = h->stream;
    const size_t vb = (size_t)n * sizeof(double);
    if (w->ref_r.bytes() < vb + 16) CULIPX_TRY(w->ref_r.alloc(h, vb + 16));
    if (w->ref_d.bytes() < vb + 16) CULIPX_TRY(w->ref_d.alloc(h, vb + 16));
    if (w->ref_best.bytes() < vb + 16) CULIPX_TRY(w->ref_best.alloc(h, vb + 16));
    const size_t pb = std::max<size_t>((size_t)num * (sizeof(double) + 2 * sizeof(int)), kRGrid * sizeof(double));
    if (w->ref_part.bytes() < pb) CULIPX_TRY(w->ref_part.alloc(h, pb));
    double* r = w->ref_r.as<double>();
    double* d = w->ref_d.as<double>();
    double* best = w->ref_best.as<double>();
    double* sums = w->ref_part.as<double>();
    int* keep_d = reinterpret_cast<int*>(sums + num);
    int* take_d = keep_d + num;
    std::vector<double> nb(num), nr(num);
    std::vector<int> keep(num), take(num), its(num, 0), steps(num, 0), st(num, CULIPX_OK), it_k(num), st_k(num);
    std::vector<int> fails(num, 0);
    CULIPX_CUDA(cudaMemsetAsync(x, 0, vb, s));
    CULIPX_CUDA(cudaMemsetAsync(best, 0, vb, s));
    CULIPX_CUDA(cudaMemcpyAsync(r, b, vb, cudaMemcpyDeviceToDevice, s));
    CULIPX_TRY(seg_norms(b, bt, sums, nb, s));
    std::vector<double> rel(num), best_rel(num);
    for (int k = 0; k < num; ++k) best_rel[k] = rel[k] = nb[k] > 0.0 ? 1.0 : 0.0;
    auto seg_copy = [&](double* dst, const double* src, const std::vector<int>& flag) -> int {
        CULIPX_CUDA(cudaMemcpyAsync(take_d, flag.data(), num * sizeof(int), cudaMemcpyHostToDevice, s));
        k_seg_take<<<std::min(num, 148 * 8), kRT, 0, s>>>(dst, src, bt->d_row_off.as<int>(), num, take_d);
        h->launches += 1;
        return launch_check("k_seg_take");
    };
    for (int step = 0; step < max_refine; ++step) {
        int active = 0;
        for (int k = 0; k < num; ++k) {
            keep[k] = rel[k] > tol && st[k] == CULIPX_OK;
            active += keep[k];
        }
        if (!active) break;
        // r holds b - K x of every active system; zero elsewhere
        CULIPX_CUDA(cudaMemcpyAsync(keep_d, keep.data(), num * sizeof(int), cudaMemcpyHostToDevice, s));
        k_seg_mask<<<std::min(num, 148 * 8), kRT, 0, s>>>(r, bt->d_row_off.as<int>(), num, keep_d);
        h->launches += 1;
        CULIPX_TRY(launch_check("k_seg_mask"));
        CULIPX_TRY(batch_sqmr_solve(bt, A, M, r, d, inner_tol, inner_max_it, nullptr, it_k.data(), st_k.data(), w));
        k_add<<<kRGrid, kRT, 0, s>>>(x, d, n);
        h->launches += 1;
        CULIPX_TRY(launch_check("k_add"));
        CULIPX_CUDA(cudaMemcpyAsync(r, b, vb, cudaMemcpyDeviceToDevice, s));
        CULIPX_TRY(csr_spmv(A, x, r, -1.0, 1.0, 0, s));
        h->launches += 1;
        CULIPX_TRY(seg_norms(r, bt, sums, nr, s));
        int taken = 0;
        for (int k = 0; k < num; ++k) {
            take[k] = 0;
            if (!keep[k]) continue;
            its[k] += it_k[k];
            steps[k] += 1;
            rel[k] = nr[k] / nb[k];
            if (st_k[k] == CULIPX_BREAKDOWN || !std::isfinite(rel[k])) {
                st[k] = CULIPX_BREAKDOWN;
            } else if (rel[k] < best_rel[k]) {
                best_rel[k] = rel[k];
                fails[k] = 0;
                take[k] = 1;
                ++taken;
            } else if (++fails[k] >= kRefinePatience) {
                st[k] = CULIPX_STALLED;
            }
        }
        if (taken) CULIPX_TRY(seg_copy(best, x, take));
    }
    // every system ends on its best iterate
    int back = 0;
    for (int k = 0; k < num; ++k) {
        take[k] = best_rel[k] < rel[k] || !std::isfinite(rel[k]);
        back += take[k];
    }
    if (back) CULIPX_TRY(seg_copy(x, best, take));
    CULIPX_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < num; ++k) {
        if (st[k] == CULIPX_OK) st[k] = best_rel[k] <= tol ? CULIPX_OK : CULIPX_MAXIT;
        if (h_relres) h_relres[k] = best_rel[k];
        if (h_its) h_its[k] = its[k];
        if (h_steps) h_steps[k] = steps[k];
        if (h_status) h_status[k] = st[k];
    }
    return CULIPX_OK;
}

int sqmr_refine(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, double inner_tol,
                int inner_max_it, int max_refine, double* relres, int* iterations, int* steps, Sqmr* w)
{
    if (!A || !M || !b || !x || !w) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_refine: null argument");
    if (A->precision != CULIPX_F64 || A->m != A->n)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_refine: A must be square FP64");
    if (!M->computed || M->pat->n != A->m)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_refine: preconditioner not computed or wrong size");
    if (!(tol >= 0.0) || !(inner_tol >= 0.0) || inner_max_it < 0 || max_refine < 0)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_refine: bad tolerance or limit");
    const int n = A->m;
    cudaStream_t s = h->stream;
    const size_t vb = (size_t)n * sizeof(double);
    if (w->ref_r.bytes() < vb + 16) CULIPX_TRY(w->ref_r.alloc(h, vb + 16));
    if (w->ref_d.bytes() < vb + 16) CULIPX_TRY(w->ref_d.alloc(h, vb + 16));
    if (w->ref_best.bytes() < vb + 16) CULIPX_TRY(w->ref_best.alloc(h, vb + 16));
    if (w->ref_part.bytes() < kRGrid * sizeof(double)) CULIPX_TRY(w->ref_part.alloc(h, kRGrid * sizeof(double)));
    double* r = w->ref_r.as<double>();
    double* d = w->ref_d.as<double>();
    double* best = w->ref_best.as<double>();
    double* part = w->ref_part.as<double>();
    std::vector<double> part_h(kRGrid);

    CULIPX_CUDA(cudaMemsetAsync(x, 0, vb, s));
    CULIPX_CUDA(cudaMemsetAsync(best, 0, vb, s));
    CULIPX_CUDA(cudaMemcpyAsync(r, b, vb, cudaMemcpyDeviceToDevice, s));
    double nb = 0.0, nr = 0.0;
    CULIPX_TRY(norm2(b, n, part, part_h.data(), s, h, &nb));
    int total = 0, k = 0, fails = 0, status = CULIPX_OK;
    double rel = (nb > 0.0) ? 1.0 : 0.0, best_rel = rel;
    while (rel > tol && k < max_refine) {
        int its = 0;
        double res = 0.0;
        const int st = sqmr_solve(h, A, M, r, d, inner_tol, inner_max_it, &res, &its, w);
        if (st != CULIPX_OK && st != CULIPX_MAXIT) {
            status = st;
            break;
        }
        total += its;
        k += 1;
        k_add<<<kRGrid, kRT, 0, s>>>(x, d, n);
        h->launches += 1;
        CULIPX_TRY(launch_check("k_add"));
        // r = b - K x in FP64
        CULIPX_CUDA(cudaMemcpyAsync(r, b, vb, cudaMemcpyDeviceToDevice, s));
        CULIPX_TRY(csr_spmv(A, x, r, -1.0, 1.0, 0, s));
        h->launches += 1;
        CULIPX_TRY(norm2(r, n, part, part_h.data(), s, h, &nr));
        rel = nr / nb;
        if (!std::isfinite(rel)) {
            status = fail(CULIPX_BREAKDOWN, "culipx_sqmr_refine: non-finite residual");
            break;
        }
        if (rel < best_rel) {
            best_rel = rel;
            fails = 0;
            CULIPX_CUDA(cudaMemcpyAsync(best, x, vb, cudaMemcpyDeviceToDevice, s));
        } else if (++fails >= kRefinePatience) {
            status = CULIPX_STALLED;
            break;
        }
    }
    if (best_rel < rel || !std::isfinite(rel)) CULIPX_CUDA(cudaMemcpyAsync(x, best, vb, cudaMemcpyDeviceToDevice, s));
    CULIPX_CUDA(cudaStreamSynchronize(s));
    if (relres) *relres = best_rel;
    if (iterations) *iterations = total;
    if (steps) *steps = k;
    if (status != CULIPX_OK) return status;
    return best_rel <= tol ? CULIPX_OK : CULIPX_MAXIT;
}

// The same loop for several right-hand sides (column-major n x nrhs): per
// column its own residual, step count and stopping test; each step solves the
// corrections of the columns still above tol together (sqmr_solve_multi, up
// to four per launch, every launch reading the factor and K once for all).
int sqmr_refine_multi(culipx_handle_t* h, Csr* A, Factor* M, int nrhs, const double* B, double* X, double tol,
                      double inner_tol, int inner_max_it, int max_refine, double* h_relres, int* h_its, int* h_steps,
                      int* h_status, Sqmr* w)
{
    if (!A || !M || !B || !X || !w || nrhs < 1) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_refine_multi: bad argument");
    if (A->precision != CULIPX_F64 || A->m != A->n)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_refine_multi: A must be square FP64");
    if (!M->computed || M->pat->n != A->m)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_refine_multi: preconditioner not computed or wrong size");
    if (!(tol >= 0.0) || !(inner_tol >= 0.0) || inner_max_it < 0 || max_refine < 0)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_refine_multi: bad tolerance or limit");
    const size_t n = A->m;
    cudaStream_t s = h->stream;
    const size_t vb = n * sizeof(double);
    if (w->ref_r.bytes() < vb * nrhs + 16) CULIPX_TRY(w->ref_r.alloc(h, vb * nrhs + 16));
    if (w->ref_d.bytes() < vb * nrhs + 16) CULIPX_TRY(w->ref_d.alloc(h, vb * nrhs + 16));
    if (w->ref_best.bytes() < vb * nrhs + 16) CULIPX_TRY(w->ref_best.alloc(h, vb * nrhs + 16));
    if (w->ref_part.bytes() < kRGrid * sizeof(double)) CULIPX_TRY(w->ref_part.alloc(h, kRGrid * sizeof(double)));
    double* R = w->ref_r.as<double>();  // residuals of the active columns, packed in column order
    double* D = w->ref_d.as<double>();  // their corrections
    double* Best = w->ref_best.as<double>();  // per column its best iterate
    double* part = w->ref_part.as<double>();
    std::vector<double> part_h(kRGrid), nb(nrhs), rel(nrhs), best_rel(nrhs);
    std::vector<int> its(nrhs, 0), steps(nrhs, 0), st(nrhs, CULIPX_OK), it_k(nrhs), st_k(nrhs), fails(nrhs, 0);
    std::vector<int> act, pos(nrhs, -1);  // pos[j]: column of R holding column j's residual

    CULIPX_CUDA(cudaMemsetAsync(X, 0, vb * nrhs, s));
    CULIPX_CUDA(cudaMemsetAsync(Best, 0, vb * nrhs, s));
    for (int j = 0; j < nrhs; ++j) {
        CULIPX_TRY(norm2(B + j * n, (int)n, part, part_h.data(), s, h, &nb[j]));
        best_rel[j] = rel[j] = nb[j] > 0.0 ? 1.0 : 0.0;
        // x = 0: the first residual is b
        CULIPX_CUDA(cudaMemcpyAsync(R + j * n, B + j * n, vb, cudaMemcpyDeviceToDevice, s));
        pos[j] = j;
    }
    for (int step = 0; step < max_refine; ++step) {
        act.clear();
        for (int j = 0; j < nrhs; ++j)
            if (rel[j] > tol && st[j] == CULIPX_OK) act.push_back(j);
        if (act.empty()) break;
        // pack: positions only move left, so copying in increasing order is safe
        for (int a = 0; a < (int)act.size(); ++a) {
            const int j = act[a];
            if (pos[j] != a)
                CULIPX_CUDA(cudaMemcpyAsync(R + a * n, R + pos[j] * n, vb, cudaMemcpyDeviceToDevice, s));
            pos[j] = a;
        }
        const int na = (int)act.size();
        CULIPX_TRY(sqmr_solve_multi(h, A, M, na, R, D, inner_tol, inner_max_it, nullptr, it_k.data(), st_k.data(), w));
        for (int a = 0; a < na; ++a) {
            const int j = act[a];
            double* x = X + j * n;
            double* r = R + a * n;
            k_add<<<kRGrid, kRT, 0, s>>>(x, D + a * n, (int)n);
            h->launches += 1;
            CULIPX_TRY(launch_check("k_add"));
            CULIPX_CUDA(cudaMemcpyAsync(r, B + j * n, vb, cudaMemcpyDeviceToDevice, s));
            CULIPX_TRY(csr_spmv(A, x, r, -1.0, 1.0, 0, s));
            h->launches += 1;
            double nr = 0.0;
            CULIPX_TRY(norm2(r, (int)n, part, part_h.data(), s, h, &nr));
            its[j] += it_k[a];
            steps[j] += 1;
            rel[j] = nr / nb[j];
            if (st_k[a] == CULIPX_BREAKDOWN || !std::isfinite(rel[j])) {
                st[j] = CULIPX_BREAKDOWN;
            } else if (rel[j] < best_rel[j]) {
                best_rel[j] = rel[j];
                fails[j] = 0;
                CULIPX_CUDA(cudaMemcpyAsync(Best + j * n, x, vb, cudaMemcpyDeviceToDevice, s));
            } else if (++fails[j] >= kRefinePatience) {
                st[j] = CULIPX_STALLED;
            }
        }
    }
    for (int j = 0; j < nrhs; ++j)
        if (best_rel[j] < rel[j] || !std::isfinite(rel[j]))
            CULIPX_CUDA(cudaMemcpyAsync(X + j * n, Best + j * n, vb, cudaMemcpyDeviceToDevice, s));
    CULIPX_CUDA(cudaStreamSynchronize(s));
    for (int j = 0; j < nrhs; ++j) {
        if (st[j] == CULIPX_OK) st[j] = best_rel[j] <= tol ? CULIPX_OK : CULIPX_MAXIT;
        if (h_relres) h_relres[j] = best_rel[j];
        if (h_its) h_its[j] = its[j];
        if (h_steps) h_steps[j] = steps[j];
        if (h_status) h_status[j] = st[j];
    }
    return CULIPX_OK;
}

}  // namespace culipx
