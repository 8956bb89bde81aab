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
//
// ||r|| is reduced in a fixed order (per-CTA partials summed on the host), so
// the step count is deterministic.
#include "sqmr.h"
#include "factor.h"
#include "kernels_common.cuh"

#include <cmath>
#include <vector>

namespace culipx {

namespace {

constexpr int kRT = 256;
constexpr int kRGrid = 148 * 4;

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

}  // namespace

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
    if (w->ref_part.bytes() < kRGrid * sizeof(double)) CULIPX_TRY(w->ref_part.alloc(h, kRGrid * sizeof(double)));
    double* r = w->ref_r.as<double>();
    double* d = w->ref_d.as<double>();
    double* part = w->ref_part.as<double>();
    std::vector<double> part_h(kRGrid);

    CULIPX_CUDA(cudaMemsetAsync(x, 0, vb, s));
    CULIPX_CUDA(cudaMemcpyAsync(r, b, vb, cudaMemcpyDeviceToDevice, s));
    double nb = 0.0, nr = 0.0;
    CULIPX_TRY(norm2(b, n, part, part_h.data(), s, h, &nb));
    int total = 0, k = 0;
    double rel = (nb > 0.0) ? 1.0 : 0.0;
    bool converged = rel <= tol;
    while (!converged && k < max_refine) {
        int its = 0;
        double res = 0.0;
        const int st = sqmr_solve(h, A, M, r, d, inner_tol, inner_max_it, &res, &its, w);
        if (st != CULIPX_OK && st != CULIPX_MAXIT) return st;
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
        converged = rel <= tol;
        if (!std::isfinite(rel)) return fail(CULIPX_BREAKDOWN, "culipx_sqmr_refine: non-finite residual");
    }
    if (relres) *relres = rel;
    if (iterations) *iterations = total;
    if (steps) *steps = k;
    return converged ? CULIPX_OK : CULIPX_MAXIT;
}

}  // namespace culipx
