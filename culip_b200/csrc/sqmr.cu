// Simplified QMR for symmetric indefinite K with the split preconditioner
// M = (P U') D (U P') (SQMR<T>::solve, libs/la/iterative_solvers/sqmr.impl.cuh:109-355).
//
// The reference issues ~35 launches per iteration: cuBLAS nrm2/dot/axpy/scal
// plus ~22 single-thread scalar kernels (k_set_*_scalar, k_sym_ortho,
// k_sqmr_test), and synchronizes the host every 4 iterations.  Here one
// iteration is six fused kernels around the preconditioned product:
//   K1  alpha = v'(D^-1 Av) / v'(D^-1 v)
//   K2  v+ = Av - alpha v - beta v-, ||v+||
//   K3  v+ /= delta, w+ = eta delta D^-1 v+, tmp = D^-1 v+
//       Av = U'^-1 P' K P U^-1 tmp          (sweeps + SpMV)
//   K4  beta+ = w'Av / w'v, then every scalar of the QMR recurrence (eta,
//       ||A|| estimate, the two old Givens rotations, k_sym_ortho, tau, rho)
//   K5  w+ /= beta+, p = (v - beta_rr p- - eps p--) / rho, x += tau p, ||x||,
//       gamma, the convergence test and the reference's lagged check.
// Reductions are deterministic: a fixed grid, a fixed shuffle tree per CTA,
// and the last CTA (ticket) summing the per-CTA partials in index order and
// then running the scalar recurrence in FP64 on the device.
// The reference's check protocol is kept exactly: test flags are snapshot at
// iterations = 3 (mod 4) and acted on at the next iteration, so iteration
// counts match the reference's.
#include "sqmr.h"
#include "factor.h"
#include "ldu.h"
#include "kernels_common.cuh"

#include <cmath>
#include <functional>

namespace culipx {

namespace {

constexpr int kThreads = 256;
constexpr int kGrid = 148 * 2;

struct Scal {
    double alpha, beta[3], delta[3], c[3], s[3];
    double norm_A, epsilon, beta_rot, beta_rot_rot, alpha_rot, tau, rho, gamma, norm_pb, norm_x, eta;
    double inv_delta, inv_beta, inv_rho, inv_pb;
    double tol;
    int it, max_it, test0, test1, snap0, snap1, done, iters, breakdown;
    unsigned int ticket;
};

__host__ __device__ __forceinline__ int acc3(int r) { return (r % 3) + ((r < 0) ? 3 : 0); }

// block reduction of NV doubles; thread 0 gets the sums
template <int NV>
__device__ void block_sum(double (&v)[NV], double (*sh)[32])
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][w] = v[k];
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = (lane < (int)(blockDim.x >> 5)) ? sh[k][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            v[k] = t;
        }
    }
}

// writes this CTA's partials; returns true in the last CTA, whose thread 0
// then holds the totals (summed in CTA order) in v
template <int NV>
__device__ bool grid_sum(double (&v)[NV], double* partials, Scal* S)
{
    __shared__ double sh[NV][32];
    __shared__ bool last;
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partials[k * kGrid + blockIdx.x] = v[k];
        __threadfence();
        const unsigned t = atomicAdd(&S->ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // the last CTA reduces the partials with all its threads: thread t sums
    // partials t, t + blockDim, ... (fixed order), then a fixed shuffle tree
    double w[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t += __ldcg(partials + k * kGrid + b);
        w[k] = t;
    }
    block_sum<NV>(w, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] = w[k];
        S->ticket = 0;
    }
    return true;
}

// D^-1 for the pivot starting at row g (k_solve_D semantics); in[g+1] is read
// only when g starts a 2x2 pivot or g + 1 < n
__device__ __forceinline__ void dsolve_pair(const double* tri, const int* is_piv, int n, int g, double r1, double r2,
                                            double& g1, double& g2, bool& two)
{
    const int next_piv = (g < n - 1) ? is_piv[g + 1] : 1;
    two = !next_piv;
    const double p11 = tri[3 * (size_t)g + 1], p12 = tri[3 * (size_t)g + 2];
    const double p22 = two ? tri[3 * (size_t)(g + 1) + 1] : 1.0;
    const double gr = sqrt(fma_rn(p11, p11, p12 * p12));
    const double gc = p11 / gr, gs = p12 / gr;
    g1 = fma_rn(gc, r1, gs * r2);
    g2 = fma_rn(gc, r2, -(gs * r1));
    const double tp12 = fma_rn(gc, p12, gs * p22);
    const double tp22 = fma_rn(gc, p22, -(gs * p12));
    g2 = g2 / tp22;
    g1 = fma_rn(-tp12, g2, g1) / gr;
}

struct DOp {  // D as seen by the SQMR kernels (null tri: identity)
    const double* tri;
    const int* is_piv;
};

using PrecFn = std::function<int(int stage, const double* in, double* out)>;

#define SQMR_GUARD \
    if (S->done) return;

__global__ void __launch_bounds__(kThreads) k_init_norm(const double* v0, int n, double* partials, Scal* S)
{
    double acc[1] = {0.0};
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x)
        acc[0] = fma_rn(v0[g], v0[g], acc[0]);
    if (grid_sum<1>(acc, partials, S) && threadIdx.x == 0) {
        S->norm_pb = sqrt(acc[0]);
        S->inv_pb = 1.0 / S->norm_pb;
        S->gamma = S->norm_pb;
        if (!isfinite(S->inv_pb)) { S->breakdown = 1; S->done = 1; }
    }
}

// v0 *= 1/||v0||, w0 = D^-1 v0 (eta applied in k_init_eta), tmp = D^-1 v0, ||w0||^2
__global__ void __launch_bounds__(kThreads) k_init_vw(double* v0, double* w0, double* tmp, DOp D, int n,
                                                      double* partials, Scal* S)
{
    SQMR_GUARD
    const double sc = S->inv_pb;
    double acc[1] = {0.0};
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        if (!D.tri) {
            const double v = v0[g] * sc;
            v0[g] = v;
            w0[g] = v;
            tmp[g] = v;
            acc[0] = fma_rn(v, v, acc[0]);
            continue;
        }
        if (!D.is_piv[g]) continue;
        const double r1 = v0[g] * sc;
        const double r2 = (g < n - 1) ? v0[g + 1] * sc : 0.0;
        double g1, g2;
        bool two;
        dsolve_pair(D.tri, D.is_piv, n, g, r1, r2, g1, g2, two);
        v0[g] = r1;
        w0[g] = g1;
        tmp[g] = g1;
        acc[0] = fma_rn(g1, g1, acc[0]);
        if (two) {
            v0[g + 1] = r2;
            w0[g + 1] = g2;
            tmp[g + 1] = g2;
            acc[0] = fma_rn(g2, g2, acc[0]);
        }
    }
    if (grid_sum<1>(acc, partials, S) && threadIdx.x == 0) {
        S->eta = 1.0 / sqrt(acc[0]);
        if (!isfinite(S->eta)) { S->breakdown = 1; S->done = 1; }
    }
}

__global__ void k_init_eta(double* w0, int n, Scal* S)
{
    SQMR_GUARD
    const double e = S->eta;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) w0[g] *= e;
}

// K1: alpha
__global__ void __launch_bounds__(kThreads) k_alpha(const double* vk, const double* Av, DOp D, int n,
                                                    double* partials, Scal* S)
{
    SQMR_GUARD
    double acc[2] = {0.0, 0.0};
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        if (!D.tri) {
            acc[0] = fma_rn(vk[g], Av[g], acc[0]);
            acc[1] = fma_rn(vk[g], vk[g], acc[1]);
            continue;
        }
        if (!D.is_piv[g]) continue;
        const bool has_next = g < n - 1;
        double a1, a2, b1, b2;
        bool two;
        dsolve_pair(D.tri, D.is_piv, n, g, Av[g], has_next ? Av[g + 1] : 0.0, a1, a2, two);
        dsolve_pair(D.tri, D.is_piv, n, g, vk[g], has_next ? vk[g + 1] : 0.0, b1, b2, two);
        acc[0] = fma_rn(vk[g], a1, acc[0]);
        acc[1] = fma_rn(vk[g], b1, acc[1]);
        if (two) {
            acc[0] = fma_rn(vk[g + 1], a2, acc[0]);
            acc[1] = fma_rn(vk[g + 1], b2, acc[1]);
        }
    }
    if (grid_sum<2>(acc, partials, S) && threadIdx.x == 0) {
        S->alpha = acc[0] / acc[1];
        if (!isfinite(S->alpha)) { S->breakdown = 1; S->done = 1; }
    }
}

// K2: v+ = Av - alpha vk - beta_k vkm1, ||v+||
__global__ void __launch_bounds__(kThreads) k_vnext(const double* Av, const double* vk, const double* vkm1,
                                                    double* vk1, int n, int k0, int k1, double* partials, Scal* S)
{
    SQMR_GUARD
    const double na = -S->alpha, nb = -S->beta[k0];
    double acc[1] = {0.0};
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        double v = Av[g];
        v = fma_rn(na, vk[g], v);
        v = fma_rn(nb, vkm1[g], v);
        vk1[g] = v;
        acc[0] = fma_rn(v, v, acc[0]);
    }
    if (grid_sum<1>(acc, partials, S) && threadIdx.x == 0) {
        S->delta[k1] = sqrt(acc[0]);
        S->inv_delta = 1.0 / S->delta[k1];
    }
}

// K3: v+ /= delta, w+ = (eta delta) D^-1 v+, tmp = D^-1 v+
__global__ void __launch_bounds__(kThreads) k_scale_vw(double* vk1, double* wk1, double* tmp, DOp D, int n,
                                                       int k1, Scal* S)
{
    SQMR_GUARD
    const double sc = S->inv_delta;
    const double we = S->eta * S->delta[k1];
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        if (!D.tri) {
            const double v = vk1[g] * sc;
            vk1[g] = v;
            wk1[g] = v * we;
            tmp[g] = v;
            continue;
        }
        if (!D.is_piv[g]) continue;
        const double r1 = vk1[g] * sc;
        const double r2 = (g < n - 1) ? vk1[g + 1] * sc : 0.0;
        double g1, g2;
        bool two;
        dsolve_pair(D.tri, D.is_piv, n, g, r1, r2, g1, g2, two);
        vk1[g] = r1;
        wk1[g] = g1 * we;
        tmp[g] = g1;
        if (two) {
            vk1[g + 1] = r2;
            wk1[g + 1] = g2 * we;
            tmp[g + 1] = g2;
        }
    }
}

__device__ double sgn(double v) { return v < 0 ? -1.0 : 1.0; }

// k_sym_ortho (libs/la/helper_kernels.impl.cuh:662-700)
__device__ void sym_ortho(double a, double b, double& c, double& s, double& r)
{
    if (b == 0) { s = 0; r = fabs(a); c = (a == 0) ? 1 : sgn(a); }
    else if (a == 0) { c = 0; s = sgn(b); r = fabs(b); }
    else if (fabs(b) >= fabs(a)) {
        const double tao = a / b;
        s = sgn(b) / sqrt(fma_rn(tao, tao, 1.0));
        c = s * tao;
        r = b / s;
    } else {
        const double tao = b / a;
        c = sgn(a) / sqrt(fma_rn(tao, tao, 1.0));
        s = c * tao;
        r = a / c;
    }
}

// K4: beta+ and the scalar recurrence
__global__ void __launch_bounds__(kThreads) k_beta(const double* wk, const double* Av, const double* vk, int n,
                                                   int k0, int k1, int km1, double* partials, Scal* S)
{
    SQMR_GUARD
    double acc[2] = {0.0, 0.0};
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        acc[0] = fma_rn(wk[g], Av[g], acc[0]);
        acc[1] = fma_rn(wk[g], vk[g], acc[1]);
    }
    if (grid_sum<2>(acc, partials, S) && threadIdx.x == 0) {
        const double b = acc[0] / acc[1];
        S->beta[k1] = b;
        S->inv_beta = 1.0 / b;
        S->eta = (S->delta[k1] / b) * S->eta;
        const double na = sqrt(fma_rn(S->delta[k1], S->delta[k1], fma_rn(S->alpha, S->alpha, S->beta[k0] * S->beta[k0])));
        S->norm_A = fmax(S->norm_A, na);
        S->epsilon = S->s[km1] * S->beta[k0];
        S->beta_rot = (-S->c[km1]) * S->beta[k0];
        S->beta_rot_rot = fma_rn(S->c[k0], S->beta_rot, S->s[k0] * S->alpha);
        S->alpha_rot = fma_rn(S->s[k0], S->beta_rot, (-S->c[k0]) * S->alpha);
        double c, s, r;
        sym_ortho(S->alpha_rot, S->delta[k1], c, s, r);
        S->c[k1] = c;
        S->s[k1] = s;
        S->rho = r;
        S->inv_rho = 1.0 / r;
        S->tau = c * S->gamma;
        if (!isfinite(S->inv_beta) || !isfinite(S->inv_rho) || !isfinite(S->eta) || !isfinite(S->inv_delta)) {
            S->breakdown = 1;
            S->done = 1;
        }
    }
}

// K5: w+ /= beta+, p update, x += tau p, ||x||, gamma, test, lagged check
__global__ void __launch_bounds__(kThreads) k_update(double* wk1, const double* vk, double* pk, const double* pkm1,
                                                     const double* pkm2, double* x, int n, int k1, double* partials,
                                                     Scal* S)
{
    SQMR_GUARD
    const double ib = S->inv_beta, nbrr = -S->beta_rot_rot, ne = -S->epsilon, ir = S->inv_rho, tau = S->tau;
    double acc[1] = {0.0};
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        wk1[g] *= ib;
        double p = vk[g];
        p = fma_rn(nbrr, pkm1[g], p);
        p = fma_rn(ne, pkm2[g], p);
        p = p * ir;
        pk[g] = p;
        const double xv = fma_rn(tau, p, x[g]);
        x[g] = xv;
        acc[0] = fma_rn(xv, xv, acc[0]);
    }
    if (grid_sum<1>(acc, partials, S) && threadIdx.x == 0) {
        S->norm_x = sqrt(acc[0]);
        S->gamma = S->s[k1] * S->gamma;
        const int it = S->it;
        S->test0 |= (fabs(S->delta[k1]) <= S->tol);
        S->test1 |= (S->gamma / fma_rn(S->norm_A, S->norm_x, S->norm_pb) <= S->tol);
        bool stop = false;
        if (it > 0 && (it % 4) == 0) {
            if (S->snap0 || S->snap1) { stop = true; S->iters = it; }
        } else if (((it + 1) % 4) == 0) {
            S->snap0 = S->test0;
            S->snap1 = S->test1;
        }
        if (!stop) {
            S->it = it + 1;
            if (it + 1 >= S->max_it) { stop = true; S->iters = S->max_it; }
        }
        if (stop) S->done = 1;
    }
}

__global__ void k_init_scalars(Scal* S, double tol, int max_it)
{
    Scal z;
    memset(&z, 0, sizeof(z));
    z.c[0] = -1.0;
    z.tol = tol;
    z.max_it = max_it;
    *S = z;
}

}  // namespace

int sqmr_workspace(Sqmr* w, culipx_handle_t* h, int n)
{
    if (w->n == n) return CULIPX_OK;
    w->n = n;
    const size_t vb = (size_t)n * sizeof(double);
    CULIPX_TRY(w->vecs.alloc(h, 14 * vb + 64));
    CULIPX_TRY(w->partials.alloc(h, 4 * kGrid * sizeof(double)));
    CULIPX_TRY(w->scal.alloc(h, sizeof(Scal)));
    if (!w->host_flags) CULIPX_CUDA(cudaMallocHost(&w->host_flags, 64));
    return CULIPX_OK;
}

namespace {
int sqmr_phases(culipx_handle_t* h, Csr* A, DOp D, const PrecFn* pre, const double* b, double* x, double tol,
                int max_it, double* residual, int* iterations, Sqmr* w);
}

int sqmr_solve(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
               double* residual, int* iterations, Sqmr* w)
{
    if (!A || !b || !x || !w) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve: null argument");
    if (A->precision != CULIPX_F64) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve: A must be FP64");
    if (A->m != A->n) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve: A must be square");
    if (M && (!M->computed || M->pat->n != A->m))
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve: preconditioner not computed or wrong size");
    if (max_it < 0) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve: max_it < 0");
    // with a preconditioner: the single-launch persistent solver (FP64 or FP32
    // factor); block-Jacobi sweeps (SOLVE_JACOBI) run through the per-phase kernels
    if (M && !w->force_multi_kernel && M->solve_algorithm != CULIPX_SOLVE_JACOBI)
        return sqmr_solve_persistent(h, A, M, b, x, tol, max_it, residual, iterations, w);
    if (M && M->precision != CULIPX_F64)
        return fail(CULIPX_NOT_SUPPORTED, "culipx_sqmr_solve: the multi-kernel solver needs an FP64 factor");
    cudaStream_t s = h->stream;
    const DOp D = M ? DOp{M->tri.as<double>(), M->is_piv.as<int>()} : DOp{nullptr, nullptr};
    const PrecFn prec = [&](int stage, const double* in, double* out) { return prec_apply(M, stage, in, out, s); };
    return sqmr_phases(h, A, D, M ? &prec : nullptr, b, x, tol, max_it, residual, iterations, w);
}

namespace {

// The per-phase SQMR (one kernel per BLAS-1 step, as SQMR<T>::solve) with
// any split preconditioner: D (tri / is_piv, applied inside the fused
// kernels) and the left / middle / right applies through pre (null: none).
int sqmr_phases(culipx_handle_t* h, Csr* A, DOp D, const PrecFn* pre, const double* b, double* x, double tol,
                int max_it, double* residual, int* iterations, Sqmr* w)
{
    const int n = A->m;
    cudaStream_t s = h->stream;
    CULIPX_TRY(sqmr_workspace(w, h, n));
    double* base = w->vecs.as<double>();
    double *v[3], *wv[3], *p[3];
    for (int i = 0; i < 3; ++i) {
        v[i] = base + (size_t)i * n;
        wv[i] = base + (size_t)(3 + i) * n;
        p[i] = base + (size_t)(6 + i) * n;
    }
    double* Av = base + (size_t)9 * n;
    double* tmp = base + (size_t)10 * n;
    double* ev = base + (size_t)11 * n;
    double* ev2 = base + (size_t)12 * n;
    Scal* S = w->scal.as<Scal>();
    double* part = w->partials.as<double>();
    CULIPX_CUDA(cudaMemsetAsync(base, 0, (size_t)13 * n * sizeof(double), s));
    CULIPX_CUDA(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double), s));
    k_init_scalars<<<1, 1, 0, s>>>(S, tol, max_it);
    h->launches += 4;

    auto prec = [&](int stage, const double* in, double* out) -> int {
        if (pre) return (*pre)(stage, in, out);
        CULIPX_CUDA(cudaMemcpyAsync(out, in, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        return CULIPX_OK;
    };
    auto prec_spmv = [&](const double* in, double* out) -> int {
        CULIPX_TRY(prec(CULIPX_RIGHT, in, ev));
        CULIPX_TRY(csr_spmv(A, ev, ev2, 1.0, 0.0, 0, s));
        return prec(CULIPX_LEFT, ev2, out);
    };

    CULIPX_TRY(prec(CULIPX_LEFT, b, v[0]));
    k_init_norm<<<kGrid, kThreads, 0, s>>>(v[0], n, part, S);
    k_init_vw<<<kGrid, kThreads, 0, s>>>(v[0], wv[0], tmp, D, n, part, S);
    k_init_eta<<<kGrid, kThreads, 0, s>>>(wv[0], n, S);
    CULIPX_TRY(launch_check("sqmr init"));
    CULIPX_TRY(prec_spmv(tmp, Av));

    int it = 0;
    volatile int* flags = (volatile int*)w->host_flags;
    while (it < max_it) {
        const int k0 = acc3(it), k1 = acc3(it + 1), km1 = acc3(it - 1), km2 = acc3(it - 2);
        h->launches += 5;
        k_alpha<<<kGrid, kThreads, 0, s>>>(v[k0], Av, D, n, part, S);
        k_vnext<<<kGrid, kThreads, 0, s>>>(Av, v[k0], v[km1], v[k1], n, k0, k1, part, S);
        k_scale_vw<<<kGrid, kThreads, 0, s>>>(v[k1], wv[k1], tmp, D, n, k1, S);
        CULIPX_TRY(launch_check("sqmr K1-K3"));
        CULIPX_TRY(prec_spmv(tmp, Av));
        k_beta<<<kGrid, kThreads, 0, s>>>(wv[k0], Av, v[k0], n, k0, k1, km1, part, S);
        k_update<<<kGrid, kThreads, 0, s>>>(wv[k1], v[k0], p[k0], p[km1], p[km2], x, n, k1, part, S);
        CULIPX_TRY(launch_check("sqmr K4-K5"));
        ++it;
        if ((it % 4) == 0 || it >= max_it) {
            CULIPX_CUDA(cudaMemcpyAsync(w->host_flags, &S->done, sizeof(int), cudaMemcpyDeviceToHost, s));
            CULIPX_CUDA(cudaStreamSynchronize(s));
            if (flags[0]) break;
        }
    }
    // final: residual = gamma / ||M_L^-1 b||, x = P U^-1 D^-1 x~
    struct Out { double gamma, norm_pb; int iters, breakdown, done, it; } o;
    Scal hs;
    CULIPX_CUDA(cudaMemcpyAsync(&hs, S, sizeof(Scal), cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaStreamSynchronize(s));
    o.gamma = hs.gamma;
    o.norm_pb = hs.norm_pb;
    o.iters = hs.done ? hs.iters : hs.it;
    o.breakdown = hs.breakdown;
    if (max_it == 0) o.iters = 0;
    CULIPX_CUDA(cudaMemcpyAsync(Av, x, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (pre) {
        CULIPX_TRY((*pre)(CULIPX_MIDDLE, Av, tmp));
        CULIPX_TRY((*pre)(CULIPX_RIGHT, tmp, x));
    }
    CULIPX_CUDA(cudaStreamSynchronize(s));
    if (residual) *residual = o.gamma / o.norm_pb;
    if (iterations) *iterations = o.iters;
    if (o.breakdown) return fail(CULIPX_BREAKDOWN, "culipx_sqmr_solve: breakdown (non-finite scalar) at iteration %d", hs.it);
    if (!(hs.snap0 || hs.snap1) && o.iters >= max_it && max_it > 0) return CULIPX_MAXIT;
    return CULIPX_OK;
}

}  // namespace

// SQMR with an imported L D L' preconditioner (the per-phase solver: D inside
// the fused kernels, the triangular applies level by level)
int sqmr_solve_ldu(culipx_handle_t* h, Csr* A, Ldu* P, const double* b, double* x, double tol, int max_it,
                   double* residual, int* iterations, Sqmr* w)
{
    if (!A || !P || !b || !x || !w) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_ldu: null argument");
    if (A->precision != CULIPX_F64 || A->m != A->n || A->m != P->n)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_ldu: A must be square FP64 of the preconditioner's size");
    if (max_it < 0) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_ldu: max_it < 0");
    cudaStream_t s = h->stream;
    const DOp D{P->tri.as<double>(), P->is_piv.as<int>()};
    const PrecFn prec = [&](int stage, const double* in, double* out) { return ldu_apply(P, stage, in, out, s); };
    return sqmr_phases(h, A, D, &prec, b, x, tol, max_it, residual, iterations, w);
}

}  // namespace culipx
