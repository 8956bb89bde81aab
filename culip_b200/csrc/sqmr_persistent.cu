// Persistent SQMR: the whole preconditioned solve in one cooperative launch.
//
// Same recurrence, scalar update order and lagged convergence check as
// SQMR<T>::solve (libs/la/iterative_solvers/sqmr.impl.cuh:109-355) with the
// block-iLDL^T split preconditioner (solve_left / solve_middle / solve_right,
// libs/la/preconditioner/block_ildlt.impl.cuh:183-246).  Where the reference
// issues ~35 launches per iteration (cuBLAS BLAS-1, single-thread scalar
// kernels, per-level sweep kernels, cuSPARSE csrmv), one iteration here is a
// sequence of phases separated by grid-wide barriers:
//
//   A  w+ /= beta, p = (v - beta_rr p- - eps p--)/rho, x += tau p, ||x||;
//      fused with the next iteration's alpha dots v'(D^-1 Av), v'(D^-1 v)
//   B  v+ = Av - alpha v - beta v-, ||v+||
//   U  U-sweep levels (last to first), each warp on one block row: scales
//      its rows of v+ by 1/delta, applies D^-1 (w+ and the sweep's RHS),
//      subtracts the off-diagonal terms and back-substitutes with the pivot
//      tile; writes P U^-1 D^-1 v+ for the SpMV
//   S  CSR SpMV
//   L  U'-sweep levels (first to last) with the P' gather fused into the RHS
//      read; the last level's warps also accumulate beta's dots w'Av, w'v
//
// i.e. 3 + 2 x levels barriers per iteration and no scalar round trips: every
// CTA reduces the per-CTA partials in the same fixed order and runs the scalar
// recurrence itself (bit-identical across CTAs), so control flow is uniform.
#include "sqmr.h"
#include "factor.h"
#include "kernels_common.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

namespace cg = cooperative_groups;

namespace culipx {

namespace {

constexpr int kT = 256;          // threads per CTA
constexpr int kW = kT / 32;      // warps per CTA
constexpr int kMaxNV = 3;

template <class TF>
struct PArgs {
    int n, nl, max_it, spmv_lanes;
    double tol;
    const int* rowptr;
    const int* colidx;
    const double* kval;
    const TF* fval;
    const TF* tri;
    const int* is_piv;
    const int* perm;
    const int* bs;
    const int* lvl_off;
    const int* lvl_rows;
    const int* u_off;
    const int* u_col;
    const TF* u_val;
    const int* ut_off;
    const int* ut_col;
    const TF* ut_val;
    const long long* piv_off;
    const int* rowflags;
    double* v[3];
    double* w[3];
    double* p[3];
    double* Av;
    double* tvec;  // U-sweep values, unpermuted
    double* ev;    // P U^-1 (...)
    double* ev2;   // K ev
    double* x;
    const double* b;
    double* partials;  // 2 buffers x kMaxNV x gridDim
    double* out;       // [0] gamma/norm_pb, [1] iterations, [2] breakdown, [3] converged, [4] norm_pb, [5] it
    unsigned long long* ts;  // optional phase timestamps: [it * 8 + phase], it < kTsIters
};

constexpr int kTsIters = 64;

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// CTA 0 stamps phase boundaries (right after the barrier that ends a phase)
__device__ __forceinline__ void stamp(unsigned long long* ts, int it, int phase)
{
    if (ts && it < kTsIters && blockIdx.x == 0 && threadIdx.x == 0) ts[it * 8 + phase] = global_ns();
}

struct Scal {
    double alpha, beta[3], delta[3], c[3], s[3];
    double norm_A, epsilon, beta_rot, beta_rot_rot, alpha_rot, tau, rho, gamma, norm_pb, norm_x, eta;
    double inv_delta, inv_beta, inv_rho;
    int test0, test1, snap0, snap1, done, iters, breakdown, red;
};

__host__ __device__ __forceinline__ int acc3(int r) { return (r % 3) + ((r < 0) ? 3 : 0); }

// fixed-order block sum; every thread receives the totals
template <int NV>
__device__ void block_allsum(double (&v)[NV], double (*sh)[kW])
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][w] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = 0.0;
        for (int i = 0; i < kW; ++i) t += sh[k][i];
        v[k] = t;
    }
}

// grid-wide sum with a barrier; identical totals in every CTA and thread
template <int NV>
__device__ void grid_allsum(double (&v)[NV], double* partials, int& red, double (*sh)[kW], cg::grid_group& grid)
{
    block_allsum<NV>(v, sh);
    double* buf = partials + (size_t)(red & 1) * kMaxNV * gridDim.x;
    ++red;
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) buf[k * gridDim.x + blockIdx.x] = v[k];
    grid.sync();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = 0.0;
        for (int bidx = threadIdx.x; bidx < (int)gridDim.x; bidx += kT) t += __ldcg(buf + k * gridDim.x + bidx);
        v[k] = t;
    }
    block_allsum<NV>(v, sh);
}

// D^-1 inside one block row held by a warp (k_solve_D, helper_kernels.impl.cuh:720-774):
// lane r < h holds y_r; returns (D^-1 y)_r
template <class TF>
__device__ double dsolve_warp(double y, int fr, int h, const TF* tri, const int* is_piv)
{
    const int lane = lane_id();
    const double ynext = __shfl_down_sync(0xffffffffu, y, 1);
    const int ip = (lane < h) ? is_piv[fr + lane] : 1;
    const int ipn = __shfl_down_sync(0xffffffffu, ip, 1);
    const int next_piv = (lane + 1 < h) ? ipn : 1;
    double g1 = 0.0, g2 = 0.0;
    if (lane < h) {
        const double p11 = (double)tri[3 * (size_t)(fr + lane) + 1], p12 = (double)tri[3 * (size_t)(fr + lane) + 2];
        const double p22 = !next_piv ? (double)tri[3 * (size_t)(fr + lane + 1) + 1] : 1.0;
        const double r2 = (lane + 1 < h) ? ynext : 0.0;
        const double gr = sqrt(fma_rn(p11, p11, p12 * p12));
        const double gc = p11 / gr, gs = p12 / gr;
        g1 = fma_rn(gc, y, gs * r2);
        g2 = fma_rn(-gs, y, gc * r2);
        const double tp12 = fma_rn(gc, p12, gs * p22);
        const double tp22 = fma_rn(-gs, p12, gc * p22);
        g2 = g2 / tp22;
        g1 = fma_rn(-tp12, g2, g1) / gr;
    }
    const double from_prev = __shfl_up_sync(0xffffffffu, g2, 1);
    return ip ? g1 : from_prev;
}

// triangular solve with the block row's pivot tile (d_left_solve_row_major,
// block_ildlt_kernels.impl.cuh:2087-2113); UPPER: back substitution with U,
// else forward substitution with U'
template <class TF, bool UPPER>
__device__ double pivot_solve(double acc, const TF* P, int h, TF* tile)
{
    const int lane = lane_id();
    if (lane < h)
        for (int i = 0; i < h; ++i) tile[i * kTileStride + lane] = P[i * h + lane];
    __syncwarp();
    TF a = (TF)acc;
    if (UPPER) {
        for (int c = h - 1; c >= 0; --c) {
            if (lane == c) a = a / tile[c * kTileStride + c];
            const TF xc = __shfl_sync(0xffffffffu, a, c);
            if (lane < c) a = fma_rn(-tile[lane * kTileStride + c], xc, a);
        }
    } else {
        for (int r = 0; r < h; ++r) {
            if (lane == r) a = a / tile[r * kTileStride + r];
            const TF xr = __shfl_sync(0xffffffffu, a, r);
            if (lane > r && lane < h) a = fma_rn(-tile[r * kTileStride + lane], xr, a);
        }
    }
    __syncwarp();
    return (double)a;
}

// U-sweep over all levels: rhs_r = D^-1(scale * src)_r (src scaled in place if
// write_scaled, w = we * rhs if w != null), t = U^-1 rhs, out[perm[r]] = t_r
template <class TF>
__device__ void usweep(const PArgs<TF>& a, double* src, double scale, bool write_scaled, double* wout, double we,
                       double* out, TF* tile, cg::grid_group& grid)
{
    const int lane = lane_id();
    const int gw = blockIdx.x * kW + (threadIdx.x >> 5);
    const int nw = gridDim.x * kW;
    for (int L = a.nl - 1; L >= 0; --L) {
        const int r0 = a.lvl_off[L], nr = a.lvl_off[L + 1] - r0;
        for (int t = gw; t < nr; t += nw) {
            const int I = a.lvl_rows[r0 + t];
            const int fr = a.bs[I], h = a.bs[I + 1] - fr;
            double y = (lane < h) ? src[fr + lane] * scale : 0.0;
            if (write_scaled && lane < h) src[fr + lane] = y;
            const double d = dsolve_warp<TF>(y, fr, h, a.tri, a.is_piv);
            if (wout && lane < h) wout[fr + lane] = d * we;
            double acc = d;
            if (lane < h) {
                TF accf = (TF)acc;
                const int e1 = a.u_off[fr + lane + 1];
                for (int k = a.u_off[fr + lane]; k < e1; ++k)
                    accf = fma_rn(-a.u_val[k], (TF)a.tvec[a.u_col[k]], accf);
                acc = (double)accf;
            }
            if (!(a.rowflags[I] & 1)) acc = pivot_solve<TF, true>(acc, a.fval + a.piv_off[I], h, tile);
            if (lane < h) {
                a.tvec[fr + lane] = acc;
                out[a.perm[fr + lane]] = acc;
            }
        }
        grid.sync();
    }
}

// U'-sweep over all levels: rhs_r = src[perm[r]], result into dst; optional
// dots of dst with wk and of vk with wk (beta's numerator / denominator)
template <class TF>
__device__ void utsweep(const PArgs<TF>& a, const double* src, double* dst, const double* wk, const double* vk,
                        double (&dots)[2], TF* tile, cg::grid_group& grid, bool last_sync)
{
    const int lane = lane_id();
    const int gw = blockIdx.x * kW + (threadIdx.x >> 5);
    const int nw = gridDim.x * kW;
    for (int L = 0; L < a.nl; ++L) {
        const int r0 = a.lvl_off[L], nr = a.lvl_off[L + 1] - r0;
        for (int t = gw; t < nr; t += nw) {
            const int I = a.lvl_rows[r0 + t];
            const int fr = a.bs[I], h = a.bs[I + 1] - fr;
            double acc = 0.0;
            if (lane < h) {
                TF accf = (TF)src[a.perm[fr + lane]];
                const int e1 = a.ut_off[fr + lane + 1];
                for (int k = a.ut_off[fr + lane]; k < e1; ++k)
                    accf = fma_rn(-a.ut_val[k], (TF)dst[a.ut_col[k]], accf);
                acc = (double)accf;
            }
            if (!(a.rowflags[I] & 1)) acc = pivot_solve<TF, false>(acc, a.fval + a.piv_off[I], h, tile);
            if (lane < h) {
                dst[fr + lane] = acc;
                if (wk) {
                    dots[0] = fma_rn(wk[fr + lane], acc, dots[0]);
                    dots[1] = fma_rn(wk[fr + lane], vk[fr + lane], dots[1]);
                }
            }
        }
        if (L < a.nl - 1 || last_sync) grid.sync();
    }
}

template <class TF>
__device__ void spmv_phase(const PArgs<TF>& a, const double* x, double* y, cg::grid_group& grid)
{
    const int L = a.spmv_lanes;
    const int lane = lane_id();
    const int sub = lane % L;
    const long long gw = (long long)blockIdx.x * kW + (threadIdx.x >> 5);
    const long long nw = (long long)gridDim.x * kW;
    const int rpw = 32 / L;
    for (long long base = gw * rpw; base < a.n; base += nw * rpw) {
        const long long row = base + lane / L;
        double acc = 0.0;
        if (row < a.n) {
            const int e = __ldg(a.rowptr + row + 1);
            for (int k = __ldg(a.rowptr + row) + sub; k < e; k += L)
                acc = fma_rn(__ldg(a.kval + k), x[__ldg(a.colidx + k)], acc);
        }
        for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (row < a.n && sub == 0) y[row] = acc;
    }
    grid.sync();
}

__device__ double sgn(double v) { return v < 0 ? -1.0 : 1.0; }

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

// alpha's two dots over all rows: v'(D^-1 Av), v'(D^-1 v), D applied per pivot
template <class TF>
__device__ void alpha_dots(const PArgs<TF>& a, const double* vk, double (&acc)[2])
{
    for (int g = blockIdx.x * kT + threadIdx.x; g < a.n; g += gridDim.x * kT) {
        if (!a.is_piv[g]) continue;
        const int next_piv = (g < a.n - 1) ? a.is_piv[g + 1] : 1;
        const bool two = !next_piv;
        const double p11 = (double)a.tri[3 * (size_t)g + 1], p12 = (double)a.tri[3 * (size_t)g + 2];
        const double p22 = two ? (double)a.tri[3 * (size_t)(g + 1) + 1] : 1.0;
        const double gr = sqrt(fma_rn(p11, p11, p12 * p12));
        const double gc = p11 / gr, gs = p12 / gr;
        const double tp12 = fma_rn(gc, p12, gs * p22);
        const double tp22 = fma_rn(-gs, p12, gc * p22);
        const bool has_next = g < a.n - 1;
        const double av1 = a.Av[g], av2 = has_next ? a.Av[g + 1] : 0.0;
        const double v1 = vk[g], v2 = has_next ? vk[g + 1] : 0.0;
        double ga1 = fma_rn(gc, av1, gs * av2), ga2 = fma_rn(-gs, av1, gc * av2);
        ga2 = ga2 / tp22;
        ga1 = fma_rn(-tp12, ga2, ga1) / gr;
        double gv1 = fma_rn(gc, v1, gs * v2), gv2 = fma_rn(-gs, v1, gc * v2);
        gv2 = gv2 / tp22;
        gv1 = fma_rn(-tp12, gv2, gv1) / gr;
        acc[0] = fma_rn(v1, ga1, acc[0]);
        acc[1] = fma_rn(v1, gv1, acc[1]);
        if (two) {
            acc[0] = fma_rn(v2, ga2, acc[0]);
            acc[1] = fma_rn(v2, gv2, acc[1]);
        }
    }
}

template <class TF>
__global__ void __launch_bounds__(kT) k_sqmr_persistent(PArgs<TF> a)
{
    cg::grid_group grid = cg::this_grid();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TF* tile = reinterpret_cast<TF*>(smem_raw) + (size_t)(threadIdx.x >> 5) * kTileElems;
    __shared__ double sh[kMaxNV][kW];
    // every thread carries the scalar recurrence itself; all threads of all
    // CTAs compute it from the same reduced values, so it is identical
    Scal S;
    memset(&S, 0, sizeof(S));
    S.c[0] = -1.0;
    int red = 0;
    const int n = a.n;
    const int g0 = blockIdx.x * kT + threadIdx.x, gs_ = gridDim.x * kT;
    double dots2[2] = {0.0, 0.0};

    // ---- init: v0 = U'^-1 P' b; ||v0|| ----
    utsweep<TF>(a, a.b, a.v[0], nullptr, nullptr, dots2, tile, grid, true);
    {
        double acc[1] = {0.0};
        for (int g = g0; g < n; g += gs_) acc[0] = fma_rn(a.v[0][g], a.v[0][g], acc[0]);
        grid_allsum<1>(acc, a.partials, red, sh, grid);
        S.norm_pb = sqrt(acc[0]);
        S.gamma = S.norm_pb;
    }
    const double inv_pb = 1.0 / S.norm_pb;
    // v0 scaled, w0 = D^-1 v0 (eta applied below), ev = P U^-1 D^-1 v0
    usweep<TF>(a, a.v[0], inv_pb, true, a.w[0], 1.0, a.ev, tile, grid);
    {
        double acc[1] = {0.0};
        for (int g = g0; g < n; g += gs_) acc[0] = fma_rn(a.w[0][g], a.w[0][g], acc[0]);
        grid_allsum<1>(acc, a.partials, red, sh, grid);
        S.eta = 1.0 / sqrt(acc[0]);
    }
    for (int g = g0; g < n; g += gs_) a.w[0][g] *= S.eta;
    if (!isfinite(inv_pb) || !isfinite(S.eta)) { S.breakdown = 1; S.done = 1; }
    spmv_phase<TF>(a, a.ev, a.ev2, grid);
    utsweep<TF>(a, a.ev2, a.Av, nullptr, nullptr, dots2, tile, grid, true);
    // alpha dots for iteration 0
    double ad[2] = {0.0, 0.0};
    alpha_dots<TF>(a, a.v[0], ad);
    grid_allsum<2>(ad, a.partials, red, sh, grid);

    int it = 0;
    while (!S.done && it < a.max_it) {
        const int k0 = acc3(it), k1 = acc3(it + 1), km1 = acc3(it - 1), km2 = acc3(it - 2);
        stamp(a.ts, it, 0);
        S.alpha = ad[0] / ad[1];
        // ---- B: v+ and ||v+|| ----
        {
            const double na = -S.alpha, nb = -S.beta[k0];
            double acc[1] = {0.0};
            for (int g = g0; g < n; g += gs_) {
                double v = a.Av[g];
                v = fma_rn(na, a.v[k0][g], v);
                v = fma_rn(nb, a.v[km1][g], v);
                a.v[k1][g] = v;
                acc[0] = fma_rn(v, v, acc[0]);
            }
            grid_allsum<1>(acc, a.partials, red, sh, grid);
            S.delta[k1] = sqrt(acc[0]);
            S.inv_delta = 1.0 / S.delta[k1];
        }
        stamp(a.ts, it, 1);
        // ---- U: v+ /= delta, w+ = eta delta D^-1 v+, ev = P U^-1 D^-1 v+ ----
        usweep<TF>(a, a.v[k1], S.inv_delta, true, a.w[k1], S.eta * S.delta[k1], a.ev, tile, grid);
        stamp(a.ts, it, 2);
        // ---- S: ev2 = K ev ----
        spmv_phase<TF>(a, a.ev, a.ev2, grid);
        stamp(a.ts, it, 3);
        // ---- L: Av = U'^-1 P' ev2, beta dots ----
        double bd[2] = {0.0, 0.0};
        utsweep<TF>(a, a.ev2, a.Av, a.w[k0], a.v[k0], bd, tile, grid, false);
        grid_allsum<2>(bd, a.partials, red, sh, grid);
        stamp(a.ts, it, 4);
        {
            const double bt = bd[0] / bd[1];
            S.beta[k1] = bt;
            S.inv_beta = 1.0 / bt;
            S.eta = (S.delta[k1] / bt) * S.eta;
            const double nA =
                sqrt(fma_rn(S.delta[k1], S.delta[k1], fma_rn(S.alpha, S.alpha, S.beta[k0] * S.beta[k0])));
            S.norm_A = fmax(S.norm_A, nA);
            S.epsilon = S.s[km1] * S.beta[k0];
            S.beta_rot = (-S.c[km1]) * S.beta[k0];
            S.beta_rot_rot = fma_rn(S.c[k0], S.beta_rot, S.s[k0] * S.alpha);
            S.alpha_rot = fma_rn(S.s[k0], S.beta_rot, (-S.c[k0]) * S.alpha);
            double c, s, r;
            sym_ortho(S.alpha_rot, S.delta[k1], c, s, r);
            S.c[k1] = c;
            S.s[k1] = s;
            S.rho = r;
            S.inv_rho = 1.0 / r;
            S.tau = c * S.gamma;
        }
        // ---- A: w+ /= beta, p, x, ||x||, next alpha dots ----
        {
            const double ib = S.inv_beta, nbrr = -S.beta_rot_rot, ne = -S.epsilon, ir = S.inv_rho, tau = S.tau;
            double acc[1] = {0.0};
            for (int g = g0; g < n; g += gs_) {
                a.w[k1][g] *= ib;
                double p = a.v[k0][g];
                p = fma_rn(nbrr, a.p[km1][g], p);
                p = fma_rn(ne, a.p[km2][g], p);
                p = p * ir;
                a.p[k0][g] = p;
                const double xv = fma_rn(tau, p, a.x[g]);
                a.x[g] = xv;
                acc[0] = fma_rn(xv, xv, acc[0]);
            }
            double nd[2] = {0.0, 0.0};
            alpha_dots<TF>(a, a.v[k1], nd);
            // ||x||^2 and the next alpha's two dots share one barrier
            double r3[3] = {acc[0], nd[0], nd[1]};
            grid_allsum<3>(r3, a.partials, red, sh, grid);
            ad[0] = r3[1];
            ad[1] = r3[2];
            S.norm_x = sqrt(r3[0]);
        }
        stamp(a.ts, it, 5);
        S.gamma = S.s[k1] * S.gamma;
        S.test0 |= (fabs(S.delta[k1]) <= a.tol);
        S.test1 |= (S.gamma / fma_rn(S.norm_A, S.norm_x, S.norm_pb) <= a.tol);
        bool stop = false;
        if (it > 0 && (it % 4) == 0) {
            if (S.snap0 || S.snap1) { stop = true; S.iters = it; }
        } else if (((it + 1) % 4) == 0) {
            S.snap0 = S.test0;
            S.snap1 = S.test1;
        }
        if (!isfinite(S.inv_beta) || !isfinite(S.inv_rho) || !isfinite(S.eta) || !isfinite(S.inv_delta) ||
            !isfinite(S.alpha)) {
            S.breakdown = 1;
            stop = true;
            S.iters = it;
        }
        if (!stop) {
            ++it;
            if (it >= a.max_it) S.iters = a.max_it;
        }
        if (stop) S.done = 1;
    }
    if (!S.done) S.iters = it;
    // ---- x = P U^-1 D^-1 x~ ----
    for (int g = g0; g < n; g += gs_) a.ev2[g] = a.x[g];
    grid.sync();
    usweep<TF>(a, a.ev2, 1.0, false, nullptr, 0.0, a.x, tile, grid);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = S.gamma / S.norm_pb;
        a.out[1] = S.iters;
        a.out[2] = S.breakdown;
        a.out[3] = (S.snap0 || S.snap1) ? 1 : 0;
        a.out[4] = S.norm_pb;
        a.out[5] = it;
    }
}

template <class TF>
int launch_persistent(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                      double* residual, int* iterations, Sqmr* w, bool* converged, bool* breakdown)
{
    const int n = A->m;
    cudaStream_t s = h->stream;
    CULIPX_TRY(sqmr_workspace(w, h, n));
    Pattern& p = *M->pat;
    const size_t smem = (size_t)kW * kTileElems * sizeof(TF);
    static int grid_cache[2] = {0, 0};
    int& G = grid_cache[sizeof(TF) == 8 ? 0 : 1];
    if (G == 0) {
        CULIPX_CUDA(cudaFuncSetAttribute(k_sqmr_persistent<TF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0, sms = 0, dev = 0;
        CULIPX_CUDA(cudaGetDevice(&dev));
        CULIPX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CULIPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sqmr_persistent<TF>, kT, smem));
        if (per_sm < 1) return fail(CULIPX_NOT_SUPPORTED, "persistent SQMR kernel does not fit on an SM");
        G = sms * std::min(per_sm, 2);
    }
    if ((size_t)(2 * kMaxNV * G) * sizeof(double) > w->partials.bytes())
        CULIPX_TRY(w->partials.alloc(h, (size_t)2 * kMaxNV * G * sizeof(double)));
    double* base = w->vecs.as<double>();
    PArgs<TF> a;
    a.n = n;
    a.nl = p.num_levels;
    a.max_it = max_it;
    const double avg = (double)A->nnz / std::max(n, 1);
    a.spmv_lanes = (avg <= 4.5) ? 4 : (avg <= 12.0) ? 8 : (avg <= 24.0) ? 16 : 32;
    a.tol = tol;
    a.rowptr = A->rowptr;
    a.colidx = A->colidx;
    a.kval = static_cast<const double*>(A->val);
    a.fval = M->val.as<TF>();
    a.tri = M->tri.as<TF>();
    a.is_piv = M->is_piv.as<int>();
    a.perm = M->perm.as<int>();
    a.bs = p.d_bs.as<int>();
    a.lvl_off = p.d_lvl_off.as<int>();
    a.lvl_rows = p.d_lvl_rows.as<int>();
    a.u_off = M->u_off.as<int>();
    a.u_col = M->u_col.as<int>();
    a.u_val = M->u_val.as<TF>();
    a.ut_off = M->ut_off.as<int>();
    a.ut_col = M->ut_col.as<int>();
    a.ut_val = M->ut_val.as<TF>();
    a.piv_off = M->piv_off.as<long long>();
    a.rowflags = M->rowflags.as<int>();
    for (int i = 0; i < 3; ++i) {
        a.v[i] = base + (size_t)i * n;
        a.w[i] = base + (size_t)(3 + i) * n;
        a.p[i] = base + (size_t)(6 + i) * n;
    }
    a.Av = base + (size_t)9 * n;
    a.tvec = base + (size_t)10 * n;
    a.ev = base + (size_t)11 * n;
    a.ev2 = base + (size_t)12 * n;
    a.x = x;
    a.b = b;
    a.partials = w->partials.as<double>();
    a.out = base + (size_t)13 * n;
    a.ts = nullptr;
    if (w->profile) {
        if (w->ts.bytes() < (size_t)kTsIters * 8 * sizeof(unsigned long long))
            CULIPX_TRY(w->ts.alloc(h, (size_t)kTsIters * 8 * sizeof(unsigned long long)));
        CULIPX_CUDA(cudaMemsetAsync(w->ts.get(), 0, (size_t)kTsIters * 8 * sizeof(unsigned long long), s));
        a.ts = w->ts.as<unsigned long long>();
    }
    CULIPX_CUDA(cudaMemsetAsync(base, 0, (size_t)13 * n * sizeof(double), s));
    CULIPX_CUDA(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double), s));
    void* args[] = {&a};
    CULIPX_CUDA(cudaLaunchCooperativeKernel((const void*)k_sqmr_persistent<TF>, dim3(G), dim3(kT), args, smem, s));
    h->launches += 1;
    double out[6];
    CULIPX_CUDA(cudaMemcpyAsync(out, a.out, sizeof(out), cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaStreamSynchronize(s));
    if (residual) *residual = out[0];
    if (iterations) *iterations = (int)out[1];
    *breakdown = out[2] != 0.0;
    *converged = out[3] != 0.0;
    return CULIPX_OK;
}

}  // namespace

int sqmr_solve_persistent(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                          double* residual, int* iterations, Sqmr* w)
{
    bool conv = false, bd = false;
    int st;
    if (M->precision == CULIPX_F64) st = launch_persistent<double>(h, A, M, b, x, tol, max_it, residual, iterations, w, &conv, &bd);
    else st = launch_persistent<float>(h, A, M, b, x, tol, max_it, residual, iterations, w, &conv, &bd);
    if (st != CULIPX_OK) return st;
    if (bd) return fail(CULIPX_BREAKDOWN, "culipx_sqmr_solve: breakdown (non-finite scalar)");
    if (!conv && max_it > 0 && iterations && *iterations >= max_it) return CULIPX_MAXIT;
    return CULIPX_OK;
}

// ---------------------------------------------------------------------------
// SQMR without device allocation.
//
// For callers that cannot allocate device memory when they solve: processes
// whose device memory is already handed out by another allocator (a caching
// allocator such as PyTorch's, or an application-wide pool that owns the
// GPU), and latency-critical request loops, where cudaMalloc / cudaFree can
// synchronize the device and take milliseconds.  The factor (and K) are set
// up beforehand through the regular entry points; this call then uses a
// fixed scratch area compiled into the library instead of the handle's
// workspace.
//
// The scratch is a file-scope device array of kNoAllocMaxRows x 14 doubles
// plus the per-CTA reduction slots (about 7.4 MB): every GPU that loads this
// library holds it until the process exits.  All calls share it and it keeps
// the last call's contents; the call clears what must start at zero.  Calls
// whose work overlaps on the GPU (two streams, two host threads) race on it.
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current); make that first call
// before any stream capture.
namespace {

constexpr int kNoAllocMaxRows = 65536;
constexpr int kNoAllocMaxGrid = 1024;
constexpr size_t kNoAllocVecs = 14 * (size_t)kNoAllocMaxRows;
constexpr size_t kNoAllocSlots = kNoAllocVecs + (size_t)2 * kMaxNV * kNoAllocMaxGrid;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocSlots];

double* g_noalloc_ptr[64] = {nullptr};  // per-device address of g_noalloc_scratch
int g_noalloc_grid[64][2] = {{0, 0}};   // per-device grid size per factor precision

int noalloc_setup(int dev)
{
    if (dev < 0 || dev >= 64) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_noalloc: device %d out of range", dev);
    if (g_noalloc_ptr[dev]) return CULIPX_OK;
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
        cudaGetLastError();
        return fail(CULIPX_CUDA_ERROR, "culipx_sqmr_solve_noalloc: cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(e));
    }
    g_noalloc_ptr[dev] = static_cast<double*>(ptr);
    return CULIPX_OK;
}

template <class TF>
int noalloc_grid(int dev, int* G)
{
    int& g = g_noalloc_grid[dev][sizeof(TF) == 8 ? 0 : 1];
    if (g == 0) {
        const size_t smem = (size_t)kW * kTileElems * sizeof(TF);
        CULIPX_CUDA(cudaFuncSetAttribute(k_sqmr_persistent<TF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0, sms = 0;
        CULIPX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CULIPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sqmr_persistent<TF>, kT, smem));
        if (per_sm < 1) return fail(CULIPX_NOT_SUPPORTED, "persistent SQMR kernel does not fit on an SM");
        g = std::min(sms * std::min(per_sm, 2), kNoAllocMaxGrid);
    }
    *G = g;
    return CULIPX_OK;
}

template <class TF>
int launch_noalloc(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                   double* residual, int* iterations, bool* converged, bool* breakdown)
{
    const int n = A->m;
    cudaStream_t s = h->stream;
    int dev = 0;
    CULIPX_CUDA(cudaGetDevice(&dev));
    CULIPX_TRY(noalloc_setup(dev));
    int G = 0;
    CULIPX_TRY(noalloc_grid<TF>(dev, &G));
    Pattern& p = *M->pat;
    double* base = g_noalloc_ptr[dev];
    PArgs<TF> a;
    a.n = n;
    a.nl = p.num_levels;
    a.max_it = max_it;
    const double avg = (double)A->nnz / std::max(n, 1);
    a.spmv_lanes = (avg <= 4.5) ? 4 : (avg <= 12.0) ? 8 : (avg <= 24.0) ? 16 : 32;
    a.tol = tol;
    a.rowptr = A->rowptr;
    a.colidx = A->colidx;
    a.kval = static_cast<const double*>(A->val);
    a.fval = M->val.as<TF>();
    a.tri = M->tri.as<TF>();
    a.is_piv = M->is_piv.as<int>();
    a.perm = M->perm.as<int>();
    a.bs = p.d_bs.as<int>();
    a.lvl_off = p.d_lvl_off.as<int>();
    a.lvl_rows = p.d_lvl_rows.as<int>();
    a.u_off = M->u_off.as<int>();
    a.u_col = M->u_col.as<int>();
    a.u_val = M->u_val.as<TF>();
    a.ut_off = M->ut_off.as<int>();
    a.ut_col = M->ut_col.as<int>();
    a.ut_val = M->ut_val.as<TF>();
    a.piv_off = M->piv_off.as<long long>();
    a.rowflags = M->rowflags.as<int>();
    for (int i = 0; i < 3; ++i) {
        a.v[i] = base + (size_t)i * n;
        a.w[i] = base + (size_t)(3 + i) * n;
        a.p[i] = base + (size_t)(6 + i) * n;
    }
    a.Av = base + (size_t)9 * n;
    a.tvec = base + (size_t)10 * n;
    a.ev = base + (size_t)11 * n;
    a.ev2 = base + (size_t)12 * n;
    a.out = base + (size_t)13 * n;
    a.partials = base + kNoAllocVecs;
    a.ts = nullptr;
    a.x = x;
    a.b = b;
    // the scratch keeps the previous call's contents: clear the recurrence vectors
    CULIPX_CUDA(cudaMemsetAsync(base, 0, (size_t)13 * n * sizeof(double), s));
    CULIPX_CUDA(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double), s));
    const size_t smem = (size_t)kW * kTileElems * sizeof(TF);
    void* args[] = {&a};
    CULIPX_CUDA(cudaLaunchCooperativeKernel((const void*)k_sqmr_persistent<TF>, dim3(G), dim3(kT), args, smem, s));
    h->launches += 1;
    double out[6];
    CULIPX_CUDA(cudaMemcpyAsync(out, a.out, sizeof(out), cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaStreamSynchronize(s));
    if (residual) *residual = out[0];
    if (iterations) *iterations = (int)out[1];
    *breakdown = out[2] != 0.0;
    *converged = out[3] != 0.0;
    return CULIPX_OK;
}

}  // namespace

int sqmr_solve_noalloc(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                       double* residual, int* iterations)
{
    if (!A || !M || !b || !x) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_noalloc: null argument");
    if (A->precision != CULIPX_F64 || A->m != A->n)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_noalloc: A must be square FP64");
    if (!M->computed || M->pat->n != A->m)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_noalloc: preconditioner not computed or wrong size");
    if (A->m > kNoAllocMaxRows)
        return fail(CULIPX_INVALID_ARG,
                    "culipx_sqmr_solve_noalloc: n = %d exceeds the fixed scratch of %d rows; use culipx_sqmr_solve",
                    A->m, kNoAllocMaxRows);
    if (max_it < 0) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_noalloc: max_it < 0");
    bool conv = false, bd = false;
    int st;
    if (M->precision == CULIPX_F64)
        st = launch_noalloc<double>(h, A, M, b, x, tol, max_it, residual, iterations, &conv, &bd);
    else
        st = launch_noalloc<float>(h, A, M, b, x, tol, max_it, residual, iterations, &conv, &bd);
    if (st != CULIPX_OK) return st;
    if (bd) return fail(CULIPX_BREAKDOWN, "culipx_sqmr_solve_noalloc: breakdown (non-finite scalar)");
    if (!conv && max_it > 0 && iterations && *iterations >= max_it) return CULIPX_MAXIT;
    return CULIPX_OK;
}

}  // namespace culipx
