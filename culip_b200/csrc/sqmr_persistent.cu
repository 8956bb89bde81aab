// Persistent SQMR: the whole preconditioned solve in one cooperative launch.
//
// Same recurrence and lagged convergence check as SQMR<T>::solve
// (libs/la/iterative_solvers/sqmr.impl.cuh:109-355) with the block-iLDL^T
// split preconditioner (solve_left / solve_middle / solve_right,
// libs/la/preconditioner/block_ildlt.impl.cuh:183-246).  Where the reference
// issues ~35 launches per iteration (cuBLAS BLAS-1, single-thread scalar
// kernels, per-level sweep kernels, cuSPARSE csrmv), one iteration here is
// three groups of phases separated by grid-wide barriers.  A phase is a set
// of work items, one warp per block row and one lane per fine row, plus
// coalesced loops over whole vectors:
//
//   P1  v+ = Av - alpha v - beta v- (kept unscaled) and ||v+||^2 over all
//       rows; the first U-sweep level (the last level set) on v+.
//       Barrier + reduction: delta and the rotation scalars that need only
//       alpha, beta and delta (rho, tau, epsilon, gamma).
//   P2  the remaining U-sweep levels: D^-1 (k_solve_D), the off-diagonal
//       terms, back substitution with the pivot tile; the result goes
//       straight to its permuted place, ev = P U^-1 D^-1 v+.  One barrier
//       per level.
//   P3  the U'-sweep levels with the SpMV fused into the right-hand side:
//       each block row's warp computes (K ev) for its own rows (the P'
//       permutation is local to a block row), scales by 1/delta and
//       forward-substitutes into Av.  The same warp accumulates, over its
//       rows, beta's numerator v' D^-1 Av and the next alpha's dots
//       v+' D^-1 Av and v+' D^-1 v+; the first level also updates p and x.
//       Barrier + reduction: beta, the next alpha, ||x||, the tests.
//
// That is 2 x (number of levels) barriers per iteration, fewer for a KKT
// system in natural order (two levels, level 0 of simple rows): there the
// level-0 rows also compute their (K ev) in the U sweep (the U' sweep's
// level-0 phase goes away), and instead of a grid barrier between the U
// sweep's two levels every CTA counts its finished level-1 rows on a device
// counter that the level-0 rows wait for (one elected poller per CTA, a
// bounded wait: a wait that gives up ends the solve with CULIPX_TIMEOUT) --
// two grid synchronisations per iteration, both reductions.  Re-associations against the reference, all exact in
// real arithmetic:
//   * v+ is divided by delta after the U sweep instead of before it (the
//     sweep is linear); the division is applied to the SpMV result.
//   * The reference's w_k (sqmr.impl.cuh, solve_middle of v_k scaled by eta
//     and 1/beta) equals eta_k D^-1 v_k at every step, so it is not stored:
//     beta = (w' Av) / (w' v) = (v' D^-1 Av) / (v' D^-1 v), whose
//     denominator is the previous alpha's denominator.  eta is still
//     carried for the reference's breakdown test.
//   * The p / x update runs one phase later than in the reference (it needs
//     only alpha, beta_k and delta).
// Every CTA reduces the per-CTA partials in the same fixed order and its
// thread 0 runs the scalar recurrence in shared memory, so control flow is
// uniform across the grid and the result is deterministic for a given grid
// size.
//
// Data the loop reads: K (CSR), U and U' as fine-row CSR (U's columns mapped
// through P), the non-identity pivot tiles as packed upper triangles (column
// by column for U, row by row for U'), the diagonal of D for block rows with
// 1x1 pivots only (D^-1 y = y / d there, which is what the Givens form
// computes for a 1x1 pivot) and tri / is_piv for the others, and 9 vectors.
#include "sqmr.h"
#include "factor.h"
#include "pattern.h"
#include "kernels_common.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>

namespace cg = cooperative_groups;

namespace culipx {

namespace {

constexpr int kT = 512;          // threads per CTA
constexpr int kW = kT / 32;      // warps per CTA
constexpr int kCtasPerSm = 2;    // 32 resident warps per SM
constexpr int kMaxNR = 4;        // right-hand sides per launch
constexpr int kMaxNV = 4 * kMaxNR;  // values per grid reduction
constexpr int kBatch = 8;        // loads issued ahead in row sums and tile solves
constexpr int kVecs = 7;         // work vectors of n doubles
constexpr unsigned kFull = 0xffffffffu;

template <class TF>
struct PArgs {
    int n, nl, max_it;
    int fuse_l0;               // level-0 simple rows compute (K ev) in the U sweep
    double tol;
    const int* rowptr;
    const int* colidx;
    const double* kval;
    const TF* pk_col;          // pivot tile upper triangles, column by column
    const TF* pk_row;          // the same, row by row
    const long long* pk_off;   // per block row
    const unsigned* ndmask;    // per block row: non-unit diagonal entries of the pivot tile
    const TF* dg;              // diagonal of D
    const TF* tri;
    const int* is_piv;
    const int* perm;
    const int* lvl_off;
    const int* lvl_rows;
    const int* bs;
    const int* u_off;
    const int* u_colp;         // U columns mapped through P
    const TF* u_val;
    const int* ut_off;
    const int* ut_col;
    const TF* ut_val;
    const int* rowflags;
    const int* scan_s;         // simple / other block rows per level (factor.h)
    const int* scan_c;
    const int* simple_rows;
    const int* cplx;
    const CItem* citem;        // per entry of cplx: the block row's metadata
    double* v[2];              // v_k and v_k-1, v_k+1 overwrites v_k-1 in place
    double* p[2];              // p_k-1 and p_k-2, p_k overwrites p_k-2 in place
    double* Av;
    double* ev;    // P U^-1 D^-1 (...)
    double* xt;    // the iterate x~ (interleaved)
    double* x;     // the caller's solutions, column-major n x NR
    const double* b;  // the caller's right-hand sides, column-major n x NR
    double* partials;  // 2 buffers x kMaxNV x gridDim
    double* out;       // [0] gamma/norm_pb, [1] iterations, [2] breakdown, [3] converged, [4] norm_pb, [5] it
    unsigned long long* ts;  // optional phase timestamps: [it * 8 + phase], it < kTsIters
    // Level-completion counter of the fused two-level iteration (grid launches
    // only; NULL: a grid synchronisation instead): every CTA adds 1 once its
    // level-1 rows of an iteration are written, level-0 rows wait for
    // G (it + 1) before they read them.  [1]: set when a wait gave up.
    unsigned long long* lvl_done;
    unsigned long long wait_skew;  // added to the wait's target (fault injection in tests; 0)
};

// Bound of one device wait on the level counter: well above any legitimate
// wait (a few microseconds), far below a watchdog.
constexpr unsigned long long kWaitLimitNs = 200ull * 1000 * 1000;

// Shared state of a CTA's level waits: the iteration (+1) whose count the CTA
// has seen, and the iteration (+1) whose poller was elected.
struct LvlWait {
    int seen;
    int poll;
};

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_add_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// One thread spins (acquire loads, backing off) until *ctr >= target; gives up
// after kWaitLimitNs, or at once if an earlier wait gave up, and records that
// in ctr[1].  Returns false when it gave up.
__device__ bool wait_count(unsigned long long* ctr, unsigned long long target)
{
    if (ld_acquire_u64(ctr) >= target) return true;
    volatile unsigned long long* failed = ctr + 1;
    if (*failed) return false;
    unsigned long long t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (unsigned k = 0;; ++k) {
        __nanosleep(k < 8 ? 32 : 256);
        if (ld_acquire_u64(ctr) >= target) return true;
        if ((k & 15) == 15) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (*failed || t - t0 > kWaitLimitNs) {
                *failed = 1;
                return false;
            }
        }
    }
}

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

// scalar state of the recurrence, in shared memory, written by thread 0 only
struct Scal {
    double alpha, alpha_next, beta[3], delta[3], c[3], s[3];
    double norm_A, epsilon, beta_rr, tau, rho, gamma, norm_pb, norm_x, eta;
    double inv_pb, inv_delta, inv_beta, inv_rho;
    double vdv;  // v_k' D^-1 v_k
    int test0, test1, snap0, snap1, done, iters, breakdown, stop_it;
};

__host__ __device__ __forceinline__ int acc3(int r) { return (r % 3) + ((r < 0) ? 3 : 0); }

// Fixed-order sum over the grid (one barrier).  Thread 0 of every CTA gets
// the totals in v, identical in every CTA.  The caller publishes what thread
// 0 derives from them with a __syncthreads() before the next reduction.
template <int NV>
__device__ void grid_reduce(double (&v)[NV], double* partials, int& red, double (*sh)[kW], cg::grid_group& grid)
{
    const int lane = (int)lane_id(), w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(kFull, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][w] = v[k];
    __syncthreads();
    double* buf = partials + (size_t)(red & 1) * kMaxNV * gridDim.x;
    ++red;
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = 0.0;
            for (int i = 0; i < kW; ++i) t += sh[k][i];
            buf[k * gridDim.x + blockIdx.x] = t;
        }
    grid.sync();
    // the NV partials of a CTA position are loaded together (one round trip
    // to L2 for all NV sums); each sum keeps its order over c
    double t[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) t[k] = 0.0;
    for (int c = threadIdx.x; c < (int)gridDim.x; c += kT)
#pragma unroll
        for (int k = 0; k < NV; ++k) t[k] += __ldcg(buf + k * gridDim.x + c);
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        for (int o = 16; o > 0; o >>= 1) t[k] += __shfl_down_sync(kFull, t[k], o);
        if (lane == 0) sh[k][w] = t[k];
    }
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = 0.0;
            for (int i = 0; i < kW; ++i) t += sh[k][i];
            v[k] = t;
        }
}

// D^-1 of one block row (k_solve_D, helper_kernels.impl.cuh:720-774).  With
// 1x1 pivots only the Givens form reduces to y / d exactly (c = sign(d),
// s = 0, r = |d|); a block row with a 2x2 pivot keeps the Givens form, its
// pairs never straddle block rows.  Every lane of the warp calls apply().
template <class TF>
struct DBlock {
    bool two;
    double d;                       // 1x1: the pivot (1 on lanes >= h)
    double gc, gs, tp12, tp22, gr;  // Givens form
    bool ip;

    __device__ __forceinline__ void load(const PArgs<TF>& a, int fr, int h, int flags)
    {
        const int lane = (int)lane_id();
        two = (flags & kRowHas2x2) != 0;
        d = 1.0;
        gc = gs = tp12 = 0.0;
        tp22 = gr = 1.0;
        ip = true;
        if (lane >= h) return;
        const size_t r = (size_t)(fr + lane);
        if (!two) {
            d = (double)__ldg(a.dg + r);
            return;
        }
        ip = __ldg(a.is_piv + r) != 0;
        const bool np = (lane + 1 < h) ? (__ldg(a.is_piv + r + 1) != 0) : true;
        const double p11 = (double)__ldg(a.tri + 3 * r + 1), p12 = (double)__ldg(a.tri + 3 * r + 2);
        const double p22 = !np ? (double)__ldg(a.tri + 3 * (r + 1) + 1) : 1.0;
        gr = sqrt(fma_rn(p11, p11, p12 * p12));
        gc = p11 / gr;
        gs = p12 / gr;
        tp12 = fma_rn(gc, p12, gs * p22);
        tp22 = fma_rn(gc, p22, -(gs * p12));
    }

    __device__ __forceinline__ double apply(double y, int h) const
    {
        const int lane = (int)lane_id();
        if (!two) return (lane < h) ? y / d : 0.0;
        const double ynext = __shfl_down_sync(kFull, y, 1);
        double g1 = 0.0, g2 = 0.0;
        if (lane < h) {
            const double r2 = (lane + 1 < h) ? ynext : 0.0;
            g1 = fma_rn(gc, y, gs * r2);
            g2 = fma_rn(gc, r2, -(gs * y));
            g2 = g2 / tp22;
            g1 = fma_rn(-tp12, g2, g1) / gr;
        }
        const double from_prev = __shfl_up_sync(kFull, g2, 1);
        return ip ? g1 : from_prev;
    }
};

// acc[j] - sum_k val[k] x[col[k] NR + j] in increasing k for the NR
// interleaved right-hand sides (x is written during the kernel: plain loads);
// index / value loads of a batch, then its gathers (the NR values of one
// column are adjacent: 16-byte loads for even NR).  SC: the gathered values
// are stored unscaled and enter as (TF)(x * xs[j]), the value an earlier
// phase would have stored after scaling.
template <class TF, int NR, bool SC = false>
__device__ __forceinline__ void row_sub(TF (&acc)[NR], int k0, int k1, const int* __restrict__ col,
                                        const TF* __restrict__ val, const double* x,
                                        const double* xs = nullptr)
{
    constexpr int B = (NR == 1) ? kBatch : (NR == 2 ? 4 : 2);
    for (int k = k0; k < k1; k += B) {
        int c[B];
        TF v[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            c[j] = (k + j < k1) ? __ldg(col + k + j) : -1;
            v[j] = (k + j < k1) ? __ldg(val + k + j) : TF(0);
        }
        double xv[B][NR];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            if (NR % 2 == 0) {
#pragma unroll
                for (int r = 0; r < NR; r += 2) {
                    double2 q = make_double2(0.0, 0.0);
                    if (c[j] >= 0) q = *reinterpret_cast<const double2*>(x + (size_t)c[j] * NR + r);
                    xv[j][r] = q.x;
                    xv[j][r + 1] = q.y;
                }
            } else {
#pragma unroll
                for (int r = 0; r < NR; ++r) xv[j][r] = (c[j] >= 0) ? x[(size_t)c[j] * NR + r] : 0.0;
            }
        }
#pragma unroll
        for (int j = 0; j < B; ++j)
            if (k + j < k1)
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    acc[r] = fma_rn(-v[j], SC ? (TF)(xv[j][r] * xs[r]) : (TF)xv[j][r], acc[r]);
    }
}

// (K x)_q for the NR interleaved vectors, entries in increasing column order
template <class TF, int NR>
__device__ __forceinline__ void spmv_row(const PArgs<TF>& a, int q, const double* x, double (&acc)[NR])
{
    constexpr int B = (NR == 1) ? kBatch : (NR == 2 ? 4 : 2);
    const int k0 = __ldg(a.rowptr + q), k1 = __ldg(a.rowptr + q + 1);
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.0;
    for (int k = k0; k < k1; k += B) {
        int c[B];
        double v[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            c[j] = (k + j < k1) ? __ldg(a.colidx + k + j) : -1;
            v[j] = (k + j < k1) ? __ldg(a.kval + k + j) : 0.0;
        }
        double xv[B][NR];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            if (NR % 2 == 0) {
#pragma unroll
                for (int r = 0; r < NR; r += 2) {
                    double2 q2 = make_double2(0.0, 0.0);
                    if (c[j] >= 0) q2 = *reinterpret_cast<const double2*>(x + (size_t)c[j] * NR + r);
                    xv[j][r] = q2.x;
                    xv[j][r + 1] = q2.y;
                }
            } else {
#pragma unroll
                for (int r = 0; r < NR; ++r) xv[j][r] = (c[j] >= 0) ? x[(size_t)c[j] * NR + r] : 0.0;
            }
        }
#pragma unroll
        for (int j = 0; j < B; ++j)
            if (k + j < k1)
#pragma unroll
                for (int r = 0; r < NR; ++r) acc[r] = fma_rn(v[j], xv[j][r], acc[r]);
    }
}

// Back substitution with the block row's pivot tile, upper triangle packed
// column by column (U sweep; d_left_solve_row_major,
// block_ildlt_kernels.impl.cuh:2087-2113): for c = h-1 .. 0:
// x_c = t_c / U_cc, t_r -= U_rc x_c (r < c), for each right-hand side.  The
// division is taken only where bit c of nd says U_cc != 1 (t / 1 == t
// exactly); with nd == 0 the chain is shuffle + fma per step.
// SM: P is a copy of the column-packed triangle in shared memory
template <bool SM, class TF>
__device__ __forceinline__ TF tile_ld(const TF* p)
{
    if (SM) return *p;
    return __ldg(p);
}

template <class TF, int NR, bool DIV, bool SM>
__device__ __forceinline__ void tile_upper_t(TF (&t)[NR], const TF* __restrict__ P, int h, unsigned nd)
{
    const int lane = (int)lane_id();
    constexpr int B = (NR == 1) ? kBatch : 4;
    for (int c0 = h - 1; c0 >= 0; c0 -= B) {
        TF u[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            const int c = c0 - j;
            u[j] = (c >= 0 && lane <= c) ? tile_ld<SM>(P + c * (c + 1) / 2 + lane) : TF(0);
        }
#pragma unroll
        for (int j = 0; j < B; ++j) {
            const int c = c0 - j;
            if (c >= 0) {
                if (DIV && ((nd >> c) & 1u)) {
                    if (lane == c)
#pragma unroll
                        for (int r = 0; r < NR; ++r) t[r] = t[r] / u[j];
                }
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    const TF xc = __shfl_sync(kFull, t[r], c);
                    if (lane < c) t[r] = fma_rn(-u[j], xc, t[r]);
                }
            }
        }
    }
}

// Forward substitution with the upper triangle packed row by row (U'
// sweep): for r = 0 .. h-1: x_r = t_r / U_rr, t_c -= U_rc x_r (r < c < h);
// divisions as in tile_upper_t.  With SM the triangle is the column-packed
// copy in shared memory, read along its rows: lane c reads c(c+1)/2 + r, and
// c(c+1)/2 mod 16 is a permutation of 0..15 on each half-warp, so the
// 8-byte reads of a half-warp hit distinct banks.
template <class TF, int NR, bool DIV, bool SM>
__device__ __forceinline__ void tile_lower_t(TF (&t)[NR], const TF* __restrict__ P, int h, unsigned nd)
{
    const int lane = (int)lane_id();
    constexpr int B = (NR == 1) ? kBatch : 4;
    for (int r0 = 0; r0 < h; r0 += B) {
        TF u[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            const int r = r0 + j;
            u[j] = (r < h && lane >= r && lane < h)
                       ? (SM ? P[lane * (lane + 1) / 2 + r] : __ldg(P + r * h - r * (r - 1) / 2 + lane - r))
                       : TF(0);
        }
#pragma unroll
        for (int j = 0; j < B; ++j) {
            const int r = r0 + j;
            if (r < h) {
                if (DIV && ((nd >> r) & 1u)) {
                    if (lane == r)
#pragma unroll
                        for (int q = 0; q < NR; ++q) t[q] = t[q] / u[j];
                }
#pragma unroll
                for (int q = 0; q < NR; ++q) {
                    const TF xr = __shfl_sync(kFull, t[q], r);
                    if (lane > r && lane < h) t[q] = fma_rn(-u[j], xr, t[q]);
                }
            }
        }
    }
}

template <class TF, int NR, bool SM = false>
__device__ __forceinline__ void tile_upper(double (&v)[NR], const TF* P, int h, unsigned nd)
{
    TF t[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) t[r] = (TF)v[r];
    if (nd) tile_upper_t<TF, NR, true, SM>(t, P, h, nd);
    else tile_upper_t<TF, NR, false, SM>(t, P, h, 0u);
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = (double)t[r];
}

template <class TF, int NR, bool SM = false>
__device__ __forceinline__ void tile_lower(double (&v)[NR], const TF* P, int h, unsigned nd)
{
    TF t[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) t[r] = (TF)v[r];
    if (nd) tile_lower_t<TF, NR, true, SM>(t, P, h, nd);
    else tile_lower_t<TF, NR, false, SM>(t, P, h, 0u);
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = (double)t[r];
}

// A work item's block-row metadata
struct ItemMeta {
    int I, fr, h, flags;
    long long pko;
    unsigned nd;
};

// from the block row (sweeps over every block row of a level)
template <class TF>
__device__ __forceinline__ ItemMeta meta_of_row(const PArgs<TF>& a, int I)
{
    ItemMeta m;
    m.I = I;
    m.fr = __ldg(a.bs + I);
    m.h = __ldg(a.bs + I + 1) - m.fr;
    m.flags = __ldg(a.rowflags + I);
    m.pko = __ldg(a.pk_off + I);
    m.nd = __ldg(a.ndmask + I);
    return m;
}

// from entry t of the pivot-tile block rows: two independent 16-byte loads
// instead of the chain cplx -> (bs, rowflags, pk_off, ndmask)
template <class TF>
__device__ __forceinline__ ItemMeta meta_of_item(const PArgs<TF>& a, int t)
{
    const int4* p = reinterpret_cast<const int4*>(a.citem + t);
    const int4 u = __ldg(p), w = __ldg(p + 1);
    ItemMeta m;
    m.I = u.x;
    m.fr = u.y;
    m.h = u.z;
    m.flags = u.w;
    m.pko = (long long)(((unsigned long long)(unsigned)w.y << 32) | (unsigned)w.x);
    m.nd = (unsigned)w.z;
    return m;
}

// Shared-memory copy of one warp's pivot-tile work item, loaded once per
// solve.  Each warp of the persistent kernel keeps the same item of a level
// for the whole solve (item c0 + wid), so the level with the most such items
// keeps, per warp slot, the item's metadata, its lanes' permuted rows and U /
// U' row ranges, D's diagonal (block rows without 2x2 pivots) and the pivot
// tile's upper triangle (column-packed).  The item's per-iteration chain of
// dependent loads (descriptor, permutation and offsets, four batches of tile
// values, D) becomes shared-memory reads.
constexpr int kResSlots = 12;  // warps per CTA with a resident item
constexpr int kTileMax = 32 * 33 / 2;

template <class TF>
struct ResSlot {
    ItemMeta m;  // m.h == 0: the warp has no item of the resident level
    int q[32];   // perm[fr + lane]
    int u0[32], u1[32], ut0[32], ut1[32];
    double d[32];
    TF tile[kTileMax];
};

// warp-collective: fills the slot with item t of the citem list (has) or marks it empty
template <class TF>
__device__ void res_load(const PArgs<TF>& a, ResSlot<TF>& rs, int t, bool has)
{
    const int lane = (int)lane_id();
    if (!has) {
        if (lane == 0) rs.m.h = 0;
        return;
    }
    const ItemMeta m = meta_of_item(a, t);
    if (lane == 0) rs.m = m;
    const int fr = m.fr, h = m.h;
    if (lane < h) {
        const int g = fr + lane;
        rs.q[lane] = (m.flags & kRowPermIdentity) ? g : __ldg(a.perm + g);
        rs.u0[lane] = __ldg(a.u_off + g);
        rs.u1[lane] = __ldg(a.u_off + g + 1);
        rs.ut0[lane] = __ldg(a.ut_off + g);
        rs.ut1[lane] = __ldg(a.ut_off + g + 1);
        rs.d[lane] = (m.flags & kRowHas2x2) ? 1.0 : (double)__ldg(a.dg + g);
    }
    if (!(m.flags & kRowIdentity))
        for (int e = lane; e < h * (h + 1) / 2; e += 32) rs.tile[e] = __ldg(a.pk_col + m.pko + e);
}

// D of a resident item: its diagonal from the slot, or the Givens form from
// global memory when the block row has a 2x2 pivot
template <class TF>
__device__ __forceinline__ DBlock<TF> dblock_res(const PArgs<TF>& a, const ResSlot<TF>& rs)
{
    DBlock<TF> D;
    const int flags = rs.m.flags, h = rs.m.h;
    if (flags & kRowHas2x2) {
        D.load(a, rs.m.fr, h, flags);
        return D;
    }
    const int lane = (int)lane_id();
    D.two = false;
    D.d = (lane < h) ? rs.d[lane] : 1.0;
    D.gc = D.gs = D.tp12 = 0.0;
    D.tp22 = D.gr = 1.0;
    D.ip = true;
    return D;
}

// One U-sweep work item: block row I (rows fr .. fr+h-1), lane's right-hand
// sides y: d = D^-1 y; t = U_II^-1 (d - U_I* t); out[perm[r]] = t (NR
// interleaved).  The gathers of the later levels' t read out through the
// permuted columns.  d receives D^-1 y (0 on lanes >= h).
template <class TF, int NR>
__device__ __forceinline__ void u_item(const PArgs<TF>& a, const ItemMeta& m, const double (&y)[NR], double* out,
                                       double (&d)[NR])
{
    const int lane = (int)lane_id();
    const int fr = m.fr, h = m.h, flags = m.flags;
    DBlock<TF> D;
    D.load(a, fr, h, flags);
#pragma unroll
    for (int r = 0; r < NR; ++r) d[r] = D.apply(y[r], h);
    double t[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) t[r] = d[r];
    if (lane < h) {
        TF acc[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] = (TF)d[r];
        row_sub<TF, NR>(acc, __ldg(a.u_off + fr + lane), __ldg(a.u_off + fr + lane + 1), a.u_colp, a.u_val, out);
#pragma unroll
        for (int r = 0; r < NR; ++r) t[r] = (double)acc[r];
    }
    if (!(flags & kRowIdentity)) tile_upper<TF, NR>(t, a.pk_col + m.pko, h, m.nd);
    if (lane < h) {
        const int q = (flags & kRowPermIdentity) ? fr + lane : __ldg(a.perm + fr + lane);
#pragma unroll
        for (int r = 0; r < NR; ++r) out[(size_t)q * NR + r] = t[r];
    }
}

// Where a U'-sweep item's right-hand side comes from
enum RhsFrom {
    kRhsCaller = 0,  // b[r n + perm[row]] of the caller's column-major right-hand sides
    kRhsSpmv = 1,    // sc[r] * (K src)[perm[row]], src interleaved
    kRhsPre = 2,     // dst[perm[row]]: sc (K src) stored there by an earlier phase
};

// One U'-sweep work item: dst[row] = U_II'^-1 (rhs - U'_I* dst) (interleaved)
// with the lane's right-hand sides taken as FROM says.  t receives the
// lane's results (0 for lanes >= h).
template <class TF, int NR, int FROM, bool SCG = false>
__device__ __forceinline__ void ut_item(const PArgs<TF>& a, const ItemMeta& m, const double* src,
                                        const double (&sc)[NR], double* dst, double (&t)[NR])
{
    const int lane = (int)lane_id();
    const int fr = m.fr, h = m.h, flags = m.flags;
#pragma unroll
    for (int r = 0; r < NR; ++r) t[r] = 0.0;
    if (lane < h) {
        const int q = (flags & kRowPermIdentity) ? fr + lane : __ldg(a.perm + fr + lane);
        double y[NR];
        if (FROM == kRhsSpmv) {
            spmv_row<TF, NR>(a, q, src, y);
#pragma unroll
            for (int r = 0; r < NR; ++r) y[r] *= sc[r];
        } else if (FROM == kRhsPre) {
#pragma unroll
            for (int r = 0; r < NR; ++r) y[r] = dst[(size_t)q * NR + r];
        } else {
#pragma unroll
            for (int r = 0; r < NR; ++r) y[r] = src[(size_t)r * a.n + q];
        }
        TF acc[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] = (TF)y[r];
        row_sub<TF, NR, SCG>(acc, __ldg(a.ut_off + fr + lane), __ldg(a.ut_off + fr + lane + 1), a.ut_col, a.ut_val,
                             dst, sc);
#pragma unroll
        for (int r = 0; r < NR; ++r) t[r] = (double)acc[r];
    }
    // with kRhsPre the lanes read dst inside this block row: all reads before any write
    if (FROM == kRhsPre) __syncwarp();
    if (!(flags & kRowIdentity)) tile_lower<TF, NR>(t, a.pk_row + m.pko, h, m.nd);
    if (lane < h)
#pragma unroll
        for (int r = 0; r < NR; ++r) dst[(size_t)(fr + lane) * NR + r] = t[r];
}

// u_item / ut_item of a resident item (same arithmetic, data from the slot)
template <class TF, int NR>
__device__ __forceinline__ void u_item_res(const PArgs<TF>& a, const ResSlot<TF>& rs, const double (&y)[NR],
                                           double* out, double (&d)[NR])
{
    const int lane = (int)lane_id();
    const int h = rs.m.h, flags = rs.m.flags;
    const DBlock<TF> D = dblock_res(a, rs);
#pragma unroll
    for (int r = 0; r < NR; ++r) d[r] = D.apply(y[r], h);
    double t[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) t[r] = d[r];
    if (lane < h) {
        TF acc[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] = (TF)d[r];
        row_sub<TF, NR>(acc, rs.u0[lane], rs.u1[lane], a.u_colp, a.u_val, out);
#pragma unroll
        for (int r = 0; r < NR; ++r) t[r] = (double)acc[r];
    }
    if (!(flags & kRowIdentity)) tile_upper<TF, NR, true>(t, rs.tile, h, rs.m.nd);
    if (lane < h) {
        const int q = rs.q[lane];
#pragma unroll
        for (int r = 0; r < NR; ++r) out[(size_t)q * NR + r] = t[r];
    }
}

template <class TF, int NR, int FROM, bool SCG = false>
__device__ __forceinline__ void ut_item_res(const PArgs<TF>& a, const ResSlot<TF>& rs, const double* src,
                                            const double (&sc)[NR], double* dst, double (&t)[NR])
{
    const int lane = (int)lane_id();
    const int fr = rs.m.fr, h = rs.m.h, flags = rs.m.flags;
#pragma unroll
    for (int r = 0; r < NR; ++r) t[r] = 0.0;
    if (lane < h) {
        const int q = rs.q[lane];
        double y[NR];
        if (FROM == kRhsSpmv) {
            spmv_row<TF, NR>(a, q, src, y);
#pragma unroll
            for (int r = 0; r < NR; ++r) y[r] *= sc[r];
        } else if (FROM == kRhsPre) {
#pragma unroll
            for (int r = 0; r < NR; ++r) y[r] = dst[(size_t)q * NR + r];
        } else {
#pragma unroll
            for (int r = 0; r < NR; ++r) y[r] = src[(size_t)r * a.n + q];
        }
        TF acc[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] = (TF)y[r];
        row_sub<TF, NR, SCG>(acc, rs.ut0[lane], rs.ut1[lane], a.ut_col, a.ut_val, dst, sc);
#pragma unroll
        for (int r = 0; r < NR; ++r) t[r] = (double)acc[r];
    }
    if (FROM == kRhsPre) __syncwarp();
    if (!(flags & kRowIdentity)) tile_lower<TF, NR, true>(t, rs.tile, h, rs.m.nd);
    if (lane < h)
#pragma unroll
        for (int r = 0; r < NR; ++r) dst[(size_t)(fr + lane) * NR + r] = t[r];
}

__device__ double sgn(double v) { return v < 0 ? -1.0 : 1.0; }

// k_sym_ortho (helper_kernels.impl.cuh:662-700)
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

// Fixed-order sum over one CTA: thread 0 gets the totals (same protocol as
// grid_reduce).
template <int NV>
__device__ void cta_reduce(double (&v)[NV], double (*sh)[kW])
{
    const int lane = (int)lane_id(), w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(kFull, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][w] = v[k];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = 0.0;
            for (int i = 0; i < kW; ++i) t += sh[k][i];
            v[k] = t;
        }
}

// Where one solve runs: the whole grid of a cooperative launch (one system)
// or one CTA of a batched launch (one system per CTA at a time).  Work items
// go to warps wid, wid + nwarps, ...; vector loops to threads g0, g0 + gstride.
struct GridCtx {
    cg::grid_group grid;
    double* partials;
    int red;
    int wid, nwarps, g0, gstride;
    __device__ void sync() { grid.sync(); }
    template <int NV>
    __device__ void reduce(double (&v)[NV], double (*sh)[kW])
    {
        grid_reduce<NV>(v, partials, red, sh, grid);
    }
};

struct CtaCtx {
    int wid, nwarps, g0, gstride;
    __device__ void sync() const { __syncthreads(); }
    template <int NV>
    __device__ void reduce(double (&v)[NV], double (*sh)[kW])
    {
        cta_reduce<NV>(v, sh);
    }
};

// The system a solve works on: its rows [row0, row1) and, for each level L,
// its block rows' positions [qb[L], qe[L]) in the level lists; out receives
// per right-hand side r at out + 8 r: [0] gamma/norm_pb, [1] iterations,
// [2] breakdown, [3] converged, [4] norm_pb, [5] it.
struct SysView {
    int row0, row1;
    const int* qb;
    const int* qe;
    double* out;
};

// Per-RHS coefficients of the p / x update and of the dots' scaling
template <int NR>
struct Coef {
    double sc[NR], nbrr[NR], ne[NR], ir[NR], tau[NR];
    double na[NR], nb[NR];  // the U sweep's -alpha, -beta_k
    const double* vk;       // the iteration's v_k, v_k+1 (= v_k-1 on entry), p_k (= p_k-2 on entry), p_k-1
    double* vk1;
    double* pk;
    const double* pkm1;
    bool act[NR];  // right-hand sides still iterating (x of the others is final)
};

// Per-row tail of the U' sweep for a row of a simple block row (1x1 pivot
// d): v+ scaled in place, beta's numerator v_k' D^-1 Av, the next alpha's
// dots v+' D^-1 Av and v+' D^-1 v+, and p_k = (v_k - beta_rr p_k-1 -
// epsilon p_k-2) / rho, x += tau p_k with ||x||^2 (r[k NR + rhs]).
template <class TF, int NR>
__device__ __forceinline__ void simple_epilogue(const PArgs<TF>& a, int g, const double (&av)[NR], const double* vk,
                                                double* vk1, const double* pkm1, const double* pkm2, double* pk,
                                                const volatile Coef<NR>& cf, double (&r)[4 * NR])
{
    const double dd = (double)__ldg(a.dg + g);
#pragma unroll
    for (int j = 0; j < NR; ++j) {
        const size_t o = (size_t)g * NR + j;
        const double vkr = vk[o];
        const double vs = vk1[o] * cf.sc[j];
        vk1[o] = vs;
        if (cf.act[j]) {
            double p = vkr;
            p = fma_rn(cf.nbrr[j], pkm1[o], p);
            p = fma_rn(cf.ne[j], pkm2[o], p);
            p = p * cf.ir[j];
            pk[o] = p;
            const double xv = fma_rn(cf.tau[j], p, a.xt[o]);
            a.xt[o] = xv;
            r[3 * NR + j] = fma_rn(xv, xv, r[3 * NR + j]);
        }
        const double da = av[j] / dd, dv = vs / dd;
        r[j] = fma_rn(vkr, da, r[j]);
        r[NR + j] = fma_rn(vs, da, r[NR + j]);
        r[2 * NR + j] = fma_rn(vs, dv, r[2 * NR + j]);
    }
}

// The whole preconditioned SQMR solve of one system for NR right-hand sides
// at once (see the top of the file): every work item loads the factor and
// K once for all of them; each right-hand side has its own scalars and stops
// on its own test (its x is final from then on).
// A level's work lists: pivot-tile items [c0, c1) of citem, simple rows
// [s0, s1) of simple_rows.  The first kLvlCache levels' bounds are kept in
// shared memory for the whole solve (each phase starts by reading them).
struct LvlBounds {
    int c0, c1, s0, s1;
};
constexpr int kLvlCache = 32;

template <class TF>
__device__ __forceinline__ LvlBounds level_bounds(const PArgs<TF>& a, const SysView& sv, int L)
{
    const int q0 = __ldg(sv.qb + L), q1 = __ldg(sv.qe + L);
    return LvlBounds{__ldg(a.scan_c + q0), __ldg(a.scan_c + q1), __ldg(a.scan_s + q0), __ldg(a.scan_s + q1)};
}

template <class TF, int NR, class Ctx>
__device__ void sqmr_body(const PArgs<TF>& a, Ctx& ctx, const SysView& sv, Scal (&S)[NR], double (*sh)[kW],
                          ResSlot<TF>* slots = nullptr)
{
    const int tid = threadIdx.x, lane = (int)lane_id();
    const int wid = ctx.wid, nwarps = ctx.nwarps;
    const int row0 = sv.row0, row1 = sv.row1;
    __shared__ Coef<NR> cfs;  // the U' phase's coefficients, written by thread 0
    __shared__ LvlBounds lvb[kLvlCache];
    __shared__ long long npre_s;  // rows of the pivot-tile items of levels >= 1
    if (tid < kLvlCache && tid < a.nl) lvb[tid] = level_bounds(a, sv, tid);
    if (tid == 0) {
        for (int j = 0; j < NR; ++j) {
            memset(&S[j], 0, sizeof(Scal));
            S[j].c[0] = -1.0;
            cfs.sc[j] = 1.0;  // the scale of the Av that the initial phase leaves
        }
        long long np = 0;
        for (int L = 1; L < a.nl; ++L) {
            const LvlBounds b = level_bounds(a, sv, L);
            np += 32LL * (b.c1 - b.c0);
        }
        npre_s = np;
    }
    __syncthreads();
    auto lvl = [&](int L) -> LvlBounds { return L < kLvlCache ? lvb[L] : level_bounds(a, sv, L); };
    // Two levels, level 0 all simple block rows whose K rows reach only
    // themselves and level-1 rows (a natural-order KKT system): each level-0
    // row computes its (K ev) in the U sweep, right after its ev, and the U'
    // sweep's level-0 phase and its barrier go away.  Level-0 Av is then kept
    // unscaled (the 1/delta it needs is known only after the U sweep's
    // reduction); every reader applies the scale of the iteration that wrote
    // it, at the point where the unfused path rounded it, so the results are
    // the unfused path's bit for bit.
    const bool fused = a.fuse_l0 && a.nl == 2 && lvb[0].c1 == lvb[0].c0;
    // fused grid launches hand level 1 to level 0 through the level counter
    const bool counted = fused && a.lvl_done != nullptr;
    if (counted && blockIdx.x == 0 && tid == 0) {
        a.lvl_done[0] = 0;  // read only after the initial phases' grid synchronisations
        a.lvl_done[1] = 0;
    }
    __shared__ LvlWait lw;
    if (tid == 0) {
        lw.seen = 0;
        lw.poll = 0;
    }
    // the calling warp's active lanes wait until the count for iteration it is
    // reached: the first warp of the CTA to get here polls global memory, the
    // others watch the CTA's shared flag; then every lane reads the counter
    // itself with an acquire load and checks it (at once satisfied, or at once
    // given up after a timeout), which orders its own later loads after every
    // CTA's release
    auto level_wait = [&](int it) {
        const unsigned mask = __activemask();
        const int want = it + 1;
        const unsigned long long target = (unsigned long long)gridDim.x * (unsigned long long)want + a.wait_skew;
        const int leader = __ffs(mask) - 1;
        if (*(volatile int*)&lw.seen < want && lane == leader) {
            if (atomicMax(&lw.poll, want) < want) {
                wait_count(a.lvl_done, target);
                __threadfence_block();
                *(volatile int*)&lw.seen = want;
            } else {
                unsigned long long t0, t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
                for (unsigned k = 0; *(volatile int*)&lw.seen < want; ++k) {
                    __nanosleep(64);
                    if ((k & 15) == 15) {
                        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                        if (t - t0 > 2 * kWaitLimitNs) {
                            *(volatile unsigned long long*)(a.lvl_done + 1) = 1;
                            break;
                        }
                    }
                }
            }
        }
        __syncwarp(mask);
        wait_count(a.lvl_done, target);
    };

    // the level with the most pivot-tile items keeps its first kResSlots x
    // (grid) items in the warps' shared-memory slots
    __shared__ int res_level_s;
    if (tid == 0) {
        int best = -1, most = 0;
        if (slots)
            for (int L = 0; L < a.nl; ++L) {
                const LvlBounds b = lvl(L);
                if (b.c1 - b.c0 > most) {
                    most = b.c1 - b.c0;
                    best = L;
                }
            }
        res_level_s = best;
    }
    __syncthreads();
    const int res_level = res_level_s;
    ResSlot<TF>* const rs = (res_level >= 0 && (tid >> 5) < kResSlots) ? slots + (tid >> 5) : nullptr;
    int res_t = -1;  // the item of the resident level this warp holds
    if (rs) {
        const LvlBounds rb = lvl(res_level);
        const int t = rb.c0 + wid;
        res_load(a, *rs, t, t < rb.c1);
        if (t < rb.c1) res_t = t;
    }
    __syncthreads();

    // ---- init: v0 = U'^-1 P' b; ||v0|| ----
    {
        double one[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) one[j] = 1.0;
        for (int L = 0; L < a.nl; ++L) {
            const int r0 = __ldg(sv.qb + L), nr = __ldg(sv.qe + L) - r0;
            for (int t = wid; t < nr; t += nwarps) {
                const ItemMeta m = meta_of_row(a, __ldg(a.lvl_rows + r0 + t));
                double tt[NR];
                ut_item<TF, NR, kRhsCaller>(a, m, a.b, one, a.v[0], tt);
            }
            ctx.sync();
        }
    }
    {
        double r[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) r[j] = 0.0;
        for (int g = row0 + ctx.g0; g < row1; g += ctx.gstride)
#pragma unroll
            for (int j = 0; j < NR; ++j) r[j] = fma_rn(a.v[0][(size_t)g * NR + j], a.v[0][(size_t)g * NR + j], r[j]);
        ctx.template reduce<NR>(r, sh);
        if (tid == 0)
            for (int j = 0; j < NR; ++j) {
                S[j].norm_pb = sqrt(r[j]);
                S[j].gamma = S[j].norm_pb;
                S[j].inv_pb = 1.0 / S[j].norm_pb;
            }
        __syncthreads();
    }
    // v0 /= ||v0|| (in place), ev = P U^-1 D^-1 v0, ||D^-1 v0||^2
    double ww[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) ww[j] = 0.0;
    {
        double inv_pb[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) inv_pb[j] = S[j].inv_pb;
        for (int L = a.nl - 1; L >= 0; --L) {
            const int r0 = __ldg(sv.qb + L), nr = __ldg(sv.qe + L) - r0;
            for (int t = wid; t < nr; t += nwarps) {
                const ItemMeta m = meta_of_row(a, __ldg(a.lvl_rows + r0 + t));
                const int fr = m.fr, h = m.h;
                double y[NR], d[NR];
#pragma unroll
                for (int j = 0; j < NR; ++j) {
                    y[j] = 0.0;
                    if (lane < h) {
                        const size_t o = (size_t)(fr + lane) * NR + j;
                        y[j] = a.v[0][o] * inv_pb[j];
                        a.v[0][o] = y[j];
                    }
                }
                u_item<TF, NR>(a, m, y, a.ev, d);
#pragma unroll
                for (int j = 0; j < NR; ++j) ww[j] = fma_rn(d[j], d[j], ww[j]);
            }
            ctx.sync();
        }
    }
    // Av = U'^-1 P' K ev; alpha's dots for iteration 0; eta_0 = 1/||D^-1 v0||
    {
        double r[3 * NR];
        double one[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            r[j] = ww[j];
            r[NR + j] = 0.0;
            r[2 * NR + j] = 0.0;
            one[j] = 1.0;
        }
        for (int L = 0; L < a.nl; ++L) {
            const int r0 = __ldg(sv.qb + L), nr = __ldg(sv.qe + L) - r0;
            for (int t = wid; t < nr; t += nwarps) {
                const ItemMeta m = meta_of_row(a, __ldg(a.lvl_rows + r0 + t));
                const int fr = m.fr, h = m.h, flags = m.flags;
                double av[NR];
                ut_item<TF, NR, kRhsSpmv>(a, m, a.ev, one, a.Av, av);
                DBlock<TF> D;
                D.load(a, fr, h, flags);
#pragma unroll
                for (int j = 0; j < NR; ++j) {
                    const double vs = (lane < h) ? a.v[0][(size_t)(fr + lane) * NR + j] : 0.0;
                    const double da = D.apply(av[j], h), dv = D.apply(vs, h);
                    if (lane < h) {
                        r[NR + j] = fma_rn(vs, da, r[NR + j]);
                        r[2 * NR + j] = fma_rn(vs, dv, r[2 * NR + j]);
                    }
                }
            }
            if (L < a.nl - 1) ctx.sync();
        }
        ctx.template reduce<3 * NR>(r, sh);
        if (tid == 0)
            for (int j = 0; j < NR; ++j) {
                S[j].eta = 1.0 / sqrt(r[j]);
                S[j].alpha_next = r[NR + j] / r[2 * NR + j];
                S[j].vdv = r[2 * NR + j];
                if (!isfinite(S[j].inv_pb) || !isfinite(S[j].eta)) {
                    S[j].breakdown = 1;
                    S[j].done = 1;
                }
            }
        __syncthreads();
    }

    int it = 0;
    for (;;) {
        bool any = false;
#pragma unroll
        for (int j = 0; j < NR; ++j) any |= !S[j].done;
        if (!any || it >= a.max_it) break;
        const int k0 = acc3(it), k1 = acc3(it + 1), km1 = acc3(it - 1);
        if (NR == 1) stamp(a.ts, it, 0);
        // -alpha and -beta_k of each right-hand side, read from shared memory
        // where used (registers are the kernel's scarce resource)
        if (tid == 0) {
            for (int j = 0; j < NR; ++j) {
                cfs.na[j] = -S[j].alpha_next;
                cfs.nb[j] = -S[j].beta[k0];
            }
            cfs.vk = a.v[it & 1];
            cfs.vk1 = a.v[(it + 1) & 1];
            cfs.pk = a.p[it & 1];
            cfs.pkm1 = a.p[(it + 1) & 1];
        }
        __syncthreads();
        const volatile Coef<NR>& cv = cfs;
        const volatile double* const na = cfs.na;
        const volatile double* const nb = cfs.nb;
        // ---- U sweep on v+ = Av - alpha v - beta v- (each item computes and
        //      stores its rows' v+, kept unscaled), ||v+||^2 ----
        {
            double r[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) r[j] = 0.0;
            for (int L = a.nl - 1; L >= 0; --L) {
                const LvlBounds lb = lvl(L);
                // block rows with a pivot tile, swaps or 2x2 pivots: warp per block row
                const int c1 = lb.c1;
                for (int t = lb.c0 + wid; t < c1; t += nwarps) {
                    const bool res = (t == res_t && L == res_level);
                    const ItemMeta m = res ? rs->m : meta_of_item(a, t);
                    const int fr = m.fr, h = m.h;
                    double y[NR], d[NR];
#pragma unroll
                    for (int j = 0; j < NR; ++j) {
                        y[j] = 0.0;
                        if (lane < h) {
                            const size_t o = (size_t)(fr + lane) * NR + j;
                            double v = a.Av[o];
                            double* const vk1 = cv.vk1;  // vk1 holds v_k-1 until written
                            v = fma_rn(na[j], cv.vk[o], v);
                            v = fma_rn(nb[j], vk1[o], v);
                            vk1[o] = v;
                            r[j] = fma_rn(v, v, r[j]);
                            y[j] = v;
                        }
                    }
                    if (res) u_item_res<TF, NR>(a, *rs, y, a.ev, d);
                    else u_item<TF, NR>(a, m, y, a.ev, d);
                }
                // rows of simple block rows: thread per row (u_item with D = d,
                // an identity tile and no swaps)
                const int s1 = lb.s1;
                const bool fz = fused && L == 0;
                bool ready = !(counted && L == 0);
                for (int i = lb.s0 + ctx.g0; i < s1; i += ctx.gstride) {
                    const int g = __ldg(a.simple_rows + i);
                    const double dd = (double)__ldg(a.dg + g);
                    TF acc[NR];
#pragma unroll
                    for (int j = 0; j < NR; ++j) {
                        const size_t o = (size_t)g * NR + j;
                        // fused level 0: Av holds the last iteration's unscaled (K ev)
                        double v = fz ? (double)(TF)(a.Av[o] * cv.sc[j]) : a.Av[o];
                        double* const vk1 = cv.vk1;
                        v = fma_rn(na[j], cv.vk[o], v);
                        v = fma_rn(nb[j], vk1[o], v);
                        vk1[o] = v;
                        r[j] = fma_rn(v, v, r[j]);
                        acc[j] = (TF)(v / dd);
                    }
                    if (!ready) {
                        // v+ and D^-1 v+ above need no level-1 value; the gathers below do
                        level_wait(it);
                        ready = true;
                    }
                    row_sub<TF, NR>(acc, __ldg(a.u_off + g), __ldg(a.u_off + g + 1), a.u_colp, a.u_val, a.ev);
#pragma unroll
                    for (int j = 0; j < NR; ++j) a.ev[(size_t)g * NR + j] = (double)acc[j];
                    if (fz) {
                        // K row g reaches only ev[g] (written just above) and level-1
                        // rows (final since the last barrier)
                        double y[NR];
                        spmv_row<TF, NR>(a, g, a.ev, y);
#pragma unroll
                        for (int j = 0; j < NR; ++j) a.Av[(size_t)g * NR + j] = y[j];
                    }
                }
                if (L > 0) {
                    if (counted) {
                        // this CTA's level-1 rows are written: count it (release);
                        // level-0 rows wait for every CTA's count before reading them
                        __syncthreads();
                        if (tid == 0) red_release_add_u64(a.lvl_done, 1ull);
                    } else {
                        ctx.sync();
                    }
                    if (NR == 1 && L == a.nl - 1) stamp(a.ts, it, 1);
                }
            }
            ctx.template reduce<NR>(r, sh);
            if (tid == 0)
                for (int j = 0; j < NR; ++j) {
                    if (S[j].done) continue;
                    Scal& Q = S[j];
                    const double alpha = Q.alpha_next;
                    Q.alpha = alpha;
                    const double bk = Q.beta[k0];
                    const double dl = sqrt(r[j]);
                    Q.delta[k1] = dl;
                    Q.inv_delta = 1.0 / dl;
                    const double nA = sqrt(fma_rn(dl, dl, fma_rn(alpha, alpha, bk * bk)));
                    Q.norm_A = fmax(Q.norm_A, nA);
                    Q.epsilon = Q.s[km1] * bk;
                    const double beta_rot = (-Q.c[km1]) * bk;
                    Q.beta_rr = fma_rn(Q.c[k0], beta_rot, Q.s[k0] * alpha);
                    const double alpha_rot = fma_rn(Q.s[k0], beta_rot, (-Q.c[k0]) * alpha);
                    double c, s, rr;
                    sym_ortho(alpha_rot, dl, c, s, rr);
                    Q.c[k1] = c;
                    Q.s[k1] = s;
                    Q.rho = rr;
                    Q.inv_rho = 1.0 / rr;
                    Q.tau = c * Q.gamma;
                    Q.gamma = s * Q.gamma;
                }
            if (tid == 0)
                for (int j = 0; j < NR; ++j) {
                    cfs.sc[j] = S[j].inv_delta;
                    cfs.nbrr[j] = -S[j].beta_rr;
                    cfs.ne[j] = -S[j].epsilon;
                    cfs.ir[j] = S[j].inv_rho;
                    cfs.tau[j] = S[j].tau;
                    cfs.act[j] = !S[j].done;
                }
            __syncthreads();
        }
        if (NR == 1) {
            if (a.nl == 1) stamp(a.ts, it, 1);
            stamp(a.ts, it, 2);
        }
        // ---- U' sweep with the fused SpMV; beta's and alpha's dots; p, x ----
        {
            double r[4 * NR];
#pragma unroll
            for (int j = 0; j < 4 * NR; ++j) r[j] = 0.0;
            const volatile Coef<NR>& cf = cfs;
            for (int L = 0; L < a.nl; ++L) {
                // fused: level 0 has no items and its rows' products are done
                if (fused && L == 0) continue;
                const LvlBounds lb = lvl(L);
                const int c1 = lb.c1;
                for (int t = lb.c0 + wid; t < c1; t += nwarps) {
                    const bool res = (t == res_t && L == res_level);
                    const ItemMeta m = res ? rs->m : meta_of_item(a, t);
                    const int fr = m.fr, h = m.h, flags = m.flags;
                    double av[NR];
                    double scv[NR];
#pragma unroll
                    for (int j = 0; j < NR; ++j) scv[j] = cf.sc[j];
                    DBlock<TF> D;
                    if (res) {
                        if (fused) ut_item_res<TF, NR, kRhsSpmv, true>(a, *rs, a.ev, scv, a.Av, av);
                        else if (L == 0) ut_item_res<TF, NR, kRhsSpmv>(a, *rs, a.ev, scv, a.Av, av);
                        else ut_item_res<TF, NR, kRhsPre>(a, *rs, a.ev, scv, a.Av, av);
                        D = dblock_res(a, *rs);
                    } else {
                        if (fused) ut_item<TF, NR, kRhsSpmv, true>(a, m, a.ev, scv, a.Av, av);
                        else if (L == 0) ut_item<TF, NR, kRhsSpmv>(a, m, a.ev, scv, a.Av, av);
                        else ut_item<TF, NR, kRhsPre>(a, m, a.ev, scv, a.Av, av);
                        D.load(a, fr, h, flags);
                    }
#pragma unroll
                    for (int j = 0; j < NR; ++j) {
                        double vkr = 0.0, vs = 0.0;
                        if (lane < h) {
                            const size_t o = (size_t)(fr + lane) * NR + j;
                            double* const vk1 = cv.vk1;
                            vkr = cv.vk[o];
                            vs = vk1[o] * cf.sc[j];
                            vk1[o] = vs;
                            if (cf.act[j]) {
                                // p_k = (v_k - beta_rr p_k-1 - epsilon p_k-2) / rho, x += tau p_k
                                double p = vkr;
                                double* const pk = cv.pk;  // holds p_k-2 until written
                                p = fma_rn(cf.nbrr[j], cv.pkm1[o], p);
                                p = fma_rn(cf.ne[j], pk[o], p);
                                p = p * cf.ir[j];
                                pk[o] = p;
                                const double xv = fma_rn(cf.tau[j], p, a.xt[o]);
                                a.xt[o] = xv;
                                r[3 * NR + j] = fma_rn(xv, xv, r[3 * NR + j]);
                            }
                        }
                        const double da = D.apply(av[j], h), dv = D.apply(vs, h);
                        if (lane < h) {
                            r[j] = fma_rn(vkr, da, r[j]);
                            r[NR + j] = fma_rn(vs, da, r[NR + j]);
                            r[2 * NR + j] = fma_rn(vs, dv, r[2 * NR + j]);
                        }
                    }
                }
                // simple rows of this level: Av; their dots and the p / x
                // update wait for the next level's phase, whose threads are
                // mostly free (the last level does them at once)
                const bool last = (L == a.nl - 1);
                const int s0 = lb.s0, s1 = lb.s1;
                // Level 0 also computes (K ev) / delta for the rows of the later
                // levels' pivot-tile block rows and leaves it in Av at those rows:
                // their items read it there instead of running the product on
                // the critical path of a level of few, long items.  Units
                // [0, npre) are those rows (lane ln of item t), the rest this
                // level's simple rows, both spread over all threads.
                const long long npre = (L == 0) ? npre_s : 0;
                const long long nunits = npre + (s1 - s0);
                for (long long k = ctx.g0; k < nunits; k += ctx.gstride) {
                    if (k < npre) {
                        long long u = k;
                        int L2 = 1;
                        LvlBounds b2 = lvl(L2);
                        for (;;) {
                            const long long len = 32LL * (b2.c1 - b2.c0);
                            if (u < len) break;
                            u -= len;
                            b2 = lvl(++L2);
                        }
                        const ItemMeta m = meta_of_item(a, b2.c0 + (int)(u >> 5));
                        const int ln = (int)(u & 31), fr = m.fr;
                        if (ln < m.h) {
                            double y[NR];
                            spmv_row<TF, NR>(a, fr + ln, a.ev, y);
#pragma unroll
                            for (int j = 0; j < NR; ++j) a.Av[(size_t)(fr + ln) * NR + j] = y[j] * cf.sc[j];
                        }
                        continue;
                    }
                    const int g = __ldg(a.simple_rows + s0 + (int)(k - npre));
                    double y[NR];
                    spmv_row<TF, NR>(a, g, a.ev, y);
                    TF acc[NR];
                    double scv[NR];
#pragma unroll
                    for (int j = 0; j < NR; ++j) {
                        scv[j] = cf.sc[j];
                        acc[j] = (TF)(y[j] * scv[j]);
                    }
                    if (fused)  // level 1: its U' rows gather the unscaled level-0 Av
                        row_sub<TF, NR, true>(acc, __ldg(a.ut_off + g), __ldg(a.ut_off + g + 1), a.ut_col, a.ut_val,
                                              a.Av, scv);
                    else
                        row_sub<TF, NR>(acc, __ldg(a.ut_off + g), __ldg(a.ut_off + g + 1), a.ut_col, a.ut_val, a.Av);
                    double av[NR];
#pragma unroll
                    for (int j = 0; j < NR; ++j) {
                        av[j] = (double)acc[j];
                        a.Av[(size_t)g * NR + j] = av[j];
                    }
                    if (last) simple_epilogue<TF, NR>(a, g, av, cv.vk, cv.vk1, cv.pkm1, cv.pk, cv.pk, cf, r);
                }
                if (L > 0) {
                    // warps without a block row in this level take the tails;
                    // if every warp has one, all threads do, after their items
                    const LvlBounds pb = lvl(L - 1);
                    const int e1 = pb.s1;
                    const int items = c1 - lb.c0;
                    const bool spare = items < nwarps;
                    if (!spare || wid >= items) {
                        const int t0 = spare ? (wid - items) * 32 + lane : ctx.g0;
                        const int ts = spare ? (nwarps - items) * 32 : ctx.gstride;
                        for (int i = pb.s0 + t0; i < e1; i += ts) {
                            const int g = __ldg(a.simple_rows + i);
                            double av[NR];
#pragma unroll
                            for (int j = 0; j < NR; ++j) {
                                const double w = a.Av[(size_t)g * NR + j];
                                av[j] = (fused && L == 1) ? (double)(TF)(w * cf.sc[j]) : w;
                            }
                            simple_epilogue<TF, NR>(a, g, av, cv.vk, cv.vk1, cv.pkm1, cv.pk, cv.pk, cf, r);
                        }
                    }
                }
                if (L < a.nl - 1) {
                    ctx.sync();
                    if (NR == 1 && L == 0) stamp(a.ts, it, 4);
                }
            }
            ctx.template reduce<4 * NR>(r, sh);
            if (tid == 0)
                for (int j = 0; j < NR; ++j) {
                    Scal& Q = S[j];
                    if (Q.done) continue;
                    const double bt = r[j] / Q.vdv;
                    Q.beta[k1] = bt;
                    Q.inv_beta = 1.0 / bt;
                    Q.eta = (Q.delta[k1] / bt) * Q.eta;
                    Q.alpha_next = r[NR + j] / r[2 * NR + j];
                    Q.vdv = r[2 * NR + j];
                    Q.norm_x = sqrt(r[3 * NR + j]);
                    Q.test0 |= (fabs(Q.delta[k1]) <= a.tol);
                    Q.test1 |= (Q.gamma / fma_rn(Q.norm_A, Q.norm_x, Q.norm_pb) <= a.tol);
                    bool stop = false;
                    if (it > 0 && (it % 4) == 0) {
                        if (Q.snap0 || Q.snap1) {
                            stop = true;
                            Q.iters = it;
                        }
                    } else if (((it + 1) % 4) == 0) {
                        Q.snap0 = Q.test0;
                        Q.snap1 = Q.test1;
                    }
                    if (!isfinite(Q.inv_beta) || !isfinite(Q.inv_rho) || !isfinite(Q.eta) ||
                        !isfinite(Q.inv_delta) || !isfinite(Q.alpha)) {
                        Q.breakdown = 1;
                        stop = true;
                        Q.iters = it;
                    }
                    if (!stop && it + 1 >= a.max_it) Q.iters = a.max_it;
                    if (stop) {
                        Q.done = 1;
                        Q.stop_it = it;
                    }
                }
            __syncthreads();
        }
        if (NR == 1) stamp(a.ts, it, 3);
        bool more = false;
#pragma unroll
        for (int j = 0; j < NR; ++j) more |= !S[j].done;
        if (more) ++it;
        else break;
    }
    // ---- x = P U^-1 D^-1 x~ into ev, then x (column-major) ----
    for (int L = a.nl - 1; L >= 0; --L) {
        const int r0 = __ldg(sv.qb + L), nr = __ldg(sv.qe + L) - r0;
        for (int t = wid; t < nr; t += nwarps) {
            const ItemMeta m = meta_of_row(a, __ldg(a.lvl_rows + r0 + t));
            const int fr = m.fr, h = m.h;
            double y[NR], d[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) y[j] = (lane < h) ? a.xt[(size_t)(fr + lane) * NR + j] : 0.0;
            u_item<TF, NR>(a, m, y, a.ev, d);
        }
        ctx.sync();
    }
    for (int g = row0 + ctx.g0; g < row1; g += ctx.gstride)
#pragma unroll
        for (int j = 0; j < NR; ++j) a.x[(size_t)j * a.n + g] = a.ev[(size_t)g * NR + j];
    if (sv.out && tid == 0)
        for (int j = 0; j < NR; ++j) {
            const Scal& Q = S[j];
            double* o = sv.out + 8 * j;
            o[0] = Q.gamma / Q.norm_pb;
            o[1] = Q.done ? Q.iters : it;
            o[2] = Q.breakdown;
            o[3] = (Q.snap0 || Q.snap1) ? 1 : 0;
            o[4] = Q.norm_pb;
            o[5] = Q.done ? Q.stop_it : it;
            // a level wait that gave up: the results are invalid
            o[6] = (counted && *(volatile unsigned long long*)(a.lvl_done + 1)) ? 1.0 : 0.0;
            if (o[6] != 0.0) o[2] = 1.0;
        }
    __syncthreads();
}

// launched with kResSlots ResSlot<TF> of dynamic shared memory
template <class TF, int CTAS, int NR>
__global__ void __launch_bounds__(kT, CTAS) k_sqmr_persistent(PArgs<TF> a)
{
    __shared__ Scal S[NR];
    __shared__ double sh[kMaxNV][kW];
    extern __shared__ __align__(16) unsigned char res_smem[];
    const int G = gridDim.x;
    GridCtx ctx{cg::this_grid(), a.partials, 0, (int)(threadIdx.x >> 5) * G + (int)blockIdx.x,  // items interleaved
                G * kW, (int)(blockIdx.x * kT + threadIdx.x), G * kT};
    const SysView sv{0, a.n, a.lvl_off, a.lvl_off + 1, blockIdx.x == 0 ? a.out : nullptr};
    sqmr_body<TF, NR>(a, ctx, sv, S, sh, reinterpret_cast<ResSlot<TF>*>(res_smem));
}

template <class TF>
constexpr size_t res_smem_bytes()
{
    return (size_t)kResSlots * sizeof(ResSlot<TF>);
}

// Batched solves of independent systems stored as one block-diagonal union
// (one pattern, one factor): each CTA takes the next unsolved system from a
// counter and runs its whole SQMR with CTA barriers only.  A system's result
// does not depend on the others or on which CTA solves it.
struct BatchArgs {
    int num;
    const int* row_off;  // num + 1
    const int* qb;       // num x nl
    const int* qe;
    double* out;         // num x 8
    int* next;           // counter, 0 at launch
};

template <class TF>
__global__ void __launch_bounds__(kT, kCtasPerSm) k_sqmr_batched(PArgs<TF> a, BatchArgs bt)
{
    __shared__ Scal S[1];
    __shared__ double sh[kMaxNV][kW];
    __shared__ int sys;
    CtaCtx ctx{(int)(threadIdx.x >> 5), kW, (int)threadIdx.x, kT};
    for (;;) {
        if (threadIdx.x == 0) sys = atomicAdd(bt.next, 1);
        __syncthreads();
        const int s = sys;
        __syncthreads();
        if (s >= bt.num) break;
        const SysView sv{__ldg(bt.row_off + s), __ldg(bt.row_off + s + 1), bt.qb + (size_t)s * a.nl,
                         bt.qe + (size_t)s * a.nl, bt.out + (size_t)s * 8};
        sqmr_body<TF, 1>(a, ctx, sv, S, sh);
    }
}

// Batched solves of independent systems that each have their own pattern,
// factor, matrix and vectors (the serving path): the CTA copies system s's
// argument block into shared memory and runs the same body over its rows,
// for nr[s] (1, 2 or 4) right-hand sides of that system at once.  Systems are
// handed out in index order, so the host lists the longest first.  MULTI =
// false compiles the one-right-hand-side body alone (every nr[s] == 1): the
// 2- and 4-wide bodies in the same kernel cost the common case registers.
template <class TF, bool MULTI>
__global__ void __launch_bounds__(kT, kCtasPerSm) k_sqmr_many(const PArgs<TF>* __restrict__ sys_args,
                                                             const int* __restrict__ nr, int num, int* next)
{
    __shared__ Scal S[kMaxNR];
    __shared__ double sh[kMaxNV][kW];
    __shared__ int sys;
    __shared__ PArgs<TF> pa;
    static_assert(sizeof(PArgs<TF>) % 8 == 0, "argument block copied in 8-byte words");
    CtaCtx ctx{(int)(threadIdx.x >> 5), kW, (int)threadIdx.x, kT};
    for (;;) {
        if (threadIdx.x == 0) sys = atomicAdd(next, 1);
        __syncthreads();
        const int s = sys;
        if (s >= num) break;
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(sys_args + s);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&pa);
        for (int i = threadIdx.x; i < (int)(sizeof(PArgs<TF>) / 8); i += kT) dst[i] = src[i];
        __syncthreads();
        const SysView sv{0, pa.n, pa.lvl_off, pa.lvl_off + 1, pa.out};
        if constexpr (MULTI) {
            const int r = __ldg(nr + s);
            if (r == 4) sqmr_body<TF, 4>(pa, ctx, sv, reinterpret_cast<Scal(&)[4]>(S), sh);
            else if (r == 2) sqmr_body<TF, 2>(pa, ctx, sv, reinterpret_cast<Scal(&)[2]>(S), sh);
            else sqmr_body<TF, 1>(pa, ctx, sv, reinterpret_cast<Scal(&)[1]>(S), sh);
        } else {
            sqmr_body<TF, 1>(pa, ctx, sv, reinterpret_cast<Scal(&)[1]>(S), sh);
        }
    }
}

// kernel arguments over a work area of kVecs n nr doubles + 8 nr (vectors, then out)
template <class TF>
PArgs<TF> make_args(Csr* A, Factor* M, double* base, double* partials, const double* b, double* x, double tol,
                    int max_it, int nr = 1)
{
    Pattern& p = *M->pat;
    const int n = A->m;
    PArgs<TF> a;
    a.n = n;
    a.nl = p.num_levels;
    a.max_it = max_it;
    a.fuse_l0 = (p.l0_diagonal && A->nnz == p.nnz && A->m == p.n) ? 1 : 0;
    a.tol = tol;
    a.rowptr = A->rowptr;
    a.colidx = A->colidx;
    a.kval = static_cast<const double*>(A->val);
    a.pk_col = M->pk_col.as<TF>();
    a.pk_row = M->pk_row.as<TF>();
    a.pk_off = M->pk_off.as<long long>();
    a.ndmask = M->ndmask.as<unsigned>();
    a.dg = M->dg.as<TF>();
    a.tri = M->tri.as<TF>();
    a.is_piv = M->is_piv.as<int>();
    a.perm = M->perm.as<int>();
    a.lvl_off = p.d_lvl_off.as<int>();
    a.lvl_rows = p.d_lvl_rows.as<int>();
    a.bs = p.d_bs.as<int>();
    a.u_off = M->u_off.as<int>();
    a.u_colp = M->u_colp.as<int>();
    a.u_val = M->u_val.as<TF>();
    a.ut_off = M->ut_off.as<int>();
    a.ut_col = M->ut_col.as<int>();
    a.ut_val = M->ut_val.as<TF>();
    a.rowflags = M->rowflags.as<int>();
    a.scan_s = M->scan_s.as<int>();
    a.scan_c = M->scan_c.as<int>();
    a.simple_rows = M->simple_rows.as<int>();
    a.cplx = M->cplx.as<int>();
    a.citem = M->citem.as<CItem>();
    const size_t vn = (size_t)n * nr;
    for (int i = 0; i < 2; ++i) {
        a.v[i] = base + (size_t)i * vn;
        a.p[i] = base + (size_t)(2 + i) * vn;
    }
    a.Av = base + (size_t)4 * vn;
    a.ev = base + (size_t)5 * vn;
    a.xt = base + (size_t)6 * vn;
    a.out = base + (size_t)kVecs * vn;
    a.partials = partials;
    a.ts = nullptr;
    a.lvl_done = nullptr;
    a.wait_skew = 0;
    a.x = x;
    a.b = b;
    return a;
}

int ctas_per_sm()
{
    static int c = [] {
        const char* e = getenv("CULIPX_SQMR_CTAS");
        return (e && atoi(e) == 1) ? 1 : kCtasPerSm;
    }();
    return c;
}

template <class TF, int NR>
const void* persistent_kernel()
{
    return ctas_per_sm() == 1 ? (const void*)k_sqmr_persistent<TF, 1, NR> : (const void*)k_sqmr_persistent<TF, 2, NR>;
}

// resident CTAs for the cooperative launch
template <class TF, int NR>
int persistent_grid(int dev, int* G)
{
    int per_sm = 0, sms = 0;
    CULIPX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // the resident item slots need more than the default 48 KB of dynamic shared memory
    CULIPX_CUDA(cudaFuncSetAttribute(persistent_kernel<TF, NR>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)res_smem_bytes<TF>()));
    CULIPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_kernel<TF, NR>(), kT,
                                                              res_smem_bytes<TF>()));
    if (per_sm < 1) return fail(CULIPX_NOT_SUPPORTED, "persistent SQMR kernel does not fit on an SM");
    *G = sms * std::min(per_sm, ctas_per_sm());
    return CULIPX_OK;
}

// Grid sizes depend on the device (SM count, occupancy), so each launch
// site keeps one entry per device of the current process.  Entries are
// written at most once with the same value, so concurrent first calls from
// several host threads at worst compute the size twice.
constexpr int kMaxDevices = 64;

struct DeviceGridCache {
    std::atomic<int> g[kMaxDevices];
};

// *G = the cached grid for the current device, computed by size(dev, &g) once
template <class SizeFn>
int cached_grid(DeviceGridCache& c, SizeFn size, int* G, int* dev_out = nullptr)
{
    int dev = 0;
    CULIPX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(CULIPX_NOT_SUPPORTED, "device %d beyond %d devices", dev, kMaxDevices);
    int g = c.g[dev].load(std::memory_order_acquire);
    if (g == 0) {
        CULIPX_TRY(size(dev, &g));
        c.g[dev].store(g, std::memory_order_release);
    }
    *G = g;
    if (dev_out) *dev_out = dev;
    return CULIPX_OK;
}

// launch and wait; out_host receives 8 values per right-hand side
template <class TF, int NR>
int run_persistent(culipx_handle_t* h, PArgs<TF>& a, int G, double* out_host, bool wait = true)
{
    cudaStream_t s = h->stream;
    // the recurrence vectors start at zero; x is zeroed as in the reference
    CULIPX_CUDA(cudaMemsetAsync(a.v[0], 0, (size_t)kVecs * a.n * NR * sizeof(double), s));
    CULIPX_CUDA(cudaMemsetAsync(a.x, 0, (size_t)a.n * NR * sizeof(double), s));
    void* args[] = {&a};
    CULIPX_CUDA(cudaLaunchCooperativeKernel(persistent_kernel<TF, NR>(), dim3(G), dim3(kT), args,
                                            res_smem_bytes<TF>(), s));
    h->launches += 1;
    CULIPX_CUDA(cudaMemcpyAsync(out_host, a.out, (size_t)8 * NR * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (wait) CULIPX_CUDA(cudaStreamSynchronize(s));
    return CULIPX_OK;
}

template <class TF, int NR>
int launch_persistent(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                      Sqmr* w, double* out_host, bool wait = true)
{
    const int n = A->m;
    cudaStream_t s = h->stream;
    const size_t need = ((size_t)kVecs * n * NR + 8 * NR + 64) * sizeof(double);
    if (w->vecs.bytes() < need) {
        CULIPX_TRY(w->vecs.alloc(h, need));
        w->n = -1;  // the single-RHS workspace size is no longer known
    }
    static DeviceGridCache grid_cache;  // one per <TF, NR> instantiation
    int G = 0;
    CULIPX_TRY(cached_grid(grid_cache, persistent_grid<TF, NR>, &G));
    if ((size_t)(2 * kMaxNV * G) * sizeof(double) > w->partials.bytes())
        CULIPX_TRY(w->partials.alloc(h, (size_t)2 * kMaxNV * G * sizeof(double)));
    PArgs<TF> a = make_args<TF>(A, M, w->vecs.as<double>(), w->partials.as<double>(), b, x, tol, max_it, NR);
    // the level counter in the spare slots after the results (need: 8 NR + 64 values)
    a.lvl_done = reinterpret_cast<unsigned long long*>(a.out + 8 * kMaxNR);
    a.wait_skew = w->wait_skew;
    if (w->profile && NR == 1) {
        if (w->ts.bytes() < (size_t)kTsIters * 8 * sizeof(unsigned long long))
            CULIPX_TRY(w->ts.alloc(h, (size_t)kTsIters * 8 * sizeof(unsigned long long)));
        CULIPX_CUDA(cudaMemsetAsync(w->ts.get(), 0, (size_t)kTsIters * 8 * sizeof(unsigned long long), s));
        a.ts = w->ts.as<unsigned long long>();
    }
    return run_persistent<TF, NR>(h, a, G, out_host, wait);
}

template <class TF>
int launch_nr(int nr, culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
              Sqmr* w, double* out_host)
{
    switch (nr) {
    case 1: return launch_persistent<TF, 1>(h, A, M, b, x, tol, max_it, w, out_host);
    case 2: return launch_persistent<TF, 2>(h, A, M, b, x, tol, max_it, w, out_host);
    default: return launch_persistent<TF, 4>(h, A, M, b, x, tol, max_it, w, out_host);
    }
}

int status_of(const double* o, int max_it)
{
    if (o[6] != 0.0) return fail(CULIPX_TIMEOUT, "persistent SQMR: a bounded device wait gave up (results invalid)");
    if (o[2] != 0.0) return CULIPX_BREAKDOWN;
    if (o[3] == 0.0 && max_it > 0 && (int)o[1] >= max_it) return CULIPX_MAXIT;
    return CULIPX_OK;
}

}  // namespace

// nrhs right-hand sides (column-major n x nrhs) in launches of up to
// kMaxNR at a time; per right-hand side the quasi-residual, iterations and
// status (OK / MAXIT / BREAKDOWN)
int sqmr_solve_multi(culipx_handle_t* h, Csr* A, Factor* M, int nrhs, const double* B, double* X, double tol,
                     int max_it, double* h_res, int* h_its, int* h_status, Sqmr* w)
{
    if (!A || !M || !B || !X || !w || nrhs < 1) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_multi: bad argument");
    if (A->precision != CULIPX_F64 || A->m != A->n || !M->computed || M->pat->n != A->m)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_multi: A must be square FP64 and M its computed factor");
    if (M->solve_algorithm == CULIPX_SOLVE_JACOBI)
        return fail(CULIPX_NOT_SUPPORTED, "culipx_sqmr_solve_multi: SOLVE_JACOBI needs culipx_sqmr_solve");
    if (max_it < 0) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_multi: max_it < 0");
    const size_t n = A->m;
    double out[8 * kMaxNR];
    for (int r0 = 0; r0 < nrhs; r0 += kMaxNR) {
        const int nr = std::min(kMaxNR, nrhs - r0);
        // 3 right-hand sides run as 4, the fourth a copy of the third: it stops
        // when the third does and its x is dropped
        const int nl = (nr == 1) ? 1 : (nr == 2) ? 2 : 4;
        const double* b = B + r0 * n;
        double* x = X + r0 * n;
        DeviceBuffer pad_b, pad_x;
        if (nl != nr) {
            CULIPX_TRY(pad_b.alloc(h, nl * n * sizeof(double)));
            CULIPX_TRY(pad_x.alloc(h, nl * n * sizeof(double)));
            CULIPX_CUDA(cudaMemcpyAsync(pad_b.get(), b, nr * n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
            CULIPX_CUDA(cudaMemcpyAsync(pad_b.as<double>() + nr * n, b + (nr - 1) * n, n * sizeof(double),
                                        cudaMemcpyDeviceToDevice, h->stream));
            b = pad_b.as<double>();
            x = pad_x.as<double>();
        }
        const int st = (M->precision == CULIPX_F64) ? launch_nr<double>(nl, h, A, M, b, x, tol, max_it, w, out)
                                                    : launch_nr<float>(nl, h, A, M, b, x, tol, max_it, w, out);
        if (st != CULIPX_OK) return st;
        if (nl != nr) {
            CULIPX_CUDA(cudaMemcpyAsync(X + r0 * n, x, nr * n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
            CULIPX_CUDA(cudaStreamSynchronize(h->stream));
        }
        for (int j = 0; j < nr; ++j) {
            const double* o = out + 8 * j;
            if (h_res) h_res[r0 + j] = o[0];
            if (h_its) h_its[r0 + j] = (int)o[1];
            if (h_status) h_status[r0 + j] = status_of(o, max_it);
        }
    }
    return CULIPX_OK;
}

// The right-hand sides of one system in groups of 4 (then 2 and 1: no
// padding, so nothing is allocated per call) enqueued on h's stream without
// waiting; right-hand side r's 8 result values go to out_host + 8 r (pinned
// memory for a truly asynchronous call).  Groups run one after another on
// the stream and share the workspace.
int sqmr_solve_multi_async(culipx_handle_t* h, Csr* A, Factor* M, int nrhs, const double* B, double* X, double tol,
                           int max_it, Sqmr* w, double* out_host)
{
    if (!A || !M || !B || !X || !w || !out_host || nrhs < 1)
        return fail(CULIPX_INVALID_ARG, "sqmr_solve_multi_async: bad argument");
    if (A->precision != CULIPX_F64 || A->m != A->n || !M->computed || M->pat->n != A->m)
        return fail(CULIPX_INVALID_ARG, "sqmr_solve_multi_async: A must be square FP64 and M its computed factor");
    const size_t n = A->m;
    const bool f64 = M->precision == CULIPX_F64;
    for (int r0 = 0; r0 < nrhs;) {
        const int rem = nrhs - r0;
        const int nr = rem >= 4 ? 4 : (rem >= 2 ? 2 : 1);
        const double* b = B + r0 * n;
        double* x = X + r0 * n;
        double* o = out_host + (size_t)8 * r0;
        int st;
        if (nr == 4)
            st = f64 ? launch_persistent<double, 4>(h, A, M, b, x, tol, max_it, w, o, false)
                     : launch_persistent<float, 4>(h, A, M, b, x, tol, max_it, w, o, false);
        else if (nr == 2)
            st = f64 ? launch_persistent<double, 2>(h, A, M, b, x, tol, max_it, w, o, false)
                     : launch_persistent<float, 2>(h, A, M, b, x, tol, max_it, w, o, false);
        else
            st = f64 ? launch_persistent<double, 1>(h, A, M, b, x, tol, max_it, w, o, false)
                     : launch_persistent<float, 1>(h, A, M, b, x, tol, max_it, w, o, false);
        if (st != CULIPX_OK) return st;
        r0 += nr;
    }
    return CULIPX_OK;
}

// ---------------------------------------------------------------------------
// Batched solves (no counterpart in the reference, which solves one system
// per SQMR object): systems given as consecutive row ranges of one
// block-diagonal union pattern.
namespace {

template <class TF>
int launch_batched(Batch* bt, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it, Sqmr* w)
{
    culipx_handle_t* h = bt->h;
    cudaStream_t s = h->stream;
    const int n = A->m;
    CULIPX_TRY(sqmr_workspace(w, h, n));
    static DeviceGridCache grid_cache;  // one per factor precision
    int G = 0;
    CULIPX_TRY(cached_grid(
        grid_cache,
        [](int dev, int* g) {
            int per_sm = 0, sms = 0;
            CULIPX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            CULIPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sqmr_batched<TF>, kT, 0));
            if (per_sm < 1) return fail(CULIPX_NOT_SUPPORTED, "batched SQMR kernel does not fit on an SM");
            *g = sms * std::min(per_sm, kCtasPerSm);
            return (int)CULIPX_OK;
        },
        &G));
    PArgs<TF> a = make_args<TF>(A, M, w->vecs.as<double>(), w->partials.as<double>(), b, x, tol, max_it);
    BatchArgs ba;
    ba.num = bt->num;
    ba.row_off = bt->d_row_off.as<int>();
    ba.qb = bt->d_qb.as<int>();
    ba.qe = bt->d_qe.as<int>();
    ba.out = bt->d_out.as<double>();
    ba.next = bt->d_next.as<int>();
    CULIPX_CUDA(cudaMemsetAsync(a.v[0], 0, (size_t)kVecs * n * sizeof(double), s));
    CULIPX_CUDA(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double), s));
    CULIPX_CUDA(cudaMemsetAsync(ba.next, 0, sizeof(int), s));
    k_sqmr_batched<TF><<<std::min(G, bt->num), kT, 0, s>>>(a, ba);
    h->launches += 1;
    return launch_check("k_sqmr_batched");
}

}  // namespace

int batch_create(culipx_handle_t* h, const Pattern* p, int num, const int* h_row_off, Batch** out)
{
    if (!p || !h_row_off || !out || num < 1) return fail(CULIPX_INVALID_ARG, "culipx_batch_create: bad argument");
    if (h_row_off[0] != 0 || h_row_off[num] != p->n)
        return fail(CULIPX_INVALID_ARG, "culipx_batch_create: row offsets must run from 0 to n");
    const int cm = p->num_blocks, nl = p->num_levels;
    // system of every block row; every system boundary must be a block boundary
    std::vector<int> sys(cm);
    int s = 0;
    for (int I = 0; I < cm; ++I) {
        while (s < num && h_row_off[s + 1] <= p->bs[I]) ++s;
        if (s >= num || h_row_off[s] > p->bs[I] || p->bs[I + 1] > h_row_off[s + 1])
            return fail(CULIPX_INVALID_ARG, "culipx_batch_create: a system boundary splits block row %d", I);
        sys[I] = s;
    }
    for (int k = 0; k < num; ++k)
        if (h_row_off[k + 1] <= h_row_off[k]) return fail(CULIPX_INVALID_ARG, "culipx_batch_create: empty system %d", k);
    // the systems must be independent: no block of the (filled) pattern couples two of them
    for (int b = 0; b < p->coarse_nnz; ++b)
        if (sys[p->blk_row[b]] != sys[p->blk_col[b]])
            return fail(CULIPX_INVALID_ARG, "culipx_batch_create: block (%d, %d) couples systems %d and %d",
                        p->blk_row[b], p->blk_col[b], sys[p->blk_row[b]], sys[p->blk_col[b]]);
    // per system and level: its (contiguous) run in the level's ascending block list
    std::vector<int> qb((size_t)num * std::max(nl, 1), 0), qe((size_t)num * std::max(nl, 1), 0);
    for (int L = 0; L < nl; ++L)
        for (int q = p->lvl_off[L]; q < p->lvl_off[L + 1]; ++q) {
            const int k = sys[p->lvl_rows[q]];
            int& b0 = qb[(size_t)k * nl + L];
            int& e0 = qe[(size_t)k * nl + L];
            if (e0 == b0) b0 = q;
            else if (e0 != q) return fail(CULIPX_INVALID_ARG, "culipx_batch_create: level list not grouped by system");
            e0 = q + 1;
        }
    auto* bt = new culipx_batch_t();
    bt->h = h;
    bt->pat = p;
    bt->num = num;
    bt->nl = nl;
    bt->row_off.assign(h_row_off, h_row_off + num + 1);
    int st = bt->d_row_off.upload(h, h_row_off, (size_t)(num + 1) * sizeof(int));
    if (st == CULIPX_OK) st = bt->d_qb.upload(h, qb.data(), qb.size() * sizeof(int));
    if (st == CULIPX_OK) st = bt->d_qe.upload(h, qe.data(), qe.size() * sizeof(int));
    if (st == CULIPX_OK) st = bt->d_out.alloc(h, (size_t)num * 8 * sizeof(double));
    if (st == CULIPX_OK) st = bt->d_next.alloc(h, sizeof(int));
    if (st != CULIPX_OK) {
        delete bt;
        return st;
    }
    *out = bt;
    return CULIPX_OK;
}

namespace {

// the batch's results (8 values per system) to per-system residual, iterations, status
int batch_results(Batch* bt, int max_it, double* h_res, int* h_its, int* h_status)
{
    std::vector<double> out((size_t)bt->num * 8);
    CULIPX_CUDA(cudaMemcpyAsync(out.data(), bt->d_out.get(), out.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                bt->h->stream));
    CULIPX_CUDA(cudaStreamSynchronize(bt->h->stream));
    for (int k = 0; k < bt->num; ++k) {
        const double* o = out.data() + (size_t)k * 8;
        if (h_res) h_res[k] = o[0];
        if (h_its) h_its[k] = (int)o[1];
        if (h_status)
            h_status[k] = (o[2] != 0.0) ? CULIPX_BREAKDOWN
                          : (o[3] == 0.0 && max_it > 0 && (int)o[1] >= max_it) ? CULIPX_MAXIT
                                                                               : CULIPX_OK;
    }
    return CULIPX_OK;
}

int batch_check(Batch* bt, Csr* A, Factor* M, const double* b, double* x, int max_it, const char* what)
{
    if (!bt || !A || !M || !b || !x) return fail(CULIPX_INVALID_ARG, "%s: null argument", what);
    if (A->precision != CULIPX_F64 || A->m != A->n || A->m != bt->pat->n)
        return fail(CULIPX_INVALID_ARG, "%s: A must be the FP64 union matrix of the batch", what);
    if (M->pat != bt->pat) return fail(CULIPX_INVALID_ARG, "%s: M must be a factor of the batch's pattern", what);
    if (M->solve_algorithm == CULIPX_SOLVE_JACOBI) return fail(CULIPX_NOT_SUPPORTED, "%s: SOLVE_JACOBI is not batched", what);
    if (max_it < 0) return fail(CULIPX_INVALID_ARG, "%s: max_it < 0", what);
    return CULIPX_OK;
}

}  // namespace

Batch::~Batch()
{
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (capture_stream) cudaStreamDestroy(capture_stream);
    delete gw;
}

// The numeric factorization of the union and the batched solve as one CUDA
// graph launch.  The first call for a given set of buffers (values, A, M, b,
// x) and settings factors and solves by ordinary launches -- which sizes
// every buffer, the batch's own solver workspace included -- and captures
// the same sequence on a stream of the batch's own; later calls replay it
// (the contents of the buffers may change in between).
int batch_factor_solve_graph(Batch* bt, Csr* A, Factor* M, const void* d_vals, int pivot, double threshold,
                             const double* b, double* x, double tol, int max_it, double* h_res, int* h_its,
                             int* h_status)
{
    CULIPX_TRY(batch_check(bt, A, M, b, x, max_it, "culipx_batch_factor_solve_graph"));
    if (!d_vals) return fail(CULIPX_INVALID_ARG, "culipx_batch_factor_solve_graph: null values");
    if (pivot < CULIPX_PIV_STATIC || pivot > CULIPX_PIV_ROOK)
        return fail(CULIPX_INVALID_ARG, "culipx_batch_factor_solve_graph: bad pivot method %d", pivot);
    culipx_handle_t* h = bt->h;
    if (!bt->gw) bt->gw = new Sqmr();
    Batch::Key key;
    key.vals = d_vals;
    key.A = A->serial;
    key.M = M->serial;
    key.b = b;
    key.x = x;
    key.pivot = pivot;
    key.max_it = max_it;
    key.threshold = threshold;
    key.tol = tol;
    key.piv64 = M->pivot_fp64;
    auto solve = [&]() -> int {
        return (M->precision == CULIPX_F64) ? launch_batched<double>(bt, A, M, b, x, tol, max_it, bt->gw)
                                            : launch_batched<float>(bt, A, M, b, x, tol, max_it, bt->gw);
    };
    if (!bt->graph_exec || !(bt->graph_key == key)) {
        CULIPX_TRY(factor_compute(M, d_vals, nullptr, pivot, threshold));
        CULIPX_TRY(solve());
        CULIPX_TRY(batch_results(bt, max_it, h_res, h_its, h_status));
        if (bt->graph_exec) cudaGraphExecDestroy(bt->graph_exec);
        if (bt->graph) cudaGraphDestroy(bt->graph);
        bt->graph_exec = nullptr;
        bt->graph = nullptr;
        if (!bt->capture_stream) CULIPX_CUDA(cudaStreamCreateWithFlags(&bt->capture_stream, cudaStreamNonBlocking));
        cudaStream_t s = h->stream;
        const long long launches0 = h->launches;
        CULIPX_CUDA(cudaStreamBeginCapture(bt->capture_stream, cudaStreamCaptureModeThreadLocal));
        h->stream = bt->capture_stream;
        M->capturing = true;
        int st = factor_compute(M, d_vals, nullptr, pivot, threshold);
        if (st == CULIPX_OK) st = solve();
        M->capturing = false;
        h->stream = s;
        bt->graph_launches = (int)(h->launches - launches0);
        h->launches = launches0;  // captured, not launched
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(bt->capture_stream, &g);
        if (st != CULIPX_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return st != CULIPX_OK ? st
                                   : fail(CULIPX_CUDA_ERROR, "culipx_batch_factor_solve_graph: capture failed: %s",
                                          cudaGetErrorString(e));
        }
        cudaGraphExec_t ge = nullptr;
        if (cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) {
            cudaGraphDestroy(g);
            cudaGetLastError();
            return fail(CULIPX_CUDA_ERROR, "culipx_batch_factor_solve_graph: graph instantiation failed");
        }
        bt->graph = g;
        bt->graph_exec = ge;
        bt->graph_key = key;
        return CULIPX_OK;  // the ordinary run above factored and solved
    }
    CULIPX_CUDA(cudaGraphLaunch(bt->graph_exec, h->stream));
    h->launches += bt->graph_launches;
    M->pivot = pivot;
    M->threshold = threshold;
    M->computed = true;
    return batch_results(bt, max_it, h_res, h_its, h_status);
}

int batch_sqmr_solve(Batch* bt, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                     double* h_res, int* h_its, int* h_status, Sqmr* w)
{
    if (!bt || !A || !M || !b || !x || !w) return fail(CULIPX_INVALID_ARG, "culipx_batch_sqmr_solve: null argument");
    if (A->precision != CULIPX_F64 || A->m != A->n || A->m != bt->pat->n)
        return fail(CULIPX_INVALID_ARG, "culipx_batch_sqmr_solve: A must be the FP64 union matrix of the batch");
    if (!M->computed || M->pat != bt->pat)
        return fail(CULIPX_INVALID_ARG, "culipx_batch_sqmr_solve: M must be a computed factor of the batch's pattern");
    if (M->solve_algorithm == CULIPX_SOLVE_JACOBI)
        return fail(CULIPX_NOT_SUPPORTED, "culipx_batch_sqmr_solve: SOLVE_JACOBI is not batched");
    if (max_it < 0) return fail(CULIPX_INVALID_ARG, "culipx_batch_sqmr_solve: max_it < 0");
    const int st = (M->precision == CULIPX_F64) ? launch_batched<double>(bt, A, M, b, x, tol, max_it, w)
                                                : launch_batched<float>(bt, A, M, b, x, tol, max_it, w);
    if (st != CULIPX_OK) return st;
    std::vector<double> out((size_t)bt->num * 8);
    CULIPX_CUDA(cudaMemcpyAsync(out.data(), bt->d_out.get(), out.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                bt->h->stream));
    CULIPX_CUDA(cudaStreamSynchronize(bt->h->stream));
    for (int k = 0; k < bt->num; ++k) {
        const double* o = out.data() + (size_t)k * 8;
        if (h_res) h_res[k] = o[0];
        if (h_its) h_its[k] = (int)o[1];
        if (h_status)
            h_status[k] = (o[2] != 0.0) ? CULIPX_BREAKDOWN
                          : (o[3] == 0.0 && max_it > 0 && (int)o[1] >= max_it) ? CULIPX_MAXIT
                                                                               : CULIPX_OK;
    }
    return CULIPX_OK;
}

namespace {

// Enqueues one launch per (factor precision, right-hand sides per system)
// group on h's stream.  System k solves nr[k] (1, 2 or 4) right-hand sides,
// b[k] / x[k] each n x nr[k] column-major; its results (8 values per
// right-hand side) go to out_host + 8 (nr[0] + ... + nr[k-1]) (pinned
// memory for a truly asynchronous call).  One workspace allocation serves
// every group.
// every system's work area starts on a 256-byte boundary: with NR even the
// kernel reads the interleaved vectors with 16-byte loads
double* align256(double* p)
{
    return reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(p) + 255) & ~static_cast<uintptr_t>(255));
}

template <class TF>
int launch_many_prec(culipx_handle_t* h, const std::vector<int>& ks, const int* nr, Csr* const* A, Factor* const* M,
                     const double* const* b, double* const* x, const std::vector<size_t>& slot, double tol,
                     int max_it, double*& base, double* out_host)
{
    cudaStream_t s = h->stream;
    const int num = (int)ks.size();
    std::vector<PArgs<TF>> args(num);
    std::vector<int> nrs(num);
    for (int i = 0; i < num; ++i) {
        const int k = ks[i];
        const int r = nr ? nr[k] : 1;
        const size_t m = A[k]->m;
        base = align256(base);
        args[i] = make_args<TF>(A[k], M[k], base, nullptr, b[k], x[k], tol, max_it, r);
        base += (size_t)kVecs * m * r + 8 * r;
        nrs[i] = r;
        CULIPX_CUDA(cudaMemsetAsync(args[i].v[0], 0, (size_t)kVecs * m * r * sizeof(double), s));
        CULIPX_CUDA(cudaMemsetAsync(x[k], 0, m * r * sizeof(double), s));
    }
    // argument blocks after the vectors, then the right-hand-side counts and the counter
    base = align256(base);
    PArgs<TF>* d_args = reinterpret_cast<PArgs<TF>*>(base);
    int* d_nr = reinterpret_cast<int*>(d_args + num);
    int* d_next = d_nr + num;
    base = reinterpret_cast<double*>(d_args + num) + (num + 2) / 2 + 1;
    CULIPX_CUDA(cudaMemcpyAsync(d_args, args.data(), (size_t)num * sizeof(PArgs<TF>), cudaMemcpyHostToDevice, s));
    CULIPX_CUDA(cudaMemcpyAsync(d_nr, nrs.data(), (size_t)num * sizeof(int), cudaMemcpyHostToDevice, s));
    CULIPX_CUDA(cudaMemsetAsync(d_next, 0, sizeof(int), s));
    const bool multi = std::any_of(nrs.begin(), nrs.end(), [](int r) { return r != 1; });
    static DeviceGridCache grid_caches[2];  // single / multi right-hand-side variant, per factor precision
    auto many_grid = [](const void* kern) {
        return [kern](int dev, int* g) {
            int per_sm = 0, sms = 0;
            CULIPX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            CULIPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kT, 0));
            if (per_sm < 1) return fail(CULIPX_NOT_SUPPORTED, "batched SQMR kernel does not fit on an SM");
            *g = sms * std::min(per_sm, kCtasPerSm);
            return (int)CULIPX_OK;
        };
    };
    int G = 0;
    if (multi) CULIPX_TRY(cached_grid(grid_caches[1], many_grid((const void*)k_sqmr_many<TF, true>), &G));
    else CULIPX_TRY(cached_grid(grid_caches[0], many_grid((const void*)k_sqmr_many<TF, false>), &G));
    if (multi) k_sqmr_many<TF, true><<<std::min(G, num), kT, 0, s>>>(d_args, d_nr, num, d_next);
    else k_sqmr_many<TF, false><<<std::min(G, num), kT, 0, s>>>(d_args, d_nr, num, d_next);
    h->launches += 1;
    CULIPX_TRY(launch_check("k_sqmr_many"));
    for (int i = 0; i < num; ++i)
        CULIPX_CUDA(cudaMemcpyAsync(out_host + 8 * slot[ks[i]], args[i].out, (size_t)8 * nrs[i] * sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
    return CULIPX_OK;
}

}  // namespace

int sqmr_solve_many_nr_async(culipx_handle_t* h, int num, Csr* const* A, Factor* const* M, const double* const* b,
                             double* const* x, const int* nr, double tol, int max_it, Sqmr* w, double* out_host)
{
    if (num == 0) return CULIPX_OK;
    // result slots in the caller's order; per factor precision one launch with
    // the systems longest first (rows x right-hand sides), so the CTAs that
    // take the last systems finish close together
    std::vector<size_t> slot(num);
    size_t total = 0, acc = 0;
    std::vector<int> groups[2];
    for (int k = 0; k < num; ++k) {
        const int r = nr ? nr[k] : 1;
        if (r != 1 && r != 2 && r != 4) return fail(CULIPX_INVALID_ARG, "sqmr_solve_many: nr must be 1, 2 or 4");
        slot[k] = acc;
        acc += r;
        total += (size_t)kVecs * A[k]->m * r + 8 * r + 32;  // + alignment
        groups[M[k]->precision == CULIPX_F64 ? 0 : 1].push_back(k);
    }
    size_t argbytes = 0;
    for (int p = 0; p < 2; ++p) {
        std::vector<int>& ks = groups[p];
        std::stable_sort(ks.begin(), ks.end(), [&](int a, int c) {
            return (long long)A[a]->m * (nr ? nr[a] : 1) > (long long)A[c]->m * (nr ? nr[c] : 1);
        });
        if (!ks.empty())
            argbytes += ks.size() * ((p == 0 ? sizeof(PArgs<double>) : sizeof(PArgs<float>)) + sizeof(int)) + 512;
    }
    const size_t need = total * sizeof(double) + argbytes + 256;
    if (w->many.bytes() < need) CULIPX_TRY(w->many.alloc(h, need));
    double* base = w->many.as<double>();
    if (!groups[0].empty())
        CULIPX_TRY(launch_many_prec<double>(h, groups[0], nr, A, M, b, x, slot, tol, max_it, base, out_host));
    if (!groups[1].empty())
        CULIPX_TRY(launch_many_prec<float>(h, groups[1], nr, A, M, b, x, slot, tol, max_it, base, out_host));
    return CULIPX_OK;
}

int sqmr_solve_many_async(culipx_handle_t* h, int num, Csr* const* A, Factor* const* M, const double* const* b,
                          double* const* x, double tol, int max_it, Sqmr* w, double* out_host)
{
    return sqmr_solve_many_nr_async(h, num, A, M, b, x, nullptr, tol, max_it, w, out_host);
}

void many_results(int num, int max_it, const double* out, double* h_res, int* h_its, int* h_status)
{
    for (int k = 0; k < num; ++k) {
        const double* o = out + (size_t)k * 8;
        if (h_res) h_res[k] = o[0];
        if (h_its) h_its[k] = (int)o[1];
        if (h_status)
            h_status[k] = (o[2] != 0.0) ? CULIPX_BREAKDOWN
                          : (o[3] == 0.0 && max_it > 0 && (int)o[1] >= max_it) ? CULIPX_MAXIT
                                                                               : CULIPX_OK;
    }
}

int sqmr_solve_many(culipx_handle_t* h, int num, Csr* const* A, Factor* const* M, const double* const* b,
                    double* const* x, double tol, int max_it, double* h_res, int* h_its, int* h_status, Sqmr* w)
{
    if (num < 0 || (num > 0 && (!A || !M || !b || !x)) || !w)
        return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_many: bad argument");
    if (max_it < 0) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_many: max_it < 0");
    if (num == 0) return CULIPX_OK;
    const int prec = M[0] ? M[0]->precision : CULIPX_F64;
    for (int k = 0; k < num; ++k) {
        if (!A[k] || !M[k] || !b[k] || !x[k]) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_many: null system %d", k);
        if (A[k]->precision != CULIPX_F64 || A[k]->m != A[k]->n || !M[k]->computed || M[k]->pat->n != A[k]->m)
            return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_many: system %d: A must be square FP64 and M its computed factor", k);
        if (M[k]->precision != prec)
            return fail(CULIPX_NOT_SUPPORTED, "culipx_sqmr_solve_many: all factors of one call must share a precision");
        if (M[k]->solve_algorithm == CULIPX_SOLVE_JACOBI)
            return fail(CULIPX_NOT_SUPPORTED, "culipx_sqmr_solve_many: SOLVE_JACOBI is not batched");
    }
    std::vector<double> out((size_t)num * 8, 0.0);
    CULIPX_TRY(sqmr_solve_many_async(h, num, A, M, b, x, tol, max_it, w, out.data()));
    CULIPX_CUDA(cudaStreamSynchronize(h->stream));
    many_results(num, max_it, out.data(), h_res, h_its, h_status);
    return CULIPX_OK;
}

int sqmr_solve_persistent(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                          double* residual, int* iterations, Sqmr* w)
{
    double out[8];
    const int st = (M->precision == CULIPX_F64) ? launch_persistent<double, 1>(h, A, M, b, x, tol, max_it, w, out)
                                                : launch_persistent<float, 1>(h, A, M, b, x, tol, max_it, w, out);
    if (st != CULIPX_OK) return st;
    if (residual) *residual = out[0];
    if (iterations) *iterations = (int)out[1];
    if (out[6] != 0.0) return fail(CULIPX_TIMEOUT, "culipx_sqmr_solve: a bounded device wait gave up (results invalid)");
    if (out[2] != 0.0) return fail(CULIPX_BREAKDOWN, "culipx_sqmr_solve: breakdown (non-finite scalar)");
    if (out[3] == 0.0 && max_it > 0 && (int)out[1] >= max_it) return CULIPX_MAXIT;
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
// The scratch is a file-scope device array of kNoAllocMaxRows x 8 doubles
// plus the per-CTA reduction slots (about 4.3 MB): every GPU that loads this
// library holds it until the process exits.  All calls share it and it keeps
// the last call's contents; the call clears what must start at zero.  Calls
// whose work overlaps on the GPU (two streams, two host threads) race on it.
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current); make that first call
// before any stream capture.
namespace {

constexpr int kNoAllocMaxRows = 65536;
constexpr int kNoAllocMaxGrid = 1024;
constexpr size_t kNoAllocVecs = (kVecs + 1) * (size_t)kNoAllocMaxRows;
constexpr size_t kNoAllocSlots = kNoAllocVecs + (size_t)2 * kMaxNV * kNoAllocMaxGrid;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocSlots];

std::atomic<double*> g_noalloc_ptr[kMaxDevices];  // per-device address of g_noalloc_scratch

int noalloc_setup(int dev)
{
    if (g_noalloc_ptr[dev].load(std::memory_order_acquire)) return CULIPX_OK;
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
        cudaGetLastError();
        return fail(CULIPX_CUDA_ERROR, "culipx_sqmr_solve_noalloc: cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(e));
    }
    g_noalloc_ptr[dev].store(static_cast<double*>(ptr), std::memory_order_release);
    return CULIPX_OK;
}

template <class TF>
int noalloc_grid(int dev, int* G)
{
    CULIPX_TRY((persistent_grid<TF, 1>(dev, G)));
    *G = std::min(*G, kNoAllocMaxGrid);
    return CULIPX_OK;
}

// out[0..3] = residual estimate, iterations, breakdown flag, converged flag
template <class TF>
int launch_noalloc(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                   double (&out)[8])
{
    static DeviceGridCache grid_cache;  // one per factor precision
    int G = 0, dev = 0;
    CULIPX_TRY(cached_grid(grid_cache, noalloc_grid<TF>, &G, &dev));
    CULIPX_TRY(noalloc_setup(dev));
    double* base = g_noalloc_ptr[dev].load(std::memory_order_acquire);
    // run_persistent clears the recurrence vectors the scratch kept from the last call
    PArgs<TF> a = make_args<TF>(A, M, base, base + kNoAllocVecs, b, x, tol, max_it);
    // the level counter after the results (the vectors' region holds a spare row of kNoAllocMaxRows values)
    a.lvl_done = reinterpret_cast<unsigned long long*>(a.out + 8 * kMaxNR);
    a.wait_skew = h->sqmr ? h->sqmr->wait_skew : 0;
    return run_persistent<TF, 1>(h, a, G, out);
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
    if (M->solve_algorithm == CULIPX_SOLVE_JACOBI)
        return fail(CULIPX_NOT_SUPPORTED, "culipx_sqmr_solve_noalloc: SOLVE_JACOBI needs culipx_sqmr_solve");
    if (A->m > kNoAllocMaxRows)
        return fail(CULIPX_INVALID_ARG,
                    "culipx_sqmr_solve_noalloc: n = %d exceeds the fixed scratch of %d rows; use culipx_sqmr_solve",
                    A->m, kNoAllocMaxRows);
    if (max_it < 0) return fail(CULIPX_INVALID_ARG, "culipx_sqmr_solve_noalloc: max_it < 0");
    double out[8] = {};
    const int st = M->precision == CULIPX_F64 ? launch_noalloc<double>(h, A, M, b, x, tol, max_it, out)
                                              : launch_noalloc<float>(h, A, M, b, x, tol, max_it, out);
    if (st != CULIPX_OK) return st;
    if (residual) *residual = out[0];
    if (iterations) *iterations = (int)out[1];
    if (out[6] != 0.0)
        return fail(CULIPX_TIMEOUT, "culipx_sqmr_solve_noalloc: a bounded device wait gave up (results invalid)");
    if (out[2] != 0.0) return fail(CULIPX_BREAKDOWN, "culipx_sqmr_solve_noalloc: breakdown (non-finite scalar)");
    return status_of(out, max_it);
}

}  // namespace culipx
