// Device functions of the dense pivot-tile factorization and of the sparse
// Schur updates (one warp per 32x32 tile in shared memory).  Semantics of
// libs/la/preconditioner/block_ildlt_kernels.impl.cuh as cited per function;
// all fused multiply-adds are explicit (the library builds with --fmad=false).
#pragma once

#include "kernels_common.cuh"

#include <culipx.h>

namespace culipx {

template <class T>
__device__ __forceinline__ T bk_alpha() { return (T)((1.0f + sqrtf(17.0f)) / 8.0f); }

// Out[a][b] -= sum_r R[r][b] * (Q' D_k)[a][r] for a in colmask(Q), lanes b < rh.
// Q: U_ki (bw x .), R: U_kj (bw x rh); D_k from tri at the rows of block k.
// d_multiply_block_by_block_diagonal (:372-411) + d_apply_left_right_update.
// schur_update_d takes lane r's entries of D_k (super, diagonal, sub; zero
// for r >= bw) already loaded.
template <class T>
__device__ __forceinline__ void schur_update_d(T* out, const T* Q, const T* R, unsigned colmask, int bw, int rh,
                                               T sup, T dia, T sub)
{
    const int lane = lane_id();
    while (colmask) {
        const int a = __ffs(colmask) - 1;
        colmask &= colmask - 1;
        T lv = T(0);
        if (lane < bw) {
            const T left = (lane > 0) ? Q[(lane - 1) * kTileStride + a] : T(0);
            const T mid = Q[lane * kTileStride + a];
            const T right = (lane < 31) ? Q[(lane + 1) * kTileStride + a] : T(0);
            lv = fma_rn(sub, right, fma_rn(dia, mid, sup * left));  // the reference build's rounding order
        }
        unsigned m = __ballot_sync(0xffffffffu, lv != T(0));
        T acc = T(0);
        while (m) {
            const int r = __ffs(m) - 1;
            m &= m - 1;
            const T la = shfl(lv, r);
            acc = fma_rn(R[r * kTileStride + lane], la, acc);
        }
        if (lane < rh) out[a * kTileStride + lane] -= acc;
    }
    __syncwarp();
}

template <class T>
__device__ __forceinline__ void schur_update(T* out, const T* Q, const T* R, unsigned colmask, int bw, int rh,
                                             const T* tri_k)
{
    const int lane = lane_id();
    T sup = T(0), dia = T(0), sub = T(0);
    if (lane < bw) {
        sup = tri_k[3 * lane];
        dia = tri_k[3 * lane + 1];
        sub = tri_k[3 * lane + 2];
    }
    schur_update_d(out, Q, R, colmask, bw, rh, sup, dia, sub);
}

// ---- dense pivot-block factorization (d_factor_pivot_factorize, :956-1083) ----

template <class T>
__device__ __forceinline__ void pivot_swap(T* Tt, int* perm, int p1, int p2, int len)
{
    const int l = lane_id();
    int ia, ib;
    if (l < p1) { ia = l * kTileStride + p1; ib = l * kTileStride + p2; }
    else if (l == p1) { ia = p1 * kTileStride + p1; ib = p2 * kTileStride + p2; }
    else if (l < p2) { ia = p1 * kTileStride + l; ib = l * kTileStride + p2; }
    else if (l == p2) { ia = p1 * kTileStride + p2; ib = ia; }
    else { ia = p1 * kTileStride + l; ib = p2 * kTileStride + l; }
    T va = T(0), vb = T(0);
    if (l < len) { va = Tt[ia]; vb = Tt[ib]; }
    __syncwarp();
    if (l < len) Tt[ia] = vb;
    __syncwarp();
    if (l < len) Tt[ib] = va;
    if (l == 0) { const int t = perm[p1]; perm[p1] = perm[p2]; perm[p2] = t; }
    __syncwarp();
}

// argmax of v over lanes, ties to the lowest index (value, index) = (v, i).
// A NaN score counts as 0 (no candidate): with NaNs the comparisons are no
// total order and the lanes' butterflies would end at different results.
template <class T>
__device__ __forceinline__ void warp_argmax(T& v, int& i)
{
    if (v != v) v = T(0);
    for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
    }
}

template <class T>
__device__ __forceinline__ T warp_max(T v)
{
    if (v != v) v = T(0);  // as in warp_argmax: every lane ends at the same value
    for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, v, o);
        v = (ov > v) ? ov : v;
    }
    return v;
}

template <class T>
__device__ __forceinline__ T upper_abs(const T* Tt, int a, int b)
{
    return (a < b) ? fabs(Tt[a * kTileStride + b]) : fabs(Tt[b * kTileStride + a]);
}

template <class T>
__device__ __forceinline__ void select_bk(const T* Tt, int p, int len, int& order, int& p0, int& p1)
{
    const int l = lane_id();
    const T alpha = bk_alpha<T>();
    order = 1;
    p0 = p;
    int r = (l > p + 1) ? l : p + 1;
    T w1 = (l > p && l < len) ? fabs(Tt[p * kTileStride + l]) : T(0);
    warp_argmax(w1, r);
    if (!(w1 > T(0))) return;
    const T app = fabs(Tt[p * kTileStride + p]);
    if (app >= alpha * w1) return;
    T wr = (l < p || l == r || l >= len) ? T(0) : upper_abs(Tt, l, r);
    wr = warp_max(wr);
    if (app * wr >= alpha * w1 * w1) return;
    if (fabs(Tt[r * kTileStride + r]) >= alpha * wr) { p0 = r; return; }
    order = 2;
    p0 = p;
    p1 = r;
}

template <class T>
__device__ __forceinline__ void select_rook(const T* Tt, int p, int len, int& order, int& p0, int& p1)
{
    const int l = lane_id();
    const T alpha = bk_alpha<T>();
    order = 1;
    p0 = p;
    int r = (l > p + 1) ? l : p + 1;
    T wi = (l > p && l < len) ? fabs(Tt[p * kTileStride + l]) : T(0);
    warp_argmax(wi, r);
    if (!(wi > T(0))) return;
    int i = p;
    if (fabs(Tt[p * kTileStride + p]) >= alpha * wi) return;
    for (int guard = 0; guard < 64; ++guard) {  // values strictly grow: at most len rounds
        int q = (l > p) ? l : p;
        T wr = (l >= p && l < len && l != r) ? upper_abs(Tt, l, r) : T(0);
        warp_argmax(wr, q);
        if (fabs(Tt[r * kTileStride + r]) >= alpha * wr) { p0 = r; return; }
        if (wi == wr) { order = 2; p0 = i; p1 = r; return; }
        i = r;
        r = q;
        wi = wr;
    }
    p0 = p;  // unreachable for finite values
}

template <class T>
__device__ __forceinline__ void step_1x1(T* Tt, T* D, int row, int len)
{
    const int l = lane_id();
    T d11 = Tt[row * kTileStride + row];
    const bool modified = fabs(d11) < 1e-8;
    if (modified) d11 = T(1e-6);
    const T a = (l < row) ? T(0) : Tt[row * kTileStride + l];
    const T u = a / d11;
    __syncwarp();
    Tt[row * kTileStride + l] = u;
    const T ru = u * d11;
    for (int i = row + 1; i < len; ++i) {
        const T lv = shfl(ru, i);
        if (l < len) Tt[i * kTileStride + l] = fma_rn(-lv, u, Tt[i * kTileStride + l]);
    }
    __syncwarp();
    if (modified && l == 0) Tt[row * kTileStride + row] = T(1);
    if (l < 3) D[3 * row + l] = (l != 1) ? T(0) : d11;
    __syncwarp();
}

// The Givens-form 2x2 solve of d_ldlt_2x2_step (:589-675) with its
// arithmetic in C: T itself, or double for an ill-conditioned pivot of an FP32
// factor (wide_2x2); the stored U entries and the Schur update are rounded to
// T once.  With C = T every operation is the reference's.
template <class T, class C>
__device__ __forceinline__ void step_2x2_in(T* Tt, int row, int len, C d11, C d12, C d22)
{
    const int l = lane_id();
    const C a1 = (l < row) ? C(0) : C(Tt[row * kTileStride + l]);
    const C a2 = (l < row) ? C(0) : ((l == row) ? d12 : C(Tt[(row + 1) * kTileStride + l]));
    const C gr = sqrt(fma_rn(d11, d11, d12 * d12));
    const C gc = d11 / gr, gs = d12 / gr;
    C x1 = fma_rn(gc, a1, gs * a2);
    C x2 = fma_rn(gc, a2, -(gs * a1));
    const C td11 = fma_rn(gc, d11, gs * d12);
    const C td12 = fma_rn(gc, d12, gs * d22);
    const C td22 = fma_rn(gc, d22, -(gs * d12));
    x2 = x2 / td22;
    x1 = fma_rn(-td12, x2, x1) / td11;
    __syncwarp();
    Tt[row * kTileStride + l] = (l < row) ? T(0) : T(x1);
    Tt[(row + 1) * kTileStride + l] = (l < row) ? T(0) : T(x2);
    const C r1 = fma_rn(x1, d11, x2 * d12);
    const C r2 = fma_rn(x1, d12, x2 * d22);
    for (int i = row + 2; i < len; ++i) {
        const C l1 = shfl(r1, i), l2 = shfl(r2, i);
        Tt[i * kTileStride + l] = T(C(Tt[i * kTileStride + l]) - fma_rn(l1, x1, l2 * x2));
    }
    __syncwarp();
}

template <class T>
__device__ __forceinline__ void step_2x2(T* Tt, T* D, int row, int len, double piv64)
{
    const int l = lane_id();
    T d11 = Tt[row * kTileStride + row];
    const T d12 = Tt[row * kTileStride + row + 1];
    T d22 = Tt[(row + 1) * kTileStride + row + 1];
    const bool modified = fabs(fma_rn(d11, d22, -(d12 * d12))) < 1e-8;
    if (modified) { d11 = T(1e-6); d22 = T(1e-6); }
    if (wide_2x2(d11, d12, d22, piv64))
        step_2x2_in<T, double>(Tt, row, len, d11, d12, d22);
    else
        step_2x2_in<T, T>(Tt, row, len, d11, d12, d22);
    if (modified && l == 0) {
        Tt[row * kTileStride + row] = T(1);
        Tt[row * kTileStride + row + 1] = T(0);
        Tt[(row + 1) * kTileStride + row + 1] = T(1);
    }
    if (l < 3) {
        D[3 * row + l] = (l == 0) ? T(0) : ((l == 1) ? d11 : d12);
        D[3 * (row + 1) + l] = (l == 2) ? T(0) : ((l == 0) ? d12 : d22);
    }
    __syncwarp();
}

template <class T>
__device__ __forceinline__ void factorize_tile(T* Tt, int len, int* is_piv, T* D, int* perm, int method,
                                               double piv64)
{
    const bool use_piv = method != CULIPX_PIV_STATIC;
    int p = 0;
    while (p < len) {
        int order = 1, p0 = p, p1 = p + 1;
        if (p < len - 1 && method == CULIPX_PIV_BK) select_bk(Tt, p, len, order, p0, p1);
        else if (p < len - 1 && method == CULIPX_PIV_ROOK) select_rook(Tt, p, len, order, p0, p1);
        else order = (p < len - 1 && !is_piv[p + 1]) ? 2 : 1;
        // lane 0 decides for the warp; for finite tiles every lane already
        // agrees, and the clamp keeps the pivot rows inside the tile whatever
        // the values (non-finite input yields a non-finite factor, no stray
        // swap)
        order = shfl(order, 0);
        p0 = shfl(p0, 0);
        p1 = shfl(p1, 0);
        if (p0 < p || p0 >= len || (order == 2 && (p1 <= p || p1 >= len))) {
            order = 1;
            p0 = p;
        }
        __syncwarp();
        if (order == 1) {
            if (use_piv && p != p0) pivot_swap(Tt, perm, p, p0, len);
            step_1x1(Tt, D, p, len);
            if (use_piv && lane_id() == 0) is_piv[p] = 1;
        } else {
            if (use_piv) {
                if (p0 != p) pivot_swap(Tt, perm, p, p0, len);
                pivot_swap(Tt, perm, p + 1, p1, len);
            }
            step_2x2(Tt, D, p, len, piv64);
            if (use_piv && lane_id() == 0) { is_piv[p] = 1; is_piv[p + 1] = 0; }
        }
        __syncwarp();
        p += order;
    }
}

// ------------------------------- kernels ----------------------------------

}  // namespace culipx
