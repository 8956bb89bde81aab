// Level-scheduled numeric block-iLDL^T factorization on sm_100a.
//
// Semantics follow the reference kernels in
// libs/la/preconditioner/block_ildlt_kernels.impl.cuh (cited per kernel);
// the execution model is this library's own:
//
//  * one warp per block, the block as a 32x32 tile in shared memory with a
//    padded stride, up to four warps (blocks) per CTA;
//  * Schur updates A_ij -= U_ki' D_k U_kj are enumerated sparsely: for every
//    output row a the warp builds row a of U_ki' D_k with the reference's
//    tridiagonal formula, ballots its non-zeros and accumulates only those
//    terms, in ascending inner index, with explicit fma.  A term with a zero
//    factor changes an fma-accumulated sum by at most the sign of a zero, so
//    the result equals the reference's dense 32x32x32 product bit for bit
//    (up to signed zeros).  Each update's product is rounded on its own and
//    then subtracted, as the reference does (d_apply_left_right_update,
//    :415-456);
//  * Bunch-Kaufman / Rook / static 1x1-2x2 pivoting runs warp-parallel on the
//    tile with lowest-index tie breaking, which is what the reference's
//    shfl_down argmax tree produces (:761-781);
//  * blocks are written straight to their final storage, sparse entries in
//    row-major order, dropping |v| <= NZ_EPS (d_save_block, :85-173);
//    there is no in-flight 32x32 staging buffer per level.
//
// All files are compiled with --fmad=false: every fused multiply-add is the
// explicit fma_rn written here.
#include "factor.h"
#include "kernels_common.cuh"
#include "block_io.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace culipx {

namespace {

constexpr int kWarps = 4;  // blocks per CTA

enum StateSlot { kStErr = 0, kStLeftover = 1 };
enum ErrBits { kErrOverflow = 1 };

template <class T>
__device__ __forceinline__ T bk_alpha() { return (T)((1.0f + sqrtf(17.0f)) / 8.0f); }

// Out[a][b] -= sum_r R[r][b] * (Q' D_k)[a][r] for a in colmask(Q), lanes b < rh.
// Q: U_ki (bw x .), R: U_kj (bw x rh); D_k from tri at the rows of block k.
// d_multiply_block_by_block_diagonal (:372-411) + d_apply_left_right_update.
template <class T>
__device__ void schur_update(T* out, const T* Q, const T* R, unsigned colmask, int bw, int rh,
                             const T* tri_k)
{
    const int lane = lane_id();
    T sup = T(0), dia = T(0), sub = T(0);
    if (lane < bw) {
        sup = tri_k[3 * lane];
        dia = tri_k[3 * lane + 1];
        sub = tri_k[3 * lane + 2];
    }
    while (colmask) {
        const int a = __ffs(colmask) - 1;
        colmask &= colmask - 1;
        T lv = T(0);
        if (lane < bw) {
            const T left = (lane > 0) ? Q[(lane - 1) * kTileStride + a] : T(0);
            const T mid = Q[lane * kTileStride + a];
            const T right = (lane < 31) ? Q[(lane + 1) * kTileStride + a] : T(0);
            lv = fma_rn(sub, right, fma_rn(sup, left, dia * mid));
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

// ---- dense pivot-block factorization (d_factor_pivot_factorize, :956-1083) ----

template <class T>
__device__ void pivot_swap(T* Tt, int* perm, int p1, int p2, int len)
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

// argmax of v over lanes, ties to the lowest index (value, index) = (v, i)
template <class T>
__device__ __forceinline__ void warp_argmax(T& v, int& i)
{
    for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
    }
}

template <class T>
__device__ __forceinline__ T warp_max(T v)
{
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
__device__ void select_bk(const T* Tt, int p, int len, int& order, int& p0, int& p1)
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
__device__ void select_rook(const T* Tt, int p, int len, int& order, int& p0, int& p1)
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
__device__ void step_1x1(T* Tt, T* D, int row, int len)
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

template <class T>
__device__ void step_2x2(T* Tt, T* D, int row, int len)
{
    const int l = lane_id();
    T d11 = Tt[row * kTileStride + row];
    const T d12 = Tt[row * kTileStride + row + 1];
    T d22 = Tt[(row + 1) * kTileStride + row + 1];
    const bool modified = fabs(fma_rn(d11, d22, -(d12 * d12))) < 1e-8;
    if (modified) { d11 = T(1e-6); d22 = T(1e-6); }
    const T a1 = (l < row) ? T(0) : Tt[row * kTileStride + l];
    const T a2 = (l < row) ? T(0) : ((l == row) ? d12 : Tt[(row + 1) * kTileStride + l]);
    const T gr = sqrt(fma_rn(d11, d11, d12 * d12));
    const T gc = d11 / gr, gs = d12 / gr;
    T x1 = fma_rn(gc, a1, gs * a2);
    T x2 = fma_rn(-gs, a1, gc * a2);
    const T td11 = fma_rn(gc, d11, gs * d12);
    const T td12 = fma_rn(gc, d12, gs * d22);
    const T td22 = fma_rn(-gs, d12, gc * d22);
    x2 = x2 / td22;
    x1 = fma_rn(-td12, x2, x1) / td11;
    __syncwarp();
    Tt[row * kTileStride + l] = (l < row) ? T(0) : x1;
    Tt[(row + 1) * kTileStride + l] = (l < row) ? T(0) : x2;
    const T r1 = fma_rn(x1, d11, x2 * d12);
    const T r2 = fma_rn(x1, d12, x2 * d22);
    for (int i = row + 2; i < len; ++i) {
        const T l1 = shfl(r1, i), l2 = shfl(r2, i);
        Tt[i * kTileStride + l] -= fma_rn(l1, x1, l2 * x2);
    }
    __syncwarp();
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
__device__ void factorize_tile(T* Tt, int len, int* is_piv, T* D, int* perm, int method)
{
    const bool use_piv = method != CULIPX_PIV_STATIC;
    int p = 0;
    while (p < len) {
        int order = 1, p0 = p, p1 = p + 1;
        if (p < len - 1 && method == CULIPX_PIV_BK) select_bk(Tt, p, len, order, p0, p1);
        else if (p < len - 1 && method == CULIPX_PIV_ROOK) select_rook(Tt, p, len, order, p0, p1);
        else order = (p < len - 1 && !is_piv[p + 1]) ? 2 : 1;
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
            step_2x2(Tt, D, p, len);
            if (use_piv && lane_id() == 0) { is_piv[p] = 1; is_piv[p + 1] = 0; }
        }
        __syncwarp();
        p += order;
    }
}

// ------------------------------- kernels ----------------------------------

struct FactorArgs {
    const DevBlock* desc;
    const int* bs;
    const int* csc_off;
    const int* csc_blk;
    const int* fmt;
    const int* lb;        // factor-order block list
    const int* lvl_rows;
    long long* boff;
    int* nnz;
    int* cap;
    int* idx;
    int* is_piv;
    int* perm;
    int* rowflags;
    long long* state;
};

template <class T>
__global__ void k_scatter_values(int nnzK, const int* __restrict__ a_dst, const T* __restrict__ kv,
                                 T* __restrict__ val)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnzK; p += gridDim.x * blockDim.x) {
        const int d = a_dst[p];
        if (d >= 0) val[d] = kv[p];
    }
}

__global__ void k_init_blocks(int cnz, const DevBlock* desc, long long* boff, int* got_extra)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < cnz; b += gridDim.x * blockDim.x) {
        boff[b] = desc[b].val_off;
        got_extra[b] = 0;
    }
}

__global__ void k_init_rows(int n, int* perm, int* is_piv, const int* h_is_piv_dev, int use_given)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        perm[i] = i;
        is_piv[i] = use_given ? h_is_piv_dev[i] : 1;
    }
}

// Step 1 of a level: Schur updates + factorization of the pivot blocks
// (k_factor_pivot_blocks, :1146-1283).
template <class T>
__global__ void __launch_bounds__(32 * kWarps) k_pivot_blocks(FactorArgs a, T* val, T* tri, int lb0,
                                                              int npiv, int method)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int warp = threadIdx.x >> 5;
    const int t = blockIdx.x * kWarps + warp;
    if (t >= npiv) return;
    const int lane = lane_id();
    T* Tt = smem + (size_t)warp * 2 * kTileElems;
    T* Q = Tt + kTileElems;

    const int b = a.lb[lb0 + t];
    const int I = a.desc[b].row;
    const int from = a.bs[I], len = a.bs[I + 1] - from;

    for (int e = lane; e < kTileElems; e += 32) Q[e] = T(0);
    load_block(Tt, b, a.desc, a.bs, a.boff, a.nnz, a.fmt, val, a.idx, true);

    const int q_end = a.csc_off[I + 1] - 1;  // the last block of the column is the pivot
    for (int q = a.csc_off[I]; q < q_end; ++q) {
        const int kb = a.csc_blk[q];
        const int K = a.desc[kb].row;
        const int bw = a.bs[K + 1] - a.bs[K];
        const unsigned cm = load_block(Q, kb, a.desc, a.bs, a.boff, a.nnz, a.fmt, val, a.idx, false);
        schur_update(Tt, Q, Q, cm, bw, len, tri + 3 * (size_t)a.bs[K]);
        unload_block(Q, kb, a.desc, a.bs, a.boff, a.nnz, a.fmt, a.idx);
    }
    __syncwarp();
    factorize_tile(Tt, len, a.is_piv + from, tri + 3 * (size_t)from, a.perm + from, method);

    // write the dense pivot tile and the row flags
    const long long off = a.boff[b];
    bool ident = true;
    if (lane < len)
        for (int i = 0; i < len; ++i) {
            const T v = Tt[i * kTileStride + lane];
            val[off + (long long)i * len + lane] = v;
            if (lane > i) ident &= (v == T(0));
            if (lane == i) ident &= (v == T(1));
        }
    ident = __all_sync(0xffffffffu, ident);
    bool two = false;
    if (lane < len) two = (tri[3 * (size_t)(from + lane) + 2] != T(0)) || (tri[3 * (size_t)(from + lane)] != T(0));
    two = __any_sync(0xffffffffu, two);
    if (lane == 0) a.rowflags[I] = (ident ? 1 : 0) | (two ? 2 : 0);
}

// Step 2 of a level: fan-in updates, row permutation, D^-1 U'^-1 scaling and
// compressed write of the off-diagonal blocks
// (k_update_scale_offdiagonal_blocks :1628-1803 + k_apply_block_dual_dropping
// :1866-2074 for the threshold-free case).
template <class T>
__global__ void __launch_bounds__(32 * kWarps) k_offdiag_blocks(FactorArgs a, T* val, const T* tri,
                                                                int lb_first, int noff, int pivoting)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int warp = threadIdx.x >> 5;
    const int t = blockIdx.x * kWarps + warp;
    if (t >= noff) return;
    const int lane = lane_id();
    T* Tt = smem + (size_t)warp * 3 * kTileElems;
    T* Q = Tt + kTileElems;
    T* R = Q + kTileElems;

    const int b = a.lb[lb_first + t];
    const DevBlock d = a.desc[b];
    const int I = d.row, J = d.col;
    const int from = a.bs[I], h = a.bs[I + 1] - from;
    const int w = a.bs[J + 1] - a.bs[J];

    for (int e = lane; e < kTileElems; e += 32) { Q[e] = T(0); R[e] = T(0); }
    load_block(Tt, b, a.desc, a.bs, a.boff, a.nnz, a.fmt, val, a.idx, true);

    // merge-walk the block columns I and J above the diagonal
    int ip = a.csc_off[I], jp = a.csc_off[J];
    const int ie = a.csc_off[I + 1] - 1, je = a.csc_off[J + 1] - 1;
    while (ip < ie && jp < je) {
        const int ib = a.csc_blk[ip], jb = a.csc_blk[jp];
        const int ir = a.desc[ib].row, jr = a.desc[jb].row;
        if (ir == jr) {
            const int bw = a.bs[ir + 1] - a.bs[ir];
            const unsigned cm = load_block(Q, ib, a.desc, a.bs, a.boff, a.nnz, a.fmt, val, a.idx, false);
            load_block(R, jb, a.desc, a.bs, a.boff, a.nnz, a.fmt, val, a.idx, false);
            schur_update(Tt, Q, R, cm, bw, w, tri + 3 * (size_t)a.bs[ir]);
            unload_block(Q, ib, a.desc, a.bs, a.boff, a.nnz, a.fmt, a.idx);
            unload_block(R, jb, a.desc, a.bs, a.boff, a.nnz, a.fmt, a.idx);
        }
        ip += (ir <= jr);
        jp += (ir >= jr);
    }

    if (pivoting) {
        // rows of the block follow the pivot block's local permutation
        for (int i = 0; i < h; ++i) R[i * kTileStride + lane] = Tt[i * kTileStride + lane];
        __syncwarp();
        for (int i = 0; i < h; ++i) {
            const int pi = a.perm[from + i] - from;
            Tt[i * kTileStride + lane] = R[pi * kTileStride + lane];
        }
        __syncwarp();
        for (int i = 0; i < h; ++i) R[i * kTileStride + lane] = T(0);
        __syncwarp();
    }

    // left solve with D^-1 U'^-1 (d_left_solve_with_D_Ut, :1489-1570)
    const int flags = a.rowflags[I];
    const bool ident = flags & 1;
    const int pb = a.csc_blk[a.csc_off[I + 1] - 1];
    const long long poff = a.boff[pb];
    if (!ident && lane < h)
        for (int i = 0; i < h; ++i) Q[i * kTileStride + lane] = val[poff + (long long)i * h + lane];
    __syncwarp();
    unsigned colmask = 0;
    for (int i = 0; i < h; ++i) colmask |= __ballot_sync(0xffffffffu, lane < w && Tt[i * kTileStride + lane] != T(0));
    const T* D = tri + 3 * (size_t)from;
    const int* ip_row = a.is_piv + from;
    const T d11 = (lane < h) ? D[3 * lane + 1] : T(0);
    const T d12 = (lane < h) ? D[3 * lane + 2] : T(0);
    T d22 = shfl(d11, (lane < 31) ? lane + 1 : 31);
    if (lane == h) d22 = T(0);
    if (lane == 31 && h == 32) d22 = d11;
    const bool piv1 = lane < h && ip_row[lane];
    const bool piv2 = (lane + 1) < h && !ip_row[lane + 1];
    const T gr = sqrt(fma_rn(d11, d11, d12 * d12));
    const T gc = d11 / gr, gs = d12 / gr;
    const T td11 = fma_rn(gc, d11, gs * d12);
    const T td12 = fma_rn(gc, d12, gs * d22);
    const T td22 = fma_rn(-gs, d12, gc * d22);
    while (colmask) {
        const int j = __ffs(colmask) - 1;
        colmask &= colmask - 1;
        T rhs = (lane < h) ? Tt[lane * kTileStride + j] : T(0);
        if (!ident) {
            for (int i = 0; i < h; ++i) {
                const T piv = shfl(rhs / Q[i * kTileStride + i], i);
                if (lane > i && lane < h) rhs = fma_rn(-Q[i * kTileStride + lane], piv, rhs);
            }
        }
        if (lane >= h) rhs = T(0);
        const T right = shfl(rhs, (lane < 31) ? lane + 1 : 31);
        T x1 = fma_rn(gc, rhs, gs * right);
        T x2 = fma_rn(-gs, rhs, gc * right);
        x2 = piv2 ? (x2 / td22) : T(0);
        x1 = fma_rn(-td12, x2, x1) / td11;
        __syncwarp();
        if (piv1) Tt[lane * kTileStride + j] = x1;
        if (piv2) Tt[(lane + 1) * kTileStride + j] = x2;
        __syncwarp();
    }

    // compressed write (NZ_EPS dropping) or dense copy
    const long long off = a.boff[b];
    if (a.fmt[b] == 1) {
        if (lane < w)
            for (int i = 0; i < h; ++i) val[off + (long long)i * w + lane] = Tt[i * kTileStride + lane];
        if (lane == 0) a.nnz[b] = 0;
        return;
    }
    int total = 0;
    for (int i = 0; i < h; ++i)
        total += __popc(__ballot_sync(0xffffffffu, lane < w && fabs(Tt[i * kTileStride + lane]) > T(kNzEps)));
    if (total > a.cap[b]) {
        if (lane == 0) atomicOr(reinterpret_cast<unsigned long long*>(&a.state[kStErr]), (unsigned long long)kErrOverflow);
        return;
    }
    int o = 0;
    for (int i = 0; i < h; ++i) {
        const T v = (lane < w) ? Tt[i * kTileStride + lane] : T(0);
        const bool nz = lane < w && fabs(v) > T(kNzEps);
        const unsigned m = __ballot_sync(0xffffffffu, nz);
        if (nz) {
            const int pos = o + __popc(m & ((1u << lane) - 1u));
            val[off + pos] = v;
            a.idx[off + pos] = i * w + lane;
        }
        o += __popc(m);
    }
    if (lane == 0) a.nnz[b] = total;
}

// Step 3: apply each pivot block's local permutation to the columns of the
// blocks above it (k_pivot_col_blocks, :1352-1418).
template <class T>
__global__ void k_pivot_columns(FactorArgs a, T* val, int lvl0, int nrows)
{
    const int warp = threadIdx.x >> 5;
    const int t = blockIdx.x * kWarps + warp;
    if (t >= nrows) return;
    const int lane = lane_id();
    const int I = a.lvl_rows[lvl0 + t];
    const int from = a.bs[I], bw = a.bs[I + 1] - from;
    const int lp = (lane < bw) ? a.perm[from + lane] - from : lane;
    // inverse permutation via ballots: inv[c] = l with lp[l] == c
    int inv = lane;
    for (int l = 0; l < bw; ++l) {
        const int v = shfl(lp, l);
        if (v == lane) inv = l;
    }
    if (__all_sync(0xffffffffu, lane >= bw || inv == lane)) return;
    for (int q = a.csc_off[I]; q < a.csc_off[I + 1] - 1; ++q) {
        const int b = a.csc_blk[q];
        const int hh = a.bs[a.desc[b].row + 1] - a.bs[a.desc[b].row];
        const long long off = a.boff[b];
        if (a.fmt[b] == 0) {
            const int cnt = a.nnz[b];
            for (int base = 0; base < cnt; base += 32) {
                const int e = base + lane;
                const int li = (e < cnt) ? a.idx[off + e] : 0;
                const int r = li / bw, c = li - r * bw;
                const int nc = shfl(inv, c);
                if (e < cnt) a.idx[off + e] = r * bw + nc;
            }
        } else {
            for (int i = 0; i < hh; ++i) {
                const T v = (lane < bw) ? val[off + (long long)i * bw + lane] : T(0);
                const T nv = shfl(v, lp);
                if (lane < bw) val[off + (long long)i * bw + lane] = nv;
            }
        }
    }
}

}  // namespace
}  // namespace culipx

namespace culipx {

int build_sweeps(Factor* f, cudaStream_t stream, int* launches);  // solve.cu

namespace {

template <class T>
int set_smem_limits()
{
    static bool done = false;
    if (done) return CULIPX_OK;
    CULIPX_CUDA(cudaFuncSetAttribute(k_pivot_blocks<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(kWarps * 2 * kTileElems * sizeof(T))));
    CULIPX_CUDA(cudaFuncSetAttribute(k_offdiag_blocks<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(kWarps * 3 * kTileElems * sizeof(T))));
    done = true;
    return CULIPX_OK;
}

template <class T>
int run_levels(Factor* f, const void* d_vals, cudaStream_t s, int* launches)
{
    Pattern& p = *f->pat;
    CULIPX_TRY(set_smem_limits<T>());
    T* val = f->val.as<T>();
    T* tri = f->tri.as<T>();
    const int grid_n = 148 * 8;
    k_scatter_values<T><<<grid_n, 256, 0, s>>>((int)p.nnz, p.d_a_dst.as<int>(),
                                               static_cast<const T*>(d_vals), val);
    ++*launches;
    CULIPX_TRY(launch_check("k_scatter_values"));

    FactorArgs a;
    a.desc = p.d_desc.as<DevBlock>();
    a.bs = p.d_bs.as<int>();
    a.csc_off = p.d_csc_off.as<int>();
    a.csc_blk = p.d_csc_blk.as<int>();
    a.fmt = p.d_fmt.as<int>();
    a.lb = p.d_lb.as<int>();
    a.lvl_rows = p.d_lvl_rows.as<int>();
    a.boff = f->boff.as<long long>();
    a.nnz = f->nnz.as<int>();
    a.cap = f->cap.as<int>();
    a.idx = f->idx.as<int>();
    a.is_piv = f->is_piv.as<int>();
    a.perm = f->perm.as<int>();
    a.rowflags = f->rowflags.as<int>();
    a.state = f->state.as<long long>();
    const int pivoting = (f->pivot != CULIPX_PIV_STATIC);
    for (int L = 0; L < p.num_levels; ++L) {
        const int lb0 = p.lb_off[L];
        const int npiv = p.lvl_off[L + 1] - p.lvl_off[L];
        const int noff = p.lb_off[L + 1] - lb0 - npiv;
        k_pivot_blocks<T><<<(npiv + kWarps - 1) / kWarps, 32 * kWarps,
                            kWarps * 2 * kTileElems * sizeof(T), s>>>(a, val, tri, lb0, npiv, f->pivot);
        ++*launches;
        CULIPX_TRY(launch_check("k_pivot_blocks"));
        if (noff > 0) {
            k_offdiag_blocks<T><<<(noff + kWarps - 1) / kWarps, 32 * kWarps,
                                  kWarps * 3 * kTileElems * sizeof(T), s>>>(a, val, tri, lb0 + npiv, noff,
                                                                            pivoting);
            ++*launches;
            CULIPX_TRY(launch_check("k_offdiag_blocks"));
        }
        if (pivoting) {
            k_pivot_columns<T><<<(npiv + kWarps - 1) / kWarps, 32 * kWarps, 0, s>>>(a, val, p.lvl_off[L], npiv);
            ++*launches;
            CULIPX_TRY(launch_check("k_pivot_columns"));
        }
    }
    return CULIPX_OK;
}

}  // namespace

int factor_create(Pattern* p, Factor** out)
{
    if (!p || !out) return fail(CULIPX_INVALID_ARG, "culipx_factor_create: null argument");
    auto* f = new culipx_factor_t();
    f->pat = p;
    f->precision = p->precision;
    f->vbytes = (p->precision == CULIPX_F64) ? 8 : 4;
    culipx_handle_t* h = p->handle;
    const int cnz = p->coarse_nnz, n = p->n, cm = p->num_blocks;
    f->val_cap = p->val_slots;
    long long off_slots = 0;  // capacity of the strictly off-diagonal blocks
    for (int b = 0; b < cnz; ++b)
        if (p->blk_row[b] != p->blk_col[b]) off_slots += p->desc[b].cap;
    int st = CULIPX_OK;
    auto al = [&](DeviceBuffer& buf, size_t bytes) {
        if (st == CULIPX_OK) st = buf.alloc(h, bytes ? bytes : 16);
    };
    al(f->val, f->val_cap * f->vbytes);
    al(f->idx, f->val_cap * sizeof(int));
    al(f->boff, cnz * sizeof(long long));
    al(f->nnz, cnz * sizeof(int));
    al(f->cap, cnz * sizeof(int));
    al(f->got_extra, cnz * sizeof(int));
    al(f->tri, (3 * (size_t)n + 96) * f->vbytes);
    al(f->is_piv, (n + 32) * sizeof(int));
    al(f->perm, (n + 32) * sizeof(int));
    al(f->rowflags, cm * sizeof(int));
    al(f->state, 16 * sizeof(long long));
    al(f->u_off, (n + 1) * sizeof(int));
    al(f->ut_off, (n + 1) * sizeof(int));
    al(f->u_col, off_slots * sizeof(int));
    al(f->ut_col, off_slots * sizeof(int));
    al(f->u_val, off_slots * f->vbytes);
    al(f->ut_val, off_slots * f->vbytes);
    al(f->piv_off, cm * sizeof(long long));
    al(f->work, (size_t)n * f->vbytes);
    if (st != CULIPX_OK) { delete f; return st; }
    *out = f;
    return CULIPX_OK;
}

int factor_compute(Factor* f, const void* d_vals, const int* h_is_piv, int pivot, double threshold)
{
    if (!f || !d_vals) return fail(CULIPX_INVALID_ARG, "culipx_factor_compute: null argument");
    if (pivot < CULIPX_PIV_STATIC || pivot > CULIPX_PIV_ROOK)
        return fail(CULIPX_INVALID_ARG, "culipx_factor_compute: bad pivot method %d", pivot);
    if (!(threshold >= 0.0)) return fail(CULIPX_INVALID_ARG, "culipx_factor_compute: threshold < 0");
    if (threshold != 0.0)
        return fail(CULIPX_NOT_SUPPORTED, "culipx_factor_compute: threshold dropping > 0 is not implemented yet");
    Pattern& p = *f->pat;
    culipx_handle_t* h = p.handle;
    cudaStream_t s = h->stream;
    const int n = p.n, cnz = p.coarse_nnz;
    f->pivot = pivot;
    f->threshold = threshold;
    f->computed = false;
    int launches = 0;
    CULIPX_CUDA(cudaEventRecord(h->ev_start, s));
    CULIPX_CUDA(cudaMemsetAsync(f->val.get(), 0, f->val_cap * f->vbytes, s));
    CULIPX_CUDA(cudaMemcpyAsync(f->idx.get(), p.d_idx_init.get(), p.val_slots * sizeof(int),
                                cudaMemcpyDeviceToDevice, s));
    CULIPX_CUDA(cudaMemcpyAsync(f->nnz.get(), p.d_nnz_init.get(), cnz * sizeof(int), cudaMemcpyDeviceToDevice, s));
    CULIPX_CUDA(cudaMemcpyAsync(f->cap.get(), p.d_maxnnz.get(), cnz * sizeof(int), cudaMemcpyDeviceToDevice, s));
    CULIPX_CUDA(cudaMemsetAsync(f->state.get(), 0, 16 * sizeof(long long), s));
    CULIPX_CUDA(cudaMemsetAsync(f->tri.get(), 0, (3 * (size_t)n + 96) * f->vbytes, s));
    if (h_is_piv) {
        for (int i = 0; i < n; ++i)
            if (h_is_piv[i] != 0 && h_is_piv[i] != 1)
                return fail(CULIPX_INVALID_ARG, "culipx_factor_compute: is_piv[%d] = %d is not 0/1", i, h_is_piv[i]);
        CULIPX_CUDA(cudaMemcpyAsync(f->is_piv.get(), h_is_piv, n * sizeof(int), cudaMemcpyHostToDevice, s));
    }
    k_init_rows<<<148 * 4, 256, 0, s>>>(n, f->perm.as<int>(), f->is_piv.as<int>(), f->is_piv.as<int>(),
                                        h_is_piv ? 1 : 0);
    ++launches;
    k_init_blocks<<<148 * 4, 256, 0, s>>>(cnz, p.d_desc.as<DevBlock>(), f->boff.as<long long>(),
                                          f->got_extra.as<int>());
    ++launches;
    CULIPX_TRY(launch_check("factor init"));
    if (f->precision == CULIPX_F64) CULIPX_TRY(run_levels<double>(f, d_vals, s, &launches));
    else CULIPX_TRY(run_levels<float>(f, d_vals, s, &launches));
    CULIPX_TRY(build_sweeps(f, s, &launches));
    CULIPX_CUDA(cudaEventRecord(h->ev_stop, s));
    long long st[2] = {0, 0};
    CULIPX_CUDA(cudaMemcpyAsync(st, f->state.get(), sizeof(st), cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaStreamSynchronize(s));
    CULIPX_CUDA(cudaEventElapsedTime(&f->last_ms, h->ev_start, h->ev_stop));
    f->last_launches = launches;
    h->launches += launches;
    if (st[kStErr] & kErrOverflow)
        return fail(CULIPX_NOT_SUPPORTED, "culipx_factor_compute: a sparse block exceeded its fill cap (dual dropping is not implemented yet)");
    f->computed = true;
    return CULIPX_OK;
}

int factor_export(Factor* f, int* blk_nnz, long long* blk_off, int* idx, void* val, void* tri,
                  int* is_piv, int* perm, int* got_extra, long long* total)
{
    if (!f->computed) return fail(CULIPX_INVALID_ARG, "culipx_factor_export: factor not computed");
    Pattern& p = *f->pat;
    cudaStream_t s = p.handle->stream;
    const int cnz = p.coarse_nnz, n = p.n;
    std::vector<int> h_nnz(cnz), h_idx(f->val_cap), h_extra(cnz);
    std::vector<long long> h_boff(cnz);
    std::vector<unsigned char> h_val(f->val_cap * f->vbytes);
    CULIPX_CUDA(cudaMemcpyAsync(h_nnz.data(), f->nnz.get(), cnz * sizeof(int), cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaMemcpyAsync(h_boff.data(), f->boff.get(), cnz * sizeof(long long), cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaMemcpyAsync(h_extra.data(), f->got_extra.get(), cnz * sizeof(int), cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaMemcpyAsync(h_idx.data(), f->idx.get(), f->val_cap * sizeof(int), cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaMemcpyAsync(h_val.data(), f->val.get(), f->val_cap * f->vbytes, cudaMemcpyDeviceToHost, s));
    CULIPX_CUDA(cudaStreamSynchronize(s));
    long long o = 0;
    std::vector<std::pair<int, int>> ent;
    for (int b = 0; b < cnz; ++b) {
        const int r = p.bs[p.blk_row[b] + 1] - p.bs[p.blk_row[b]];
        const int c = p.bs[p.blk_col[b] + 1] - p.bs[p.blk_col[b]];
        const long long bo = h_boff[b];
        if (blk_off) blk_off[b] = o;
        if (p.fmt[b] == kDense) {
            if (blk_nnz) blk_nnz[b] = 0;
            for (int e = 0; e < r * c; ++e) {
                if (idx) idx[o + e] = e;
                if (val) std::memcpy((unsigned char*)val + (o + e) * f->vbytes, &h_val[(bo + e) * f->vbytes], f->vbytes);
            }
            o += r * c;
        } else {
            const int cnt = h_nnz[b];
            if (blk_nnz) blk_nnz[b] = cnt;
            ent.resize(cnt);
            for (int e = 0; e < cnt; ++e) ent[e] = {h_idx[bo + e], e};
            std::sort(ent.begin(), ent.end());
            for (int e = 0; e < cnt; ++e) {
                if (idx) idx[o + e] = ent[e].first;
                if (val)
                    std::memcpy((unsigned char*)val + (o + e) * f->vbytes, &h_val[(bo + ent[e].second) * f->vbytes],
                                f->vbytes);
            }
            o += cnt;
        }
        if (got_extra) got_extra[b] = h_extra[b];
    }
    if (blk_off) blk_off[cnz] = o;
    if (total) *total = o;
    if (tri) CULIPX_CUDA(cudaMemcpy(tri, f->tri.get(), 3 * (size_t)n * f->vbytes, cudaMemcpyDeviceToHost));
    if (is_piv) CULIPX_CUDA(cudaMemcpy(is_piv, f->is_piv.get(), n * sizeof(int), cudaMemcpyDeviceToHost));
    if (perm) CULIPX_CUDA(cudaMemcpy(perm, f->perm.get(), n * sizeof(int), cudaMemcpyDeviceToHost));
    return CULIPX_OK;
}

}  // namespace culipx
