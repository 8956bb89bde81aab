// Level-scheduled numeric block-iLDL^T factorization on sm_100a.
//
// Semantics follow the reference kernels in
// libs/la/preconditioner/block_ildlt_kernels.impl.cuh (cited per kernel);
// the execution model is this library's own:
//
//  * one warp per block, the block as a 32x32 tile in shared memory with a
//    padded stride, four warps (blocks) per CTA;
//  * Schur updates A_ij -= U_ki' D_k U_kj are enumerated sparsely
//    (schur_update, pivot_tile.cuh): only non-zero terms are accumulated, in
//    ascending inner index, with explicit fma, which equals the reference's
//    dense 32x32x32 product bit for bit up to signed zeros; each update's
//    product is rounded on its own and then subtracted, as the reference does;
//  * Bunch-Kaufman / Rook / static 1x1-2x2 pivoting runs warp-parallel on the
//    tile;
//  * blocks are written straight to their final storage (sparse entries in
//    row-major order, |v| <= NZ_EPS dropped); there is no per-level in-flight
//    32x32 staging buffer.  Blocks that need the reference's dual dropping
//    (k_apply_block_dual_dropping, :1866-2074) -- more non-zeros than their
//    fill cap, or any sparse block when a relative threshold is set -- are
//    deferred: they are recomputed after a one-CTA scan has granted leftover
//    slots in level-list order (the reference's CTAs race on one counter;
//    this is the serialization by block order) and relocated to an arena
//    when granted extra slots.
#include "factor.h"
#include "kernels_common.cuh"
#include "block_io.cuh"
#include "pivot_tile.cuh"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

namespace culipx {

namespace {

constexpr int kWarps = 4;  // blocks per CTA

// device scalars in Factor::state
enum StateSlot { kStErr = 0, kStLeftover = 1, kStArena = 2, kStDeferred = 3, kStLevelAcc = 4, kStSlow = 5 };

// per block row flags set by the pivot kernel
enum ErrBits { kErrLeftoverNegative = 1 };

enum OffdiagMode { kFirst = 0, kCount = 1, kWrite = 2 };

struct FactorArgs {
    const DevBlock* desc;
    const int* bs;
    const int* cs_off;
    const int* csc_off;
    const int* csc_blk;
    const int* fmt;
    const int* lb;  // factor-order block list
    const int* lvl_rows;
    const int* row_offdiag_start;
    const int* nnz_init;  // A's entries per sparse block (pattern)
    long long* boff;
    int* nnz;
    int* cap;
    int* got_extra;
    int* idx;
    int* is_piv;
    int* perm;
    int* rowflags;
    long long* state;
    int* deferred;
    int* slowlist;        // off-diagonal positions left to the tiled kernel
    long long val_slots;  // first arena slot
    double piv64;         // FP32 factors: 2x2 pivots below this ratio are inverted in FP64
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

__global__ void k_init_rows(int n, int* perm, int* is_piv, int use_given)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        perm[i] = i;
        if (!use_given) is_piv[i] = 1;
    }
}

// Step 1 of a level: Schur updates + factorization of the pivot blocks
// (k_factor_pivot_blocks, :1146-1283), row norms of the pivot rows (:1259-1269).
template <class T>
__global__ void __launch_bounds__(32 * kWarps) k_pivot_blocks(FactorArgs a, T* val, T* tri, T* row_norm, int lb0,
                                                              int npiv, int method)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.state[kStDeferred] = 0;
        a.state[kStLevelAcc] = 0;
        a.state[kStSlow] = 0;
    }
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

    // The fan-in updates in column order.  The descriptors of 32 update blocks
    // are read at once (a lane each); the entries of a sparse block of up to 32
    // entries and the D of its rows are loaded while the previous block's
    // update runs.  The update order and arithmetic are those of one block at a
    // time.
    const int q_beg = a.csc_off[I];
    const int q_end = a.csc_off[I + 1] - 1;  // the last block of the column is the pivot
    for (int q0 = q_beg; q0 < q_end; q0 += 32) {
        const int nb = min(32, q_end - q0);
        int c_bw = 0, c_trow = 0, c_cnt = 0, c_dense = 0;
        long long c_off = 0;
        if (lane < nb) {
            const int kb = a.csc_blk[q0 + lane];
            const int K = a.desc[kb].row;
            c_trow = a.bs[K];
            c_bw = a.bs[K + 1] - c_trow;
            c_off = a.boff[kb];
            c_dense = a.fmt[kb] == 1;
            c_cnt = c_dense ? 0 : a.nnz[kb];
        }
        // block j's prefetched entry (lane e < cnt) and D rows (lane < bw)
        auto fetch = [&](int j, int& li, T& v, T& sup, T& dia, T& sub) {
            const int bw = shfl(c_bw, j), cnt = shfl(c_cnt, j), trow = shfl(c_trow, j);
            const long long off = shfl(c_off, j);
            const bool small = !shfl(c_dense, j) && cnt <= 32;
            li = 0;
            v = T(0);
            if (small && lane < cnt) {
                li = a.idx[off + lane];
                v = val[off + lane];
            }
            sup = dia = sub = T(0);
            if (lane < bw) {
                const T* tk = tri + 3 * (size_t)(trow + lane);
                sup = tk[0];
                dia = tk[1];
                sub = tk[2];
            }
        };
        int li;
        T v, sup, dia, sub;
        fetch(0, li, v, sup, dia, sub);
        for (int j = 0; j < nb; ++j) {
            int nli = 0;
            T nv = T(0), nsup = T(0), ndia = T(0), nsub = T(0);
            if (j + 1 < nb) fetch(j + 1, nli, nv, nsup, ndia, nsub);
            const int bw = shfl(c_bw, j), cnt = shfl(c_cnt, j);
            const long long off = shfl(c_off, j);
            const bool dense = shfl(c_dense, j);
            const bool small = !dense && cnt <= 32;
            unsigned cm;
            if (small) {  // the placement load_block_at does, from registers
                const int r = li / len, c = li - r * len;
                if (lane < cnt) Q[r * kTileStride + c] = v;
                cm = (lane < cnt && v != T(0)) ? (1u << c) : 0u;
                for (int o = 16; o > 0; o >>= 1) cm |= __shfl_xor_sync(0xffffffffu, cm, o);
                __syncwarp();
                schur_update_d(Tt, Q, Q, cm, bw, len, sup, dia, sub);
                if (lane < cnt) Q[r * kTileStride + c] = T(0);
                __syncwarp();
            } else {
                cm = load_block_at(Q, bw, len, dense, off, cnt, val, a.idx, false);
                schur_update_d(Tt, Q, Q, cm, bw, len, sup, dia, sub);
                unload_block_at(Q, bw, len, dense, off, cnt, a.idx);
            }
            li = nli;
            v = nv;
            sup = nsup;
            dia = ndia;
            sub = nsub;
        }
    }
    __syncwarp();
    // A diagonal tile under BK / Rook pivoting takes a 1x1 pivot at every step
    // without swaps (the off-diagonal maximum is 0); each step leaves U = I and
    // D = the diagonal (perturbed to 1e-6 below 1e-8, d_ldlt_1x1_step :556-560),
    // all other updates being fma(-0, x, y).  Done directly:
    bool diag = true;
    for (int i = 0; i < len; ++i) diag &= (lane == i || lane >= len || Tt[i * kTileStride + lane] == T(0));
    diag = __all_sync(0xffffffffu, diag) && method != CULIPX_PIV_STATIC;
    if (diag) {
        T* D = tri + 3 * (size_t)from;
        if (lane < len) {
            T d = Tt[lane * kTileStride + lane];
            if (fabs(d) < 1e-8) d = T(1e-6);
            Tt[lane * kTileStride + lane] = T(1);
            D[3 * lane] = T(0);
            D[3 * lane + 1] = d;
            D[3 * lane + 2] = T(0);
            a.is_piv[from + lane] = 1;
        }
        __syncwarp();
    } else {
        factorize_tile(Tt, len, a.is_piv + from, tri + 3 * (size_t)from, a.perm + from, method, a.piv64);
    }
    const bool perm_ident = __all_sync(0xffffffffu, lane >= len || a.perm[from + lane] == from + lane);
    const bool no_updates = (q_end == q_beg);

    if (row_norm) {
        T rs = T(0);
        for (int j = 0; j < len; ++j) rs = fma_rn(Tt[lane * kTileStride + j], Tt[lane * kTileStride + j], rs);
        if (lane < len) row_norm[from + lane] = rs;
    }

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
    if (lane == 0)
        a.rowflags[I] = (ident ? kRowIdentity : 0) | (two ? kRowHas2x2 : 0) | (perm_ident ? kRowPermIdentity : 0) |
                        (no_updates ? kRowNoUpdates : 0);
}

// U_ij entry (row r of the block) from A_ij's entry v: the Givens-form left
// solve with the 1x1 pivot D_r
template <class T>
__device__ __forceinline__ T offdiag_fast_entry(const T* D, int h, int r, T v)
{
    const T d11 = D[3 * r + 1], d12 = D[3 * r + 2];
    const T d22 = (r < 31) ? ((r + 1 < h) ? D[3 * (r + 1) + 1] : T(0)) : D[3 * 31 + 1];
    const T gr = sqrt(fma_rn(d11, d11, d12 * d12));
    const T gc = d11 / gr, gs = d12 / gr;
    const T td11 = fma_rn(gc, d11, gs * d12);
    const T td12 = fma_rn(gc, d12, gs * d22);
    T x1 = fma_rn(gc, v, gs * T(0));
    x1 = fma_rn(-td12, T(0), x1) / td11;
    return x1;
}

// Off-diagonal blocks of rows with no fan-in updates, an identity pivot tile,
// 1x1 pivots only and no swaps: U_ij = D_i^-1 A_ij entry by entry, with the
// same Givens-form arithmetic as the tiled path (d_left_solve_with_D_Ut
// :1536-1557 reduces to x = (c a) / |d|); |u| <= NZ_EPS dropped, compacted in
// place in row-major order.  Every other block goes to the slow list that
// k_offdiag<kFirst> processes.
//
// A warp takes 32 consecutive blocks of the level's list, a lane each for the
// descriptors; fast blocks of up to kLaneEntries entries are done by their
// lane (the entries in order, so the compaction is the warp path's), larger
// ones by the whole warp.  The level's leftover capacity is summed per warp
// and added once.
constexpr int kLaneEntries = 8;

template <class T>
__global__ void k_offdiag_fast(FactorArgs a, T* val, const T* tri, int lb_first, int noff, int allow)
{
    const int lane = lane_id();
    const int nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long left = 0;  // this lane's share of the level's leftover capacity
    for (int t0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; t0 < noff; t0 += nw * 32) {
        const int t = t0 + lane;
        int b = 0, cnt = 0, from = 0, h = 0, w = 1;
        long long off = 0;
        bool fast = false;
        if (t < noff) {
            b = a.lb[lb_first + t];
            const DevBlock d = a.desc[b];
            const int flags = a.rowflags[d.row];
            fast = allow && a.fmt[b] == 0 &&
                   (flags & (kRowIdentity | kRowHas2x2 | kRowPermIdentity | kRowNoUpdates)) ==
                       (kRowIdentity | kRowPermIdentity | kRowNoUpdates);
            from = a.bs[d.row];
            h = a.bs[d.row + 1] - from;
            w = a.bs[d.col + 1] - a.bs[d.col];
            off = d.val_off;
            cnt = a.nnz_init[b];
        }
        // every other block goes to the slow list
        const bool slow = t < noff && !fast;
        const unsigned sm = __ballot_sync(0xffffffffu, slow);
        if (sm) {
            int base = 0;
            if (lane == 0)
                base = (int)atomicAdd(reinterpret_cast<unsigned long long*>(&a.state[kStSlow]),
                                      (unsigned long long)__popc(sm));
            base = shfl(base, 0);
            if (slow) a.slowlist[base + __popc(sm & ((1u << lane) - 1u))] = t;
        }
        if (fast && cnt <= kLaneEntries) {
            const T* D = tri + 3 * (size_t)from;
            int o = 0;
            for (int e = 0; e < cnt; ++e) {
                const int li = a.idx[off + e];
                const T u = offdiag_fast_entry(D, h, li / w, val[off + e]);
                if (fabs(u) > T(kNzEps)) {
                    val[off + o] = u;
                    a.idx[off + o] = li;
                    ++o;
                }
            }
            a.nnz[b] = o;
            left += (unsigned long long)(long long)(a.cap[b] - o);
        }
        unsigned big = __ballot_sync(0xffffffffu, fast && cnt > kLaneEntries);
        while (big) {
            const int src = __ffs(big) - 1;
            big &= big - 1;
            const int bb = shfl(b, src), bcnt = shfl(cnt, src), bh = shfl(h, src), bw = shfl(w, src);
            const long long boff = shfl(off, src);
            const T* D = tri + 3 * (size_t)shfl(from, src);
            int o = 0;
            for (int base = 0; base < bcnt; base += 32) {
                const int e = base + lane;
                const bool valid = e < bcnt;
                const int li = valid ? a.idx[boff + e] : 0;
                const T v = valid ? val[boff + e] : T(0);
                const T u = valid ? offdiag_fast_entry(D, bh, li / bw, v) : T(0);
                const bool nz = valid && fabs(u) > T(kNzEps);
                const unsigned m = __ballot_sync(0xffffffffu, nz);
                if (nz) {
                    const int pos = o + __popc(m & ((1u << lane) - 1u));
                    val[boff + pos] = u;
                    a.idx[boff + pos] = li;
                }
                o += __popc(m);
            }
            if (lane == 0) {
                a.nnz[bb] = o;
                left += (unsigned long long)(long long)(a.cap[bb] - o);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) left += __shfl_xor_sync(0xffffffffu, left, o);
    if (lane == 0 && left) atomicAdd(reinterpret_cast<unsigned long long*>(&a.state[kStLevelAcc]), left);
}

// Off-diagonal block (I, J) up to its final values in Tt: fan-in updates over
// the block columns I and J, the pivot block's row permutation and the left
// solve with D^-1 U'^-1 (k_update_scale_offdiagonal_blocks, :1628-1778, with
// d_left_solve_with_D_Ut :1489-1570).  Q and R must be zero on entry and are
// zero on exit.
template <class T>
__device__ void offdiag_tile(const FactorArgs& a, const T* val, const T* tri, int b, T* Tt, T* Q, T* R, int pivoting)
{
    const int lane = lane_id();
    const DevBlock d = a.desc[b];
    const int I = d.row, J = d.col;
    const int from = a.bs[I], h = a.bs[I + 1] - from;
    const int w = a.bs[J + 1] - a.bs[J];

    // the block's own input (A's entries) stays at its pattern slot until the
    // block is written; a deferred block may already be relocated and its nnz
    // hold the survivor count
    const bool dense = a.fmt[b] == 1;
    load_block_at(Tt, h, w, dense, (long long)d.val_off, dense ? 0 : a.nnz_init[b], val, a.idx, true);

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

    const int flags = a.rowflags[I];
    const bool ident = flags & 1;
    const int pb = a.csc_blk[a.csc_off[I + 1] - 1];
    const long long poff = a.boff[pb];
    if (!ident && lane < h)
        for (int i = 0; i < h; ++i) Q[i * kTileStride + lane] = val[poff + (long long)i * h + lane];
    __syncwarp();
    unsigned colmask = 0;
    for (int i = 0; i < h; ++i)
        colmask |= __ballot_sync(0xffffffffu, lane < w && Tt[i * kTileStride + lane] != T(0));
    const T* D = tri + 3 * (size_t)from;
    const int* ip_row = a.is_piv + from;
    const T d11 = (lane < h) ? D[3 * lane + 1] : T(0);
    const T d12 = (lane < h) ? D[3 * lane + 2] : T(0);
    T d22 = shfl(d11, (lane < 31) ? lane + 1 : 31);
    if (lane == h) d22 = T(0);
    const bool piv1 = lane < h && ip_row[lane];
    const bool piv2 = (lane + 1) < h && !ip_row[lane + 1];
    const T gr = sqrt(fma_rn(d11, d11, d12 * d12));
    const T gc = d11 / gr, gs = d12 / gr;
    const T td11 = fma_rn(gc, d11, gs * d12);
    const T td12 = fma_rn(gc, d12, gs * d22);
    const T td22 = fma_rn(gc, d22, -(gs * d12));
    // an ill-conditioned 2x2 pivot of an FP32 factor: the same solve in FP64
    const bool wide = piv2 && wide_2x2(d11, d12, d22, a.piv64);
    const double wr = sqrt(fma_rn((double)d11, (double)d11, (double)d12 * (double)d12));
    const double wc = (double)d11 / wr, ws = (double)d12 / wr;
    const double w11 = fma_rn(wc, (double)d11, ws * (double)d12);
    const double w12 = fma_rn(wc, (double)d12, ws * (double)d22);
    const double w22 = fma_rn(wc, (double)d22, -(ws * (double)d12));
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
        T x1, x2;
        if (wide) {
            double y1 = fma_rn(wc, (double)rhs, ws * (double)right);
            double y2 = fma_rn(wc, (double)right, -(ws * (double)rhs));
            y2 = y2 / w22;
            y1 = fma_rn(-w12, y2, y1) / w11;
            x1 = T(y1);
            x2 = T(y2);
        } else {
            x1 = fma_rn(gc, rhs, gs * right);
            x2 = fma_rn(gc, right, -(gs * rhs));
            x2 = piv2 ? (x2 / td22) : T(0);
            x1 = fma_rn(-td12, x2, x1) / td11;
        }
        __syncwarp();
        if (piv1) Tt[lane * kTileStride + j] = x1;
        if (piv2) Tt[(lane + 1) * kTileStride + j] = x2;
        __syncwarp();
    }
    if (!ident) {
        if (lane < h)
            for (int i = 0; i < h; ++i) Q[i * kTileStride + lane] = T(0);
        __syncwarp();
    }
}

// threshold dropping (:1923-1945): zero |v| < threshold * ||row|| (non-zeros
// only) and count the survivors with |v| > NZ_EPS
template <class T>
__device__ int drop_and_count(T* Tt, int h, int w, const T* row_norm, int from, T threshold)
{
    const int lane = lane_id();
    int total = 0;
    for (int i = 0; i < h; ++i) {
        T v = (lane < w) ? Tt[i * kTileStride + lane] : T(0);
        bool drop = false;
        if (row_norm) {
            const T nrm = (T)sqrtf((float)row_norm[from + i]);
            drop = fabs(v) < threshold * nrm;
            if (drop && fabs(v) > T(kNzEps) && lane < w) Tt[i * kTileStride + lane] = T(0);
        }
        total += __popc(__ballot_sync(0xffffffffu, lane < w && !drop && fabs(v) > T(kNzEps)));
    }
    __syncwarp();
    return total;
}

// row-major compressed write of the entries with |v| > NZ_EPS (d_save_block)
// or, with keep != nullptr, of the tile positions flagged in keep
template <class T>
__device__ void write_sparse(const T* Tt, int h, int w, T* val, int* idx, long long off, const unsigned* keep)
{
    const int lane = lane_id();
    int o = 0;
    for (int i = 0; i < h; ++i) {
        const T v = (lane < w) ? Tt[i * kTileStride + lane] : T(0);
        const bool nz = lane < w && (keep ? ((keep[i] >> lane) & 1u) : (fabs(v) > T(kNzEps)));
        const unsigned m = __ballot_sync(0xffffffffu, nz);
        if (nz) {
            const int pos = o + __popc(m & ((1u << lane) - 1u));
            val[off + pos] = v;
            idx[off + pos] = i * w + lane;
        }
        o += __popc(m);
    }
}

// keep the `k` largest |v| (ties to the lower tile index, as CUB's stable
// descending radix sort in :2016-2061), flagged per row in keep[32]; a
// warp-level bitonic sort of (|v|, index) in the scratch tiles K, X
template <class T>
__device__ void select_largest(const T* Tt, int h, int w, int k, T* K, int* X, unsigned* keep)
{
    const int lane = lane_id();
    for (int e = lane; e < 1024; e += 32) {
        const int r = e >> 5, c = e & 31;
        K[e] = (r < h && c < w) ? fabs(Tt[r * kTileStride + c]) : T(0);
        X[e] = e;
    }
    __syncwarp();
    // sort descending by key, ascending by index: "a before b" when ka > kb or (ka == kb and ia < ib)
    for (int size = 2; size <= 1024; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int pidx = lane; pidx < 512; pidx += 32) {
                const int lo = 2 * pidx - (pidx & (stride - 1));
                const int hi = lo + stride;
                const bool up = ((lo & size) == 0);
                const T ka = K[lo], kb = K[hi];
                const int ia = X[lo], ib = X[hi];
                const bool a_first = (ka > kb) || (ka == kb && ia < ib);
                if (a_first != up) {
                    K[lo] = kb; K[hi] = ka;
                    X[lo] = ib; X[hi] = ia;
                }
            }
            __syncwarp();
        }
    if (lane < 32) keep[lane] = 0;
    __syncwarp();
    for (int e = lane; e < k; e += 32) {
        const int pos = X[e];
        atomicOr(&keep[pos >> 5], 1u << (pos & 31));
    }
    __syncwarp();
}

// Step 2: off-diagonal blocks.  kFirst: every block of the level; kCount /
// kWrite: the deferred list.
template <class T, int MODE>
__global__ void __launch_bounds__(32 * kWarps) k_offdiag(FactorArgs a, T* val, const T* tri, int lb_first, int noff,
                                                         int pivoting, T* row_norm, T* norm_part, T threshold)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int warp = threadIdx.x >> 5;
    const int lane = lane_id();
    T* Tt = smem + (size_t)warp * 3 * kTileElems;
    T* Q = Tt + kTileElems;
    T* R = Q + kTileElems;
    __shared__ unsigned keep_all[kWarps][32];

    const int count = (int)a.state[(MODE == kFirst) ? kStSlow : kStDeferred];
    const int nw = gridDim.x * kWarps;
    for (int t = blockIdx.x * kWarps + warp; t < count; t += nw) {
        // position in the level's off-diagonal list
        const int pos = (MODE == kFirst) ? a.slowlist[t] : a.deferred[t];
        const int b = a.lb[lb_first + pos];
        const DevBlock d = a.desc[b];
        const int from = a.bs[d.row], h = a.bs[d.row + 1] - from;
        const int w = a.bs[d.col + 1] - a.bs[d.col];
        const bool sparse = a.fmt[b] == 0;
        for (int e = lane; e < kTileElems; e += 32) { Q[e] = T(0); R[e] = T(0); }
        __syncwarp();
        offdiag_tile(a, val, tri, b, Tt, Q, R, pivoting);
        const long long off = a.boff[b];

        if (MODE == kFirst) {
            if (norm_part) {
                // row norms are needed before any dropping: record this block's
                // row sums (:1783-1794) and defer sparse blocks
                T rs = T(0);
                for (int j = 0; j < w; ++j) rs = fma_rn(Tt[lane * kTileStride + j], Tt[lane * kTileStride + j], rs);
                if (lane < h) norm_part[(size_t)pos * 32 + lane] = rs;
            }
            if (!sparse) {
                if (lane < w)
                    for (int i = 0; i < h; ++i) val[off + (long long)i * w + lane] = Tt[i * kTileStride + lane];
                if (lane == 0) a.nnz[b] = 0;
                continue;
            }
            if (norm_part) {
                if (lane == 0) {
                    const int slot = (int)atomicAdd(reinterpret_cast<unsigned long long*>(&a.state[kStDeferred]), 1ull);
                    a.deferred[slot] = pos;
                }
                continue;
            }
            const int total = drop_and_count<T>(Tt, h, w, nullptr, from, T(0));
            const int cp = a.cap[b];
            if (total <= cp) {
                write_sparse(Tt, h, w, val, a.idx, off, nullptr);
                if (lane == 0) {
                    a.nnz[b] = total;
                    atomicAdd(reinterpret_cast<unsigned long long*>(&a.state[kStLevelAcc]),
                              (unsigned long long)(long long)(cp - total));
                }
            } else if (lane == 0) {
                a.nnz[b] = total;  // the count, for the grant scan; entries come in kWrite
                const int slot = (int)atomicAdd(reinterpret_cast<unsigned long long*>(&a.state[kStDeferred]), 1ull);
                a.deferred[slot] = pos;
            }
            continue;
        }
        const int total = drop_and_count<T>(Tt, h, w, row_norm, from, threshold);
        if (MODE == kCount) {
            if (lane == 0) a.nnz[b] = total;
            continue;
        }
        const int cp = a.cap[b];  // after grants
        if (total <= cp) {
            write_sparse(Tt, h, w, val, a.idx, off, nullptr);
            if (lane == 0) a.nnz[b] = total;
        } else {
            unsigned* keep = keep_all[warp];
            select_largest(Tt, h, w, cp, Q, reinterpret_cast<int*>(R), keep);
            write_sparse(Tt, h, w, val, a.idx, off, keep);
            if (lane == 0) a.nnz[b] = cp;
            for (int e = lane; e < kTileElems; e += 32) { Q[e] = T(0); R[e] = T(0); }
            __syncwarp();
        }
    }
}

// row norms: pivot row sums + the off-diagonal row sums in level-list order
template <class T>
__global__ void k_row_norms(FactorArgs a, T* row_norm, const T* norm_part, int lvl0, int nrows)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= nrows) return;
    const int lane = lane_id();
    const int I = a.lvl_rows[lvl0 + warp];
    const int from = a.bs[I], h = a.bs[I + 1] - from;
    const int s = a.row_offdiag_start[lvl0 + warp];
    const int cnt = a.cs_off[I + 1] - a.cs_off[I] - 1;
    if (lane >= h) return;
    T acc = row_norm[from + lane];
    for (int j = 0; j < cnt; ++j) acc = acc + norm_part[(size_t)(s + j) * 32 + lane];
    row_norm[from + lane] = acc;
}

// Dual-dropping bookkeeping of one level (:1949-2008): grants from the
// leftover pool, capacity updates and arena relocation of the blocks granted
// extra slots.  In the reference every block of a level is a CTA that takes
// from one atomic counter before it returns its own spare slots, so a level's
// requests are served from the pool the earlier levels left, and the level's
// spare slots join the pool for the levels after it; which of a level's
// requests wins a contended slot is a race there.  Here the requests are
// served in level-list order.  One CTA; a request is x -> max(x - req, 0),
// which composes as x -> max(x + a, b): per-thread chunks are composed,
// scanned, then replayed; the spare slots are summed on the side.
constexpr long long kNeg = LLONG_MIN / 4;
constexpr int kScanT = 1024;

__global__ void __launch_bounds__(kScanT) k_level_scan(FactorArgs a, int lb_first, int noff)
{
    __shared__ long long fa[kScanT], fb[kScanT], rel[kScanT];
    const int tid = threadIdx.x;
    if (a.state[kStDeferred] == 0) {
        if (tid == 0) a.state[kStLeftover] += a.state[kStLevelAcc];
        return;
    }
    const int chunk = (noff + kScanT - 1) / kScanT;
    const int t0 = min(noff, tid * chunk), t1 = min(noff, t0 + chunk);
    long long A = 0, B = kNeg, spare = 0;
    for (int t = t0; t < t1; ++t) {
        const int b = a.lb[lb_first + t];
        if (a.fmt[b] != 0) continue;
        const long long c = a.nnz[b], m = a.cap[b];
        if (c > m) {  // a request of c - m slots: x -> max(x - (c - m), 0)
            A = A - (c - m);
            B = max(max(B - (c - m), 0LL), kNeg);
        } else {
            spare += m - c;
        }
    }
    fa[tid] = A;
    fb[tid] = B;
    rel[tid] = spare;
    __syncthreads();
    if (tid == 0) {
        // the level's spare slots, for the pool after the level
        long long s = 0;
        for (int k = 0; k < kScanT; ++k) s += rel[k];
        rel[0] = s;
    }
    __syncthreads();
    const long long level_spare = rel[0];
    __syncthreads();
    if (tid == 0) {
        // exclusive scan of the compositions: prefix_t = f_{t-1} o ... o f_0
        long long pa = 0, pb = kNeg;
        for (int k = 0; k < kScanT; ++k) {
            const long long ca = fa[k], cb = fb[k];
            fa[k] = pa;
            fb[k] = pb;
            const long long na = pa + ca;
            const long long nb = max(max(pb + ca, cb), kNeg);
            pa = na;
            pb = nb;
        }
    }
    __syncthreads();
    const long long x0 = a.state[kStLeftover];
    long long x = max(x0 + fa[tid], fb[tid]);
    long long my_rel = 0;
    for (int t = t0; t < t1; ++t) {
        const int b = a.lb[lb_first + t];
        if (a.fmt[b] != 0) continue;
        const long long c = a.nnz[b], m = a.cap[b];
        if (c > m) {
            const long long req = c - m;
            long long g = min(req, x);
            if (g < 0) g = 0;
            x -= g;
            a.got_extra[b] = (int)g;
            a.cap[b] = (int)(m + g);
            if (g > 0) my_rel += m + g;
        }
    }
    rel[tid] = my_rel;
    __syncthreads();
    if (tid == kScanT - 1) a.state[kStLeftover] = x + level_spare;  // the last chunk ends the level
    if (tid == 0) {
        long long s = 0;
        for (int k = 0; k < kScanT; ++k) {
            const long long v = rel[k];
            rel[k] = s;
            s += v;
        }
    }
    __syncthreads();
    const long long base = a.val_slots + a.state[kStArena];
    long long o = base + rel[tid];
    for (int t = t0; t < t1; ++t) {
        const int b = a.lb[lb_first + t];
        if (a.fmt[b] != 0 || a.got_extra[b] == 0) continue;
        a.boff[b] = o;
        o += a.cap[b];
    }
    __syncthreads();
    if (tid == kScanT - 1) a.state[kStArena] = o - a.val_slots;
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
    int inv = lane;  // inv[c] = l with lp[l] == c
    for (int l = 0; l < bw; ++l) {
        const int v = shfl(lp, l);
        if (v == lane) inv = l;
    }
    if (__all_sync(0xffffffffu, lane >= bw || inv == lane)) return;
    __shared__ int inv_s[kWarps][32];
    inv_s[warp][lane] = inv;
    __syncwarp();
    // 32 blocks of the column at a time, a lane each for the descriptors;
    // sparse blocks of up to kLaneEntries entries are renumbered by their lane,
    // the others by the whole warp
    const int q_end = a.csc_off[I + 1] - 1;
    for (int q0 = a.csc_off[I]; q0 < q_end; q0 += 32) {
        const int nb = min(32, q_end - q0);
        int hh = 0, cnt = 0;
        bool dense = false;
        long long off = 0;
        if (lane < nb) {
            const int b = a.csc_blk[q0 + lane];
            const int K = a.desc[b].row;
            hh = a.bs[K + 1] - a.bs[K];
            off = a.boff[b];
            dense = a.fmt[b] != 0;
            cnt = dense ? 0 : a.nnz[b];
        }
        if (lane < nb && !dense && cnt <= kLaneEntries)
            for (int e = 0; e < cnt; ++e) {
                const int li = a.idx[off + e];
                const int r = li / bw, c = li - r * bw;
                a.idx[off + e] = r * bw + inv_s[warp][c];
            }
        unsigned rest = __ballot_sync(0xffffffffu, lane < nb && (dense || cnt > kLaneEntries));
        while (rest) {
            const int src = __ffs(rest) - 1;
            rest &= rest - 1;
            const long long boff = shfl(off, src);
            if (!shfl((int)dense, src)) {
                const int bcnt = shfl(cnt, src);
                for (int base = 0; base < bcnt; base += 32) {
                    const int e = base + lane;
                    const int li = (e < bcnt) ? a.idx[boff + e] : 0;
                    const int r = li / bw, c = li - r * bw;
                    const int nc = shfl(inv, c);
                    if (e < bcnt) a.idx[boff + e] = r * bw + nc;
                }
            } else {
                const int bh = shfl(hh, src);
                for (int i = 0; i < bh; ++i) {
                    const T v = (lane < bw) ? val[boff + (long long)i * bw + lane] : T(0);
                    const T nv = shfl(v, lp);
                    if (lane < bw) val[boff + (long long)i * bw + lane] = nv;
                }
            }
        }
    }
}

template <class T>
int set_smem_limits()
{
    static bool done = false;
    if (done) return CULIPX_OK;
    const int s2 = (int)(kWarps * 2 * kTileElems * sizeof(T)), s3 = (int)(kWarps * 3 * kTileElems * sizeof(T));
    CULIPX_CUDA(cudaFuncSetAttribute(k_pivot_blocks<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, s2));
    CULIPX_CUDA(cudaFuncSetAttribute(k_offdiag<T, kFirst>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3));
    CULIPX_CUDA(cudaFuncSetAttribute(k_offdiag<T, kCount>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3));
    CULIPX_CUDA(cudaFuncSetAttribute(k_offdiag<T, kWrite>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3));
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
    k_scatter_values<T><<<148 * 8, 256, 0, s>>>((int)p.nnz, p.d_a_dst.as<int>(), static_cast<const T*>(d_vals), val);
    ++*launches;
    CULIPX_TRY(launch_check("k_scatter_values"));

    const bool thr = f->threshold > 0.0;
    if (thr) {
        const size_t nb = (size_t)p.n * sizeof(T), pb = (size_t)std::max(p.max_level_blocks, 1) * 32 * sizeof(T);
        if (f->row_norm.bytes() < nb) CULIPX_TRY(f->row_norm.alloc(p.handle, nb));
        if (f->norm_part.bytes() < pb) CULIPX_TRY(f->norm_part.alloc(p.handle, pb));
    }
    T* row_norm = thr ? f->row_norm.as<T>() : nullptr;
    T* norm_part = thr ? f->norm_part.as<T>() : nullptr;

    FactorArgs a;
    a.desc = p.d_desc.as<DevBlock>();
    a.bs = p.d_bs.as<int>();
    a.cs_off = p.d_cs_off.as<int>();
    a.csc_off = p.d_csc_off.as<int>();
    a.csc_blk = p.d_csc_blk.as<int>();
    a.fmt = p.d_fmt.as<int>();
    a.lb = p.d_lb.as<int>();
    a.lvl_rows = p.d_lvl_rows.as<int>();
    a.row_offdiag_start = p.d_row_offdiag_start.as<int>();
    a.nnz_init = p.d_nnz_init.as<int>();
    a.boff = f->boff.as<long long>();
    a.nnz = f->nnz.as<int>();
    a.cap = f->cap.as<int>();
    a.got_extra = f->got_extra.as<int>();
    a.idx = f->idx.as<int>();
    a.is_piv = f->is_piv.as<int>();
    a.perm = f->perm.as<int>();
    a.rowflags = f->rowflags.as<int>();
    a.state = f->state.as<long long>();
    a.deferred = f->deferred.as<int>();
    a.slowlist = f->slowlist.as<int>();
    a.val_slots = p.val_slots;
    a.piv64 = f->pivot_fp64;
    const int pivoting = (f->pivot != CULIPX_PIV_STATIC);
    const size_t s3 = kWarps * 3 * kTileElems * sizeof(T);
    const T thv = (T)f->threshold;
    for (int L = 0; L < p.num_levels; ++L) {
        const int lb0 = p.lb_off[L];
        const int npiv = p.lvl_off[L + 1] - p.lvl_off[L];
        const int noff = p.lb_off[L + 1] - lb0 - npiv;
        k_pivot_blocks<T><<<(npiv + kWarps - 1) / kWarps, 32 * kWarps, kWarps * 2 * kTileElems * sizeof(T), s>>>(
            a, val, tri, row_norm, lb0, npiv, f->pivot);
        ++*launches;
        CULIPX_TRY(launch_check("k_pivot_blocks"));
        if (noff > 0) {
            const int lbf = lb0 + npiv;
            const int dgrid = (std::min(noff, 148 * 16) + kWarps - 1) / kWarps;
            k_offdiag_fast<T><<<std::min((noff + 255) / 256, 148 * 8), 256, 0, s>>>(a, val, tri, lbf, noff, thr ? 0 : 1);
            k_offdiag<T, kFirst><<<dgrid, 32 * kWarps, s3, s>>>(a, val, tri, lbf, noff, pivoting, row_norm, norm_part,
                                                               thv);
            *launches += 2;
            if (thr) {
                k_row_norms<T><<<(npiv * 32 + 255) / 256, 256, 0, s>>>(a, row_norm, norm_part, p.lvl_off[L], npiv);
                k_offdiag<T, kCount><<<dgrid, 32 * kWarps, s3, s>>>(a, val, tri, lbf, noff, pivoting, row_norm,
                                                                    nullptr, thv);
                *launches += 2;
            }
            k_level_scan<<<1, kScanT, 0, s>>>(a, lbf, noff);
            k_offdiag<T, kWrite><<<dgrid, 32 * kWarps, s3, s>>>(a, val, tri, lbf, noff, pivoting, row_norm, nullptr,
                                                                thv);
            *launches += 2;
            CULIPX_TRY(launch_check("k_offdiag"));
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

int build_sweeps(Factor* f, cudaStream_t stream, int* launches);  // solve.cu

int factor_create(Pattern* p, Factor** out)
{
    if (!p || !out) return fail(CULIPX_INVALID_ARG, "culipx_factor_create: null argument");
    auto* f = new culipx_factor_t();
    f->pat = p;
    f->precision = p->precision;
    f->vbytes = (p->precision == CULIPX_F64) ? 8 : 4;
    culipx_handle_t* h = p->handle;
    const int cnz = p->coarse_nnz, n = p->n, cm = p->num_blocks;
    // pattern layout + arena for blocks relocated by dual dropping: each
    // relocated block needs cap + grant <= 2 x its cap, summed over sparse blocks
    f->val_cap = p->val_slots + 2 * p->sparse_slots;
    long long off_slots = 0;  // capacity of the strictly off-diagonal blocks
    for (int b = 0; b < cnz; ++b)
        if (p->blk_row[b] != p->blk_col[b]) off_slots += p->desc[b].cap;
    off_slots += 2 * p->sparse_slots;
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
    al(f->deferred, (size_t)std::max(p->max_level_blocks, 1) * sizeof(int));
    al(f->slowlist, (size_t)std::max(p->max_level_blocks, 1) * sizeof(int));
    al(f->u_off, (n + 1) * sizeof(int));
    al(f->ut_off, (n + 1) * sizeof(int));
    al(f->u_col, off_slots * sizeof(int));
    al(f->ut_col, off_slots * sizeof(int));
    al(f->u_val, off_slots * f->vbytes);
    al(f->ut_val, off_slots * f->vbytes);
    al(f->piv_off, cm * sizeof(long long));
    al(f->work, (size_t)n * f->vbytes);
    {
        // packed pivot tile triangles: h_I (h_I + 1) / 2 slots per block row,
        // rounded up to 4 slots so that every tile starts on a 16-byte
        // boundary (16-byte asynchronous copies into shared memory)
        std::vector<long long> pko(cm + 1, 0);
        for (int I = 0; I < cm; ++I) {
            const long long hI = p->bs[I + 1] - p->bs[I];
            pko[I + 1] = pko[I] + (hI * (hI + 1) / 2 + 3) / 4 * 4;
        }
        if (st == CULIPX_OK) st = f->pk_off.upload(h, pko.data(), (cm + 1) * sizeof(long long));
        al(f->pk_col, (size_t)pko[cm] * f->vbytes);
        al(f->pk_row, (size_t)pko[cm] * f->vbytes);
    }
    al(f->ndmask, cm * sizeof(unsigned));
    al(f->scan_s, (cm + 1) * sizeof(int));
    al(f->scan_c, (cm + 1) * sizeof(int));
    al(f->simple_rows, (size_t)n * sizeof(int));
    al(f->cplx, cm * sizeof(int));
    al(f->citem, std::max(cm, 1) * sizeof(CItem));
    al(f->u_colp, off_slots * sizeof(int));
    al(f->dg, ((size_t)n + 32) * f->vbytes);
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
    Pattern& p = *f->pat;
    culipx_handle_t* h = p.handle;
    cudaStream_t s = h->stream;
    const int n = p.n, cnz = p.coarse_nnz;
    f->pivot = pivot;
    f->threshold = threshold;
    f->computed = false;
    int launches = 0;
    if (h_is_piv)
        for (int i = 0; i < n; ++i)
            if (h_is_piv[i] != 0 && h_is_piv[i] != 1)
                return fail(CULIPX_INVALID_ARG, "culipx_factor_compute: is_piv[%d] = %d is not 0/1", i, h_is_piv[i]);
    if (!f->capturing) CULIPX_CUDA(cudaEventRecord(h->ev_start, s));
    CULIPX_CUDA(cudaMemsetAsync(f->val.get(), 0, p.val_slots * f->vbytes, s));
    CULIPX_CUDA(cudaMemcpyAsync(f->idx.get(), p.d_idx_init.get(), p.val_slots * sizeof(int),
                                cudaMemcpyDeviceToDevice, s));
    CULIPX_CUDA(cudaMemcpyAsync(f->nnz.get(), p.d_nnz_init.get(), cnz * sizeof(int), cudaMemcpyDeviceToDevice, s));
    CULIPX_CUDA(cudaMemcpyAsync(f->cap.get(), p.d_maxnnz.get(), cnz * sizeof(int), cudaMemcpyDeviceToDevice, s));
    CULIPX_CUDA(cudaMemsetAsync(f->state.get(), 0, 16 * sizeof(long long), s));
    if (h_is_piv) CULIPX_CUDA(cudaMemcpyAsync(f->is_piv.get(), h_is_piv, n * sizeof(int), cudaMemcpyHostToDevice, s));
    k_init_rows<<<148 * 4, 256, 0, s>>>(n, f->perm.as<int>(), f->is_piv.as<int>(), h_is_piv ? 1 : 0);
    k_init_blocks<<<148 * 4, 256, 0, s>>>(cnz, p.d_desc.as<DevBlock>(), f->boff.as<long long>(),
                                          f->got_extra.as<int>());
    launches += 2;
    CULIPX_TRY(launch_check("factor init"));
    if (f->precision == CULIPX_F64) CULIPX_TRY(run_levels<double>(f, d_vals, s, &launches));
    else CULIPX_TRY(run_levels<float>(f, d_vals, s, &launches));
    CULIPX_TRY(build_sweeps(f, s, &launches));
    if (!f->capturing) CULIPX_CUDA(cudaEventRecord(h->ev_stop, s));
    f->last_launches = launches;
    h->launches += launches;
    f->computed = true;
    return CULIPX_OK;
}

Factor::~Factor()
{
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (capture_stream) cudaStreamDestroy(capture_stream);
}

// The numeric factorization from a CUDA graph: the first call for a values
// pointer / pivot / threshold runs factor_compute once (which sizes every
// buffer, so the captured run allocates nothing), then captures the same
// call's launch sequence on the handle's stream; later calls with the same
// pointer replay it as one graph launch (the values behind the pointer may
// change in between).  is_piv comes from the factor's last state (no host
// array: a pageable copy cannot be captured).
int factor_compute_graph(Factor* f, const void* d_vals, int pivot, double threshold)
{
    if (!f || !d_vals) return fail(CULIPX_INVALID_ARG, "culipx_factor_compute_graph: null argument");
    Pattern& p = *f->pat;
    culipx_handle_t* h = p.handle;
    cudaStream_t s = h->stream;
    if (!f->graph_exec || f->graph_vals != d_vals || f->graph_pivot != pivot || f->graph_threshold != threshold ||
        f->graph_piv64 != f->pivot_fp64) {
        CULIPX_TRY(factor_compute(f, d_vals, nullptr, pivot, threshold));
        if (f->graph_exec) cudaGraphExecDestroy(f->graph_exec);
        if (f->graph) cudaGraphDestroy(f->graph);
        f->graph_exec = nullptr;
        f->graph = nullptr;
        // captured on a stream of the factor's own (the handle's stream may be
        // the legacy default stream, which cannot be captured); capturing
        // runs nothing, so no ordering with the handle's stream is needed
        if (!f->capture_stream) CULIPX_CUDA(cudaStreamCreateWithFlags(&f->capture_stream, cudaStreamNonBlocking));
        const long long launches0 = h->launches;
        CULIPX_CUDA(cudaStreamBeginCapture(f->capture_stream, cudaStreamCaptureModeThreadLocal));
        h->stream = f->capture_stream;
        f->capturing = true;
        const int st = factor_compute(f, d_vals, nullptr, pivot, threshold);
        f->capturing = false;
        h->stream = s;
        h->launches = launches0;  // captured, not launched
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(f->capture_stream, &g);
        if (st != CULIPX_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return st != CULIPX_OK ? st
                                   : fail(CULIPX_CUDA_ERROR, "culipx_factor_compute_graph: capture failed: %s",
                                          cudaGetErrorString(e));
        }
        cudaGraphExec_t x = nullptr;
        if (cudaGraphInstantiate(&x, g, 0) != cudaSuccess) {
            cudaGraphDestroy(g);
            cudaGetLastError();
            return fail(CULIPX_CUDA_ERROR, "culipx_factor_compute_graph: graph instantiation failed");
        }
        f->graph = g;
        f->graph_exec = x;
        f->graph_vals = d_vals;
        f->graph_pivot = pivot;
        f->graph_threshold = threshold;
        f->graph_piv64 = f->pivot_fp64;
        f->graph_launches = f->last_launches;
        return CULIPX_OK;  // the ordinary run above factored these values
    }
    CULIPX_CUDA(cudaEventRecord(h->ev_start, s));
    CULIPX_CUDA(cudaGraphLaunch(f->graph_exec, s));
    CULIPX_CUDA(cudaEventRecord(h->ev_stop, s));
    f->pivot = pivot;
    f->threshold = threshold;
    f->computed = true;
    f->last_launches = f->graph_launches;
    h->launches += f->graph_launches;
    return CULIPX_OK;
}

int factor_export(Factor* f, int* blk_nnz, long long* blk_off, int* idx, void* val, void* tri, int* is_piv, int* perm,
                  int* got_extra, long long* total)
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
