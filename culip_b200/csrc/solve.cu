// Preconditioner applies for the block-iLDL^T factor: level-scheduled block
// triangular sweeps, the 1x1/2x2 block-diagonal D solve and the pivot
// permutation.
//
// Reference: solve_left / solve_middle / solve_right
// (libs/la/preconditioner/block_ildlt.impl.cuh:183-246), solve_U_block /
// solve_Ut_block (:2378-2426, :2557-2606) with k_solve_blocks_offdiagonal_atomic
// and k_solve_blocks_diagonal_atomic (block_ildlt_kernels.impl.cuh:2353-2606),
// k_solve_D and k_permute_P / k_permute_Pt (libs/la/helper_kernels.impl.cuh:720-816).
//
// Design: after the numeric factor, the strictly off-diagonal block part of
// U is re-laid out once as two fine-row CSR arrays (rows of U for the U
// sweep, rows of U' for the U' sweep), each row sorted by column.  A sweep
// level is then one warp per block row, one lane per fine row: the lane
// subtracts its row's terms in column order (no atomics, deterministic; the
// reference adds them with atomicAdd) and the warp finishes with the
// triangular solve on the dense pivot tile, skipped when the tile is exactly
// the identity (then the reference's divide-by-1 / subtract-0 steps are
// exact no-ops).
#include "factor.h"
#include "kernels_common.cuh"
#include "block_io.cuh"

#include <algorithm>

namespace culipx {

int exclusive_scan(int* d, int n, DeviceBuffer& tmp, culipx_handle_t* h, cudaStream_t s, int* launches);

namespace {

constexpr int kSweepWarps = 4;

// ---------------------------------------------------------------------------
// exclusive scan of n+1 int counts (in place), three passes
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanChunk = kScanThreads * kScanItems;

__device__ int block_exclusive_scan(int v, int* warp_sums, int* total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        int s = (lane < nw) ? warp_sums[lane] : 0;
        int si = s;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += t;
        }
        if (lane < nw) warp_sums[lane] = si - s;
        if (lane == nw - 1) *total = si;
    }
    __syncthreads();
    const int r = warp_sums[w] + incl - v;
    __syncthreads();
    return r;
}

__global__ void k_scan_chunks(int* data, int n, int* sums)
{
    __shared__ int ws[32];
    __shared__ int tot;
    const long long base = (long long)blockIdx.x * kScanChunk + threadIdx.x * kScanItems;
    int loc[kScanItems];
    int s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const long long i = base + k;
        loc[k] = (i < n) ? data[i] : 0;
        s += loc[k];
    }
    int off = block_exclusive_scan(s, ws, &tot);
    for (int k = 0; k < kScanItems; ++k) {
        const long long i = base + k;
        if (i < n) data[i] = off;
        off += loc[k];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_scan_sums(int* sums, int m)
{
    __shared__ int ws[32];
    __shared__ int tot;
    int carry = 0;
    for (int base = 0; base < m; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = (i < m) ? sums[i] : 0;
        const int e = block_exclusive_scan(v, ws, &tot);
        if (i < m) sums[i] = carry + e;
        carry += tot;
        __syncthreads();
    }
}

__global__ void k_scan_add(int* data, int n, const int* sums)
{
    const long long base = (long long)blockIdx.x * kScanChunk;
    const int add = sums[blockIdx.x];
    for (int k = threadIdx.x; k < kScanChunk; k += blockDim.x) {
        const long long i = base + k;
        if (i < n) data[i] += add;
    }
}

// ---------------------------------------------------------------------------
struct SweepBuild {
    const DevBlock* desc;
    const int* bs;
    const int* cs_off;
    const int* csc_off;
    const int* csc_blk;
    const int* fmt;
    const long long* boff;
    const int* nnz;
    const int* idx;
};

// per fine row of U and of U': number of non-zero off-diagonal entries.  A
// warp takes 32 consecutive blocks, a lane each for the descriptors; sparse
// blocks of up to kCountLane entries are counted by their lane, the others by
// the whole warp.
constexpr int kCountLane = 8;

template <class T>
__global__ void k_count_offdiag(SweepBuild a, const T* val, int nblocks_total, int* cnt_u, int* cnt_ut)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int lane = lane_id();
    for (int b0 = warp * 32; b0 < nblocks_total; b0 += nwarps * 32) {
        const int b = b0 + lane;
        int fr = 0, h = 0, fc = 0, w = 1, cnt = 0;
        bool use = false, dense = false;
        long long off = 0;
        if (b < nblocks_total) {
            const DevBlock d = a.desc[b];
            use = d.row != d.col;
            fr = a.bs[d.row];
            h = a.bs[d.row + 1] - fr;
            fc = a.bs[d.col];
            w = a.bs[d.col + 1] - fc;
            off = a.boff[b];
            dense = a.fmt[b] == 1;
            cnt = dense ? 0 : a.nnz[b];
        }
        if (use && !dense && cnt <= kCountLane)
            for (int e = 0; e < cnt; ++e) {
                if (val[off + e] == T(0)) continue;
                const int li = a.idx[off + e];
                const int r = li / w, c = li - r * w;
                atomicAdd(&cnt_u[fr + r], 1);
                atomicAdd(&cnt_ut[fc + c], 1);
            }
        unsigned rest = __ballot_sync(0xffffffffu, use && (dense || cnt > kCountLane));
        while (rest) {
            const int src = __ffs(rest) - 1;
            rest &= rest - 1;
            const int bfr = shfl(fr, src), bh = shfl(h, src), bfc = shfl(fc, src), bw = shfl(w, src);
            const long long boff = shfl(off, src);
            if (shfl((int)dense, src)) {
                int colcount = 0;
                for (int i = 0; i < bh; ++i) {
                    const bool nz = lane < bw && val[boff + (long long)i * bw + lane] != T(0);
                    const unsigned m = __ballot_sync(0xffffffffu, nz);
                    if (lane == 0 && m) atomicAdd(&cnt_u[bfr + i], __popc(m));
                    colcount += nz;
                }
                if (lane < bw && colcount) atomicAdd(&cnt_ut[bfc + lane], colcount);
            } else {
                const int bcnt = shfl(cnt, src);
                for (int e = lane; e < bcnt; e += 32) {
                    if (val[boff + e] == T(0)) continue;
                    const int li = a.idx[boff + e];
                    const int r = li / bw, c = li - r * bw;
                    atomicAdd(&cnt_u[bfr + r], 1);
                    atomicAdd(&cnt_ut[bfc + c], 1);
                }
            }
        }
    }
}

// The fill kernels below write one fine-row CSR per triangle, skipping stored
// zeros: the rows of U (warp per block row, blocks in column order, each row
// in column order) and the rows of U' = the columns of U (warp per block
// column, blocks in row order, each row in row order).  The warp reads the descriptors of 32 blocks
// at once (one lane each).  Runs of consecutive sparse blocks of 32 entries
// or fewer in total go through one batch, a lane per entry: an entry's place
// in its fine row is the count of batch entries of the same row that precede
// it in (block, column) order (in (block, row) order for U'), added to the
// row's next free position kept in shared memory.  Other blocks (dense, or
// sparse with more than 32 entries, whose columns a pivot permutation may have
// reordered) are placed in a shared tile and read back row by row.

// per-lane descriptors of the chunk of up to 32 blocks a warp handles
struct FillChunk {
    long long off;   // value / index offset of lane's block
    int first;       // fc (U) or fr (U') of lane's block
    int ext;         // w (U) or h (U') of lane's block
    int weight;      // sparse entries, or 33 for a block that takes the tile path
    int incl;        // inclusive prefix of weight over the lanes
};

constexpr int kFillBig = 33;

__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = lane_id();
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// one batch of the small sparse blocks j..k-1 of the chunk; TRANS: U' (rows
// of U' are columns of the blocks, keyed by block and row)
template <class T, bool TRANS>
__device__ __forceinline__ void fill_small_batch(const FillChunk& ch, int j, int k, int base, int wfix,
                                                 const T* val, const int* idx, int* next, int* out_col,
                                                 T* out_val)
{
    const int lane = lane_id();
    const int E = shfl(ch.incl, k - 1) - base;
    int bl = j;  // block of this lane's entry: first l with incl[l] - base > lane
    for (int l = j; l < k - 1; ++l)
        if (shfl(ch.incl, l) - base <= lane) bl = l + 1;
    const int e = lane - (shfl(ch.incl, bl) - shfl(ch.weight, bl) - base);
    const long long off = shfl(ch.off, bl);
    const int first = shfl(ch.first, bl);
    const int w = TRANS ? wfix : shfl(ch.ext, bl);
    const bool in = lane < E;
    int li = 0;
    T v = T(0);
    if (in) {
        li = idx[off + e];
        v = val[off + e];
    }
    const int r = li / w, c = li - r * w;
    const bool nz = in && v != T(0);
    const unsigned nzm = __ballot_sync(0xffffffffu, nz);
    const int row = TRANS ? c : r;          // output row within the warp's block row / column
    const int key = bl * 32 + (TRANS ? r : c);  // order within that output row
    int rank = 0;
    for (int t = 0; t < E; ++t) {
        const int rt = shfl(row, t), kt = shfl(key, t);
        rank += (int)(((nzm >> t) & 1u) && rt == row && kt < key);
    }
    if (nz) {
        const int p = next[row] + rank;
        out_col[p] = first + (TRANS ? r : c);
        out_val[p] = v;
    }
    __syncwarp();
    if (nz) atomicAdd(&next[row], 1);
    __syncwarp();
}

template <class T>
__global__ void __launch_bounds__(32 * kSweepWarps) k_fill_u_rows(SweepBuild a, const T* val, int cm,
                                                                   const int* u_off, int* u_col, T* u_val)
{
    __shared__ T tiles[kSweepWarps][kTileElems];
    __shared__ int next_s[kSweepWarps][32];
    const int warp = threadIdx.x >> 5;
    const int I = blockIdx.x * kSweepWarps + warp;
    if (I >= cm) return;
    const int lane = lane_id();
    T* tile = tiles[warp];
    int* next = next_s[warp];  // next free position of fine row fr + i
    for (int e = lane; e < kTileElems; e += 32) tile[e] = T(0);
    const int fr = a.bs[I], h = a.bs[I + 1] - fr;
    next[lane] = (lane < h) ? u_off[fr + lane] : 0;
    __syncwarp();
    const int q_end = a.cs_off[I + 1];
    for (int q0 = a.cs_off[I] + 1; q0 < q_end; q0 += 32) {
        const int nb = min(32, q_end - q0);
        FillChunk ch{0, 0, 1, kFillBig, 0};
        if (lane < nb) {
            const int q = q0 + lane;
            const int J = a.desc[q].col;
            ch.first = a.bs[J];
            ch.ext = a.bs[J + 1] - ch.first;
            ch.off = a.boff[q];
            const int cnt = (a.fmt[q] == 1) ? kFillBig : a.nnz[q];
            ch.weight = (cnt <= 32) ? cnt : kFillBig;
        }
        ch.incl = warp_incl_scan(ch.weight);
        for (int j = 0; j < nb;) {
            const int base = shfl(ch.incl, j) - shfl(ch.weight, j);
            const unsigned take = __ballot_sync(0xffffffffu, lane >= j && lane < nb && ch.incl - base <= 32);
            const int k = j + __popc(take);
            if (k > j) {
                fill_small_batch<T, false>(ch, j, k, base, 0, val, a.idx, next, u_col, u_val);
                j = k;
                continue;
            }
            const int q = q0 + j;
            const int fc = shfl(ch.first, j), w = shfl(ch.ext, j);
            load_block(tile, q, a.desc, a.bs, a.boff, a.nnz, a.fmt, val, a.idx, false);
            int mine = 0;
            for (int i = 0; i < h; ++i) {
                const T v = (lane < w) ? tile[i * kTileStride + lane] : T(0);
                const bool nz = v != T(0);
                const unsigned m = __ballot_sync(0xffffffffu, nz);
                if (nz) {
                    const int p = next[i] + __popc(m & ((1u << lane) - 1u));
                    u_col[p] = fc + lane;
                    u_val[p] = v;
                }
                if (lane == i) mine = __popc(m);
            }
            __syncwarp();
            if (lane < h) next[lane] += mine;
            unload_block(tile, q, a.desc, a.bs, a.boff, a.nnz, a.fmt, a.idx);
            ++j;
        }
    }
}

template <class T>
__global__ void __launch_bounds__(32 * kSweepWarps) k_fill_ut_rows(SweepBuild a, const T* val, int cm,
                                                                    const int* ut_off, int* ut_col, T* ut_val)
{
    __shared__ T tiles[kSweepWarps][kTileElems];
    __shared__ int next_s[kSweepWarps][32];
    const int warp = threadIdx.x >> 5;
    const int J = blockIdx.x * kSweepWarps + warp;
    if (J >= cm) return;
    const int lane = lane_id();
    T* tile = tiles[warp];
    int* next = next_s[warp];  // next free position of U' row fc + c
    for (int e = lane; e < kTileElems; e += 32) tile[e] = T(0);
    const int fc = a.bs[J], w = a.bs[J + 1] - fc;
    next[lane] = (lane < w) ? ut_off[fc + lane] : 0;
    __syncwarp();
    const int q_end = a.csc_off[J + 1] - 1;  // the pivot block closes the column
    for (int q0 = a.csc_off[J]; q0 < q_end; q0 += 32) {
        const int nb = min(32, q_end - q0);
        FillChunk ch{0, 0, 1, kFillBig, 0};
        if (lane < nb) {
            const int b = a.csc_blk[q0 + lane];
            const int K = a.desc[b].row;
            ch.first = a.bs[K];
            ch.ext = a.bs[K + 1] - ch.first;
            ch.off = a.boff[b];
            const int cnt = (a.fmt[b] == 1) ? kFillBig : a.nnz[b];
            ch.weight = (cnt <= 32) ? cnt : kFillBig;
        }
        ch.incl = warp_incl_scan(ch.weight);
        for (int j = 0; j < nb;) {
            const int base = shfl(ch.incl, j) - shfl(ch.weight, j);
            const unsigned take = __ballot_sync(0xffffffffu, lane >= j && lane < nb && ch.incl - base <= 32);
            const int k = j + __popc(take);
            if (k > j) {
                fill_small_batch<T, true>(ch, j, k, base, w, val, a.idx, next, ut_col, ut_val);
                j = k;
                continue;
            }
            const int b = a.csc_blk[q0 + j];
            const int fr = shfl(ch.first, j), h = shfl(ch.ext, j);
            load_block(tile, b, a.desc, a.bs, a.boff, a.nnz, a.fmt, val, a.idx, false);
            if (lane < w) {  // lane c owns U' row fc + c; the block's rows in order
                int p = next[lane];
                for (int i = 0; i < h; ++i) {
                    const T v = tile[i * kTileStride + lane];
                    if (v != T(0)) {
                        ut_col[p] = fr + i;
                        ut_val[p] = v;
                        ++p;
                    }
                }
                next[lane] = p;
            }
            unload_block(tile, b, a.desc, a.bs, a.boff, a.nnz, a.fmt, a.idx);
            ++j;
        }
    }
}

__global__ void k_pivot_offsets(int cm, const int* csc_off, const int* csc_blk, const long long* boff,
                                long long* piv_off)
{
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < cm; I += gridDim.x * blockDim.x)
        piv_off[I] = boff[csc_blk[csc_off[I + 1] - 1]];
}

// Upper triangle of each non-identity pivot tile, packed twice: column by
// column (U[r][c] at c(c+1)/2 + r; the U sweep's back substitution reads one
// column per step) and row by row (U[r][c] at r h - r(r-1)/2 + c - r; the U'
// sweep reads one row per step).  Both reads are coalesced, and together the
// two copies take the room of one square tile.  ndmask[I] marks the diagonal
// entries that are not exactly 1 (only the first row of a 2x2 pivot can be):
// the substitutions divide only there, x / 1 being x.
template <class T>
__global__ void k_pack_tiles(int cm, const int* __restrict__ bs, const long long* __restrict__ piv_off,
                             const int* __restrict__ rowflags, const T* __restrict__ val,
                             const long long* __restrict__ pk_off, T* __restrict__ pk_col, T* __restrict__ pk_row,
                             unsigned* __restrict__ ndmask)
{
    const int lane = lane_id();
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; I < cm; I += nw) {
        if (rowflags[I] & kRowIdentity) continue;
        const int h = bs[I + 1] - bs[I];
        const T* P = val + piv_off[I];
        const unsigned nd = __ballot_sync(0xffffffffu, (int)lane < h && P[lane * h + lane] != T(1));
        if (lane == 0) ndmask[I] = nd;
        T* pc = pk_col + pk_off[I];
        T* pr = pk_row + pk_off[I];
        for (int r = 0; r < h; ++r) {
            const int c = lane;
            if (c >= r && c < h) {
                const T v = P[r * h + c];
                pc[c * (c + 1) / 2 + r] = v;
                pr[r * h - r * (r - 1) / 2 + c - r] = v;
            }
        }
    }
}

// Simple block rows: identity pivot tile, no swaps, 1x1 pivots only.  Their
// fine rows are independent in both sweeps.
__device__ __forceinline__ bool simple_block(int flags)
{
    return (flags & (kRowIdentity | kRowPermIdentity | kRowHas2x2)) == (kRowIdentity | kRowPermIdentity);
}

// per level-list position q: fine rows of a simple block / 1 for another block
__global__ void k_split_count(int cm, const int* __restrict__ lvl_rows, const int* __restrict__ bs,
                              const int* __restrict__ rowflags, int* __restrict__ cnt_s, int* __restrict__ cnt_c)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= cm; q += gridDim.x * blockDim.x) {
        if (q == cm) {
            cnt_s[q] = 0;
            cnt_c[q] = 0;
            continue;
        }
        const int I = lvl_rows[q];
        const bool simple = simple_block(rowflags[I]);
        cnt_s[q] = simple ? bs[I + 1] - bs[I] : 0;
        cnt_c[q] = simple ? 0 : 1;
    }
}

// after the exclusive scans: the simple fine rows and the other block rows,
// both in level-list order
__global__ void k_split_fill(int cm, const int* __restrict__ lvl_rows, const int* __restrict__ bs,
                             const int* __restrict__ rowflags, const int* __restrict__ scan_s,
                             const int* __restrict__ scan_c, int* __restrict__ simple_rows, int* __restrict__ cplx,
                             const long long* __restrict__ pk_off, const unsigned* __restrict__ ndmask,
                             CItem* __restrict__ citem)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cm; q += gridDim.x * blockDim.x) {
        const int I = lvl_rows[q];
        if (simple_block(rowflags[I])) {
            const int fr = bs[I], h = bs[I + 1] - fr;
            for (int r = 0; r < h; ++r) simple_rows[scan_s[q] + r] = fr + r;
        } else {
            cplx[scan_c[q]] = I;
            CItem c;
            c.I = I;
            c.fr = bs[I];
            c.h = bs[I + 1] - c.fr;
            c.flags = rowflags[I];
            c.pk_off = pk_off[I];
            c.nd = ndmask[I];
            c.pad = 0;
            citem[scan_c[q]] = c;
        }
    }
}

// U's column indices mapped through the pivot permutation (the persistent
// solver gathers the finished U-sweep values from P t directly), and the
// diagonal of D
template <class T>
__global__ void k_sweep_extras(const int* __restrict__ u_off, const int* __restrict__ u_col,
                               const int* __restrict__ perm, int* __restrict__ u_colp, int n,
                               const T* __restrict__ tri, T* __restrict__ dg)
{
    const long long nu = u_off[n];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nu; k += stride)
        u_colp[k] = perm[u_col[k]];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n; g += stride)
        dg[g] = tri[3 * g + 1];
}

// ---------------------------------------------------------------------------
// one level of the U (UPPER) or U' sweep, warp per block row, lane per fine
// row, each row's terms in increasing column order.
//   U' (solve_left): row r starts from (P' b)_r = src[perm[r]] (src == NULL:
//   from x[r], the permuted right-hand side already there), subtracts the
//   earlier levels' x, and writes x[r].
//   U (solve_right): row r starts from src[r], subtracts the later levels'
//   values, read at their permuted places through ucol = perm[col], and
//   writes x[perm[r]]: x = P U^-1 b with the permutation folded in (src may
//   equal x: a block row writes only its own places, after reading them).
// The non-identity pivot tile's upper triangle comes packed (column by
// column for U, row by row for U', as the persistent solver reads it) and is
// staged in shared memory for the serial substitution.
template <class T, bool UPPER>
__global__ void __launch_bounds__(32 * kSweepWarps)
    k_sweep_level(const int* __restrict__ rows, int nrows, const int* __restrict__ bs,
                  const int* __restrict__ off, const int* __restrict__ col, const T* __restrict__ vals,
                  const long long* __restrict__ pk_off, const int* __restrict__ rowflags,
                  const T* __restrict__ pk, const int* __restrict__ perm, const T* src, T* x)
{
    constexpr int kTri = 32 * 33 / 2;
    __shared__ T tiles[kSweepWarps][kTri];
    const int warp = threadIdx.x >> 5;
    const int t = blockIdx.x * kSweepWarps + warp;
    if (t >= nrows) return;
    const int lane = lane_id();
    const int I = rows[t];
    const int fr = bs[I], h = bs[I + 1] - fr;
    const int flags = rowflags[I];
    const bool pid = (flags & kRowPermIdentity) != 0;
    T acc = T(0);
    if (lane < h) {
        const int g = fr + lane;
        if (UPPER) acc = src[g];
        else acc = src ? src[pid ? g : perm[g]] : x[g];
        // the row's terms in batches of 8: index and value loads, then the
        // gathers, then the fmas in column order
        constexpr int B = 8;
        const int e1 = off[g + 1];
        for (int k = off[g]; k < e1; k += B) {
            int c[B];
            T v[B], xv[B];
#pragma unroll
            for (int j = 0; j < B; ++j) {
                c[j] = (k + j < e1) ? col[k + j] : -1;
                v[j] = (k + j < e1) ? vals[k + j] : T(0);
            }
#pragma unroll
            for (int j = 0; j < B; ++j) xv[j] = (c[j] >= 0) ? x[c[j]] : T(0);
#pragma unroll
            for (int j = 0; j < B; ++j)
                if (c[j] >= 0) acc = fma_rn(-v[j], xv[j], acc);
        }
    }
    if (!(flags & kRowIdentity)) {
        T* tile = tiles[warp];
        const T* P = pk + pk_off[I];
        for (int e = lane; e < h * (h + 1) / 2; e += 32) tile[e] = P[e];
        __syncwarp();
        if (UPPER) {
            // column c of the triangle at c (c + 1) / 2: rows 0 .. c
            for (int c = h - 1; c >= 0; --c) {
                const int cb = c * (c + 1) / 2;
                if (lane == c) acc = acc / tile[cb + c];
                const T xc = shfl(acc, c);
                if (lane < c) acc = fma_rn(-tile[cb + lane], xc, acc);
            }
        } else {
            // row r of the triangle at r h - r (r - 1) / 2: columns r .. h - 1
            for (int r = 0; r < h; ++r) {
                const int rb = r * h - r * (r - 1) / 2 - r;
                if (lane == r) acc = acc / tile[rb + r];
                const T xr = shfl(acc, r);
                if (lane > r && lane < h) acc = fma_rn(-tile[rb + lane], xr, acc);
            }
        }
    }
    __syncwarp();  // every lane has read its own place before any lane writes
    if (lane < h) {
        const int g = fr + lane;
        if (UPPER) x[pid ? g : perm[g]] = acc;
        else x[g] = acc;
    }
}

// one block-Jacobi sweep over all block rows (SOLVE_JACOBI; the stripe
// kernel of solve_U_jacobi / solve_Ut_jacobi, block_ildlt.impl.cuh:2455-2494
// and 2635-2674): x_out_I = U_II^-1 (b_I - U_I* x_in) for U (UPPER) or U'
template <class T, bool UPPER>
__global__ void __launch_bounds__(32 * kSweepWarps)
    k_sweep_jacobi(int cm, const int* __restrict__ bs, const int* __restrict__ off, const int* __restrict__ col,
                   const T* __restrict__ vals, const long long* __restrict__ piv_off,
                   const int* __restrict__ rowflags, const T* __restrict__ fval, const T* __restrict__ b,
                   const T* __restrict__ x_in, T* __restrict__ x_out)
{
    __shared__ T tiles[kSweepWarps][kTileElems];
    const int warp = threadIdx.x >> 5;
    const int I = blockIdx.x * kSweepWarps + warp;
    if (I >= cm) return;
    const int lane = lane_id();
    const int fr = bs[I], h = bs[I + 1] - fr;
    T acc = T(0);
    if (lane < h) {
        acc = b[fr + lane];
        const int e1 = off[fr + lane + 1];
        for (int k = off[fr + lane]; k < e1; ++k) acc = fma_rn(-vals[k], x_in[col[k]], acc);
    }
    if (!(rowflags[I] & kRowIdentity)) {
        T* tile = tiles[warp];
        const T* P = fval + piv_off[I];
        if (lane < h)
            for (int i = 0; i < h; ++i) tile[i * kTileStride + lane] = P[i * h + lane];
        __syncwarp();
        if (UPPER) {
            for (int c = h - 1; c >= 0; --c) {
                if (lane == c) acc = acc / tile[c * kTileStride + c];
                const T xc = shfl(acc, c);
                if (lane < c) acc = fma_rn(-tile[lane * kTileStride + c], xc, acc);
            }
        } else {
            for (int r = 0; r < h; ++r) {
                if (lane == r) acc = acc / tile[r * kTileStride + r];
                const T xr = shfl(acc, r);
                if (lane > r && lane < h) acc = fma_rn(-tile[r * kTileStride + lane], xr, acc);
            }
        }
    }
    if (lane < h) x_out[fr + lane] = acc;
}

// the Givens-form solve of one 1x1 / 2x2 pivot in C
template <class C>
__device__ __forceinline__ void givens_solve(C p11, C p12, C p22, C r1, C r2, C& g1, C& g2)
{
    const C gr = sqrt(fma_rn(p11, p11, p12 * p12));
    const C gc = p11 / gr, gs = p12 / gr;
    g1 = fma_rn(gc, r1, gs * r2);
    g2 = fma_rn(gc, r2, -(gs * r1));
    const C tp12 = fma_rn(gc, p12, gs * p22);
    const C tp22 = fma_rn(gc, p22, -(gs * p12));
    g2 = g2 / tp22;
    g1 = fma_rn(-tp12, g2, g1) / gr;
}

// k_solve_D: Givens-based 1x1 / 2x2 block-diagonal solve (out may equal in);
// an FP32 factor's ill-conditioned 2x2 pivots (wide_2x2) are solved in FP64
template <class T>
__global__ void k_solve_D(const T* __restrict__ tri, const int* __restrict__ is_piv, const T* in, T* out, int n,
                          double piv64)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const int this_piv = is_piv[g];
        const int next_piv = (g < n - 1) ? is_piv[g + 1] : 1;
        const T p11 = tri[3 * (size_t)g + 1], p12 = tri[3 * (size_t)g + 2];
        const T p22 = !next_piv ? tri[3 * (size_t)(g + 1) + 1] : T(1);
        const T r1 = in[g], r2 = (g < n - 1) ? in[g + 1] : T(0);
        T g1, g2;
        if (!next_piv && wide_2x2(p11, p12, p22, piv64)) {
            double w1, w2;
            givens_solve<double>(p11, p12, p22, r1, r2, w1, w2);
            g1 = T(w1);
            g2 = T(w2);
        } else {
            givens_solve<T>(p11, p12, p22, r1, r2, g1, g2);
        }
        if (this_piv) out[g] = g1;
        if (!next_piv) out[g + 1] = g2;
    }
}

template <class T>
__global__ void k_perm_gather(const T* __restrict__ b, T* __restrict__ x, const int* __restrict__ perm, int n)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) x[g] = b[perm[g]];
}

template <class T>
__global__ void k_perm_scatter(const T* __restrict__ b, T* __restrict__ x, const int* __restrict__ perm, int n)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) x[perm[g]] = b[g];
}


template <class T>
int build_sweeps_t(Factor* f, cudaStream_t s, int* launches)
{
    Pattern& p = *f->pat;
    const int n = p.n, cm = p.num_blocks;
    SweepBuild a;
    a.desc = p.d_desc.as<DevBlock>();
    a.bs = p.d_bs.as<int>();
    a.cs_off = p.d_cs_off.as<int>();
    a.csc_off = p.d_csc_off.as<int>();
    a.csc_blk = p.d_csc_blk.as<int>();
    a.fmt = p.d_fmt.as<int>();
    a.boff = f->boff.as<long long>();
    a.nnz = f->nnz.as<int>();
    a.idx = f->idx.as<int>();
    const T* val = f->val.as<T>();
    int* u_off = f->u_off.as<int>();
    int* ut_off = f->ut_off.as<int>();
    CULIPX_CUDA(cudaMemsetAsync(u_off, 0, (n + 1) * sizeof(int), s));
    CULIPX_CUDA(cudaMemsetAsync(ut_off, 0, (n + 1) * sizeof(int), s));
    k_count_offdiag<T><<<148 * 8, 256, 0, s>>>(a, val, p.coarse_nnz, u_off, ut_off);
    ++*launches;
    CULIPX_TRY(launch_check("k_count_offdiag"));
    CULIPX_TRY(exclusive_scan(u_off, n + 1, f->scan_tmp, p.handle, s, launches));
    CULIPX_TRY(exclusive_scan(ut_off, n + 1, f->scan_tmp, p.handle, s, launches));
    const int grid = (cm + kSweepWarps - 1) / kSweepWarps;
    k_fill_u_rows<T><<<grid, 32 * kSweepWarps, 0, s>>>(a, val, cm, u_off, f->u_col.as<int>(), f->u_val.as<T>());
    k_fill_ut_rows<T><<<grid, 32 * kSweepWarps, 0, s>>>(a, val, cm, ut_off, f->ut_col.as<int>(), f->ut_val.as<T>());
    k_pivot_offsets<<<(cm + 255) / 256, 256, 0, s>>>(cm, a.csc_off, a.csc_blk, a.boff, f->piv_off.as<long long>());
    k_pack_tiles<T><<<std::min((cm + 7) / 8, 148 * 8), 256, 0, s>>>(
        cm, a.bs, f->piv_off.as<long long>(), f->rowflags.as<int>(), val, f->pk_off.as<long long>(),
        f->pk_col.as<T>(), f->pk_row.as<T>(), f->ndmask.as<unsigned>());
    k_sweep_extras<T><<<148 * 4, 256, 0, s>>>(u_off, f->u_col.as<int>(), f->perm.as<int>(), f->u_colp.as<int>(), n,
                                              f->tri.as<T>(), f->dg.as<T>());
    const int* lvl_rows = p.d_lvl_rows.as<int>();
    const int* rowflags = f->rowflags.as<int>();
    k_split_count<<<std::min(cm / 256 + 1, 148 * 4), 256, 0, s>>>(cm, lvl_rows, a.bs, rowflags, f->scan_s.as<int>(),
                                                                  f->scan_c.as<int>());
    *launches += 6;
    CULIPX_TRY(exclusive_scan(f->scan_s.as<int>(), cm + 1, f->scan_tmp, p.handle, s, launches));
    CULIPX_TRY(exclusive_scan(f->scan_c.as<int>(), cm + 1, f->scan_tmp, p.handle, s, launches));
    k_split_fill<<<std::min(cm / 256 + 1, 148 * 4), 256, 0, s>>>(cm, lvl_rows, a.bs, rowflags, f->scan_s.as<int>(),
                                                                 f->scan_c.as<int>(), f->simple_rows.as<int>(),
                                                                 f->cplx.as<int>(), f->pk_off.as<long long>(),
                                                                 f->ndmask.as<unsigned>(), f->citem.as<CItem>());
    *launches += 1;
    return launch_check("build_sweeps");
}

template <class T>
int apply_t(Factor* f, int stage, const void* d_b, void* d_x, cudaStream_t s)
{
    Pattern& p = *f->pat;
    const int n = p.n;
    const T* b = static_cast<const T*>(d_b);
    T* x = static_cast<T*>(d_x);
    const int grid_n = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
    if (stage == CULIPX_MIDDLE) {
        k_solve_D<T><<<grid_n, 256, 0, s>>>(f->tri.as<T>(), f->is_piv.as<int>(), b, x, n, f->pivot_fp64);
        return launch_check("k_solve_D");
    }
    const T* fval = f->val.as<T>();
    if (f->solve_algorithm == CULIPX_SOLVE_JACOBI) {
        // x = 0, then `sweeps` block-Jacobi sweeps on the right-hand side rhs
        if (!f->jac_a.get()) CULIPX_TRY(f->jac_a.alloc(p.handle, (size_t)n * sizeof(T) + 16));
        if (!f->jac_b.get()) CULIPX_TRY(f->jac_b.alloc(p.handle, (size_t)n * sizeof(T) + 16));
        const int cm = p.num_blocks;
        const bool left = stage == CULIPX_LEFT;
        T* rhs = f->work.as<T>();
        if (left) k_perm_gather<T><<<grid_n, 256, 0, s>>>(b, rhs, f->perm.as<int>(), n);
        else CULIPX_CUDA(cudaMemcpyAsync(rhs, b, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
        T* xa = f->jac_a.as<T>();
        T* xb = f->jac_b.as<T>();
        CULIPX_CUDA(cudaMemsetAsync(xa, 0, n * sizeof(T), s));
        const int grid = (cm + kSweepWarps - 1) / kSweepWarps;
        for (int sw = 0; sw < f->jacobi_sweeps; ++sw) {
            if (left)
                k_sweep_jacobi<T, false><<<grid, 32 * kSweepWarps, 0, s>>>(
                    cm, p.d_bs.as<int>(), f->ut_off.as<int>(), f->ut_col.as<int>(), f->ut_val.as<T>(),
                    f->piv_off.as<long long>(), f->rowflags.as<int>(), fval, rhs, xa, xb);
            else
                k_sweep_jacobi<T, true><<<grid, 32 * kSweepWarps, 0, s>>>(
                    cm, p.d_bs.as<int>(), f->u_off.as<int>(), f->u_col.as<int>(), f->u_val.as<T>(),
                    f->piv_off.as<long long>(), f->rowflags.as<int>(), fval, rhs, xa, xb);
            std::swap(xa, xb);
        }
        if (left) CULIPX_CUDA(cudaMemcpyAsync(x, xa, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
        else k_perm_scatter<T><<<grid_n, 256, 0, s>>>(xa, x, f->perm.as<int>(), n);
        return launch_check("Jacobi sweeps");
    }
    if (stage == CULIPX_LEFT) {
        const T* src = b;
        if ((const void*)b == (void*)x) {
            // in place: P' b into x first, the sweeps then start from x
            T* t = f->work.as<T>();
            CULIPX_CUDA(cudaMemcpyAsync(t, b, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
            k_perm_gather<T><<<grid_n, 256, 0, s>>>(t, x, f->perm.as<int>(), n);
            src = nullptr;
        }
        for (int L = 0; L < p.num_levels; ++L) {
            const int nr = p.lvl_off[L + 1] - p.lvl_off[L];
            k_sweep_level<T, false><<<(nr + kSweepWarps - 1) / kSweepWarps, 32 * kSweepWarps, 0, s>>>(
                p.d_lvl_rows.as<int>() + p.lvl_off[L], nr, p.d_bs.as<int>(), f->ut_off.as<int>(),
                f->ut_col.as<int>(), f->ut_val.as<T>(), f->pk_off.as<long long>(), f->rowflags.as<int>(),
                f->pk_row.as<T>(), f->perm.as<int>(), src, x);
        }
        return launch_check("U' sweep");
    }
    // RIGHT: x = P U^-1 b, the permutation folded into the sweeps
    for (int L = p.num_levels - 1; L >= 0; --L) {
        const int nr = p.lvl_off[L + 1] - p.lvl_off[L];
        k_sweep_level<T, true><<<(nr + kSweepWarps - 1) / kSweepWarps, 32 * kSweepWarps, 0, s>>>(
            p.d_lvl_rows.as<int>() + p.lvl_off[L], nr, p.d_bs.as<int>(), f->u_off.as<int>(), f->u_colp.as<int>(),
            f->u_val.as<T>(), f->pk_off.as<long long>(), f->rowflags.as<int>(), f->pk_col.as<T>(),
            f->perm.as<int>(), b, x);
    }
    return launch_check("U sweep");
}

}  // namespace

// exclusive scan of n int counts in place (n - 1 counts and a trailing 0 give
// the offsets and the total), three launches
int exclusive_scan(int* d, int n, DeviceBuffer& tmp, culipx_handle_t* h, cudaStream_t s, int* launches)
{
    const int chunks = (n + kScanChunk - 1) / kScanChunk;
    if ((size_t)chunks * sizeof(int) > tmp.bytes()) CULIPX_TRY(tmp.alloc(h, (size_t)chunks * sizeof(int)));
    k_scan_chunks<<<chunks, kScanThreads, 0, s>>>(d, n, tmp.as<int>());
    k_scan_sums<<<1, 1024, 0, s>>>(tmp.as<int>(), chunks);
    k_scan_add<<<chunks, kScanThreads, 0, s>>>(d, n, tmp.as<int>());
    *launches += 3;
    return launch_check("exclusive_scan");
}

int build_sweeps(Factor* f, cudaStream_t s, int* launches)
{
    if (f->precision == CULIPX_F64) return build_sweeps_t<double>(f, s, launches);
    return build_sweeps_t<float>(f, s, launches);
}

int prec_apply(Factor* f, int stage, const void* d_b, void* d_x, cudaStream_t s)
{
    if (!f || !f->computed) return fail(CULIPX_INVALID_ARG, "culipx_prec_apply: factor not computed");
    if (!d_b || !d_x) return fail(CULIPX_INVALID_ARG, "culipx_prec_apply: null vector");
    if (stage < CULIPX_LEFT || stage > CULIPX_RIGHT) return fail(CULIPX_INVALID_ARG, "culipx_prec_apply: bad stage");
    Pattern& p = *f->pat;
    if (stage == CULIPX_MIDDLE) p.handle->launches += 1;
    else if (f->solve_algorithm == CULIPX_SOLVE_JACOBI) p.handle->launches += f->jacobi_sweeps + 1 + (stage == CULIPX_LEFT);
    else p.handle->launches += p.num_levels + ((stage == CULIPX_LEFT && d_b == d_x) ? 1 : 0);
    if (f->precision == CULIPX_F64) return apply_t<double>(f, stage, d_b, d_x, s);
    return apply_t<float>(f, stage, d_b, d_x, s);
}

}  // namespace culipx
