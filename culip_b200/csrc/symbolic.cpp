// Symbolic analysis of a KKT sparsity pattern for the block-iLDL^T factor.
//
// Produces the same canonical output as the reference's host phase
// (libs/la/preconditioner/block_ildlt.impl.cuh):
//   coarse upper pattern           build_initial_coarse            :352-484
//   level-of-fill + diagonals      determine_coarse_level_fill..   :492-728
//   block CSC                      build_block_csc                 :732-762
//   row level sets, block order    find_level_sets                 :766-1011
//   formats, max_nnz, storage      build_blocks                    :1015-1280
//   U' sweep order                 solve_analysis_block            :2050-2150
// with different algorithms: per-row marker sets instead of global sorts, a
// longest-path pass over the block CSC for the levels (the level of block row
// c is 1 + the largest level of any row k < c with a block (k, c)), epoch-
// stamped visit arrays for the fill BFS, and counting sorts.  Rows inside a
// level are ascending (the reference's order there comes from OpenMP atomics).
#include "pattern.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include <omp.h>

namespace culipx {

namespace {

int blk_size(const Pattern& p, int b) { return p.bs[b + 1] - p.bs[b]; }

// Coarse upper-triangular pattern with per-block counts of A's entries.
void coarse_pattern(Pattern& p, const int* rowptr, const int* colidx)
{
    const int cm = p.num_blocks;
    std::vector<std::vector<int>> rows_col(cm), rows_cnt(cm);
#pragma omp parallel
    {
        std::vector<int> cnt(cm, 0), touched;
        touched.reserve(256);
#pragma omp for schedule(dynamic, 64)
        for (int I = 0; I < cm; ++I) {
            touched.clear();
            for (int i = p.bs[I]; i < p.bs[I + 1]; ++i)
                for (int q = rowptr[i]; q < rowptr[i + 1]; ++q) {
                    const int c = colidx[q];
                    if (c < i) continue;
                    const int bc = p.row_block[c];
                    if (cnt[bc]++ == 0) touched.push_back(bc);
                }
            std::sort(touched.begin(), touched.end());
            rows_col[I].resize(touched.size());
            rows_cnt[I].resize(touched.size());
            for (size_t t = 0; t < touched.size(); ++t) {
                rows_col[I][t] = touched[t];
                rows_cnt[I][t] = cnt[touched[t]];
                cnt[touched[t]] = 0;
            }
        }
    }
    // level-of-fill and missing diagonals
    std::vector<std::vector<int>> fill(cm);
    const int max_level = p.fill_level;
#pragma omp parallel
    {
        std::vector<int> stamp(cm, -1), length(cm, 0), queue;
        queue.reserve(1024);
#pragma omp for schedule(dynamic, 16)
        for (int i = 0; i < cm; ++i) {
            if (max_level > 0) {
                queue.clear();
                queue.push_back(i);
                length[i] = 0;
                stamp[i] = i;
                for (size_t qh = 0; qh < queue.size(); ++qh) {
                    const int cur = queue[qh];
                    for (int j = p.bs[cur]; j < p.bs[cur + 1]; ++j)
                        for (int q = rowptr[j]; q < rowptr[j + 1]; ++q) {
                            const int kc = p.row_block[colidx[q]];
                            if (stamp[kc] == i) continue;
                            stamp[kc] = i;
                            if (kc < i && length[cur] < max_level) {
                                queue.push_back(kc);
                                length[kc] = length[cur] + 1;
                            }
                            if (kc > i && length[cur] > 0) fill[i].push_back(kc);
                        }
                }
            }
            // the reference inspects only the first block of the row
            const bool has_diag = !rows_col[i].empty() && rows_col[i][0] == i;
            if (!has_diag) fill[i].push_back(i);
            std::sort(fill[i].begin(), fill[i].end());
        }
    }
    p.cs_off.assign(cm + 1, 0);
    for (int I = 0; I < cm; ++I) p.cs_off[I + 1] = p.cs_off[I] + (int)(rows_col[I].size() + fill[I].size());
    p.coarse_nnz = p.cs_off[cm];
    p.fill_nnz = 0;
    for (int I = 0; I < cm; ++I) p.fill_nnz += (int)fill[I].size();
    p.cs_col.resize(p.coarse_nnz);
    p.blk_nnzA.resize(p.coarse_nnz);
#pragma omp parallel for schedule(static)
    for (int I = 0; I < cm; ++I) {
        // merge two sorted lists
        size_t a = 0, b = 0;
        int o = p.cs_off[I];
        const auto& rc = rows_col[I];
        const auto& fl = fill[I];
        while (a < rc.size() || b < fl.size()) {
            if (b >= fl.size() || (a < rc.size() && rc[a] < fl[b])) {
                p.cs_col[o] = rc[a];
                p.blk_nnzA[o] = rows_cnt[I][a];
                ++a;
            } else {
                p.cs_col[o] = fl[b];
                p.blk_nnzA[o] = 0;
                ++b;
            }
            ++o;
        }
    }
}

}  // namespace

int analyze_pattern(culipx_handle_t* h, int n, const int* rowptr, const int* colidx,
                    int num_blocks, const int* block_starts, int fill_level, double fill_factor,
                    int precision, Pattern** out, int num_systems, const int* system_row_offsets)
{
    if (!out || !rowptr || !colidx || !block_starts || n <= 0 || num_blocks <= 0 || num_blocks > n)
        return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze: bad arguments");
    if (fill_level < 0) return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze: fill_level < 0");
    if (!(fill_factor >= 1.0))
        return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze: fill_factor must be >= 1 (the driver clamps it, block_ildlt.cc:50)");
    if (precision != CULIPX_F64 && precision != CULIPX_F32)
        return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze: bad precision");
    if (rowptr[0] != 0) return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze: rowptr[0] != 0");

    auto* pp = new culipx_pattern_t();
    Pattern& p = *pp;
    p.handle = h;
    p.n = n;
    p.nnz = rowptr[n];
    p.precision = precision;
    p.fill_level = fill_level;
    p.fill_factor = fill_factor;
    p.num_blocks = num_blocks;
    const int cm = num_blocks;

    p.bs.assign(block_starts, block_starts + cm);
    p.bs.push_back(n);
    for (int b = 0; b < cm; ++b) {
        const int sz = p.bs[b + 1] - p.bs[b];
        if (sz < 1 || sz > 32) {
            delete pp;
            return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze: block %d has size %d (must be 1..32)", b, sz);
        }
    }
    if (p.bs[0] != 0) { delete pp; return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze: block_starts[0] != 0"); }
    // systems of a block-diagonal union (default: one system): per block row
    // its system's first block row and block count, for the format rule
    std::vector<int> sys_first(cm, 0), sys_blocks(cm, cm);
    if (num_systems > 1 && system_row_offsets) {
        if (system_row_offsets[0] != 0 || system_row_offsets[num_systems] != n) {
            delete pp;
            return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze_systems: row offsets must run from 0 to n");
        }
        int b0 = 0;
        for (int k = 0; k < num_systems; ++k) {
            int b1 = b0;
            while (b1 < cm && p.bs[b1] < system_row_offsets[k + 1]) ++b1;
            if (p.bs[b0] != system_row_offsets[k] || p.bs[b1] != system_row_offsets[k + 1] || b1 == b0) {
                delete pp;
                return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze_systems: system %d does not start and end on block boundaries", k);
            }
            for (int I = b0; I < b1; ++I) {
                sys_first[I] = b0;
                sys_blocks[I] = b1 - b0;
            }
            b0 = b1;
        }
    }
    for (int i = 0; i < n; ++i)
        for (int q = rowptr[i]; q < rowptr[i + 1]; ++q)
            if (colidx[q] < 0 || colidx[q] >= n || (q > rowptr[i] && colidx[q] <= colidx[q - 1])) {
                delete pp;
                return fail(CULIPX_INVALID_ARG, "culipx_pattern_analyze: row %d: columns must be sorted, unique, in range", i);
            }
    p.row_block.resize(n);
    for (int b = 0; b < cm; ++b)
        for (int j = p.bs[b]; j < p.bs[b + 1]; ++j) p.row_block[j] = b;

    coarse_pattern(p, rowptr, colidx);
    const int cnz = p.coarse_nnz;
    p.blk_row.resize(cnz);
    p.blk_col.resize(cnz);
    for (int I = 0; I < cm; ++I)
        for (int q = p.cs_off[I]; q < p.cs_off[I + 1]; ++q) { p.blk_row[q] = I; p.blk_col[q] = p.cs_col[q]; }

    // block CSC by counting sort (rows ascend within a column)
    p.csc_off.assign(cm + 1, 0);
    for (int q = 0; q < cnz; ++q) p.csc_off[p.cs_col[q] + 1]++;
    for (int c = 0; c < cm; ++c) p.csc_off[c + 1] += p.csc_off[c];
    p.csc_blk.resize(cnz);
    {
        std::vector<int> pos(p.csc_off.begin(), p.csc_off.end() - 1);
        for (int q = 0; q < cnz; ++q) p.csc_blk[pos[p.cs_col[q]]++] = q;
    }

    // levels: longest path over the upper block pattern
    p.row_level.assign(cm, 0);
    for (int c = 0; c < cm; ++c) {
        int lv = 0;
        for (int q = p.csc_off[c]; q < p.csc_off[c + 1]; ++q) {
            const int k = p.blk_row[p.csc_blk[q]];
            if (k != c) lv = std::max(lv, p.row_level[k] + 1);
        }
        p.row_level[c] = lv;
    }
    p.num_levels = 0;
    for (int c = 0; c < cm; ++c) p.num_levels = std::max(p.num_levels, p.row_level[c] + 1);
    p.l0_diagonal = true;
    for (int c = 0; c < cm && p.l0_diagonal; ++c) {
        if (p.row_level[c] != 0) continue;
        for (int i = p.bs[c]; i < p.bs[c + 1]; ++i)
            for (int q = rowptr[i]; q < rowptr[i + 1]; ++q)
                if (colidx[q] != i && p.row_block[colidx[q]] == c) p.l0_diagonal = false;
    }
    const int nl = p.num_levels;
    p.lvl_off.assign(nl + 1, 0);
    for (int c = 0; c < cm; ++c) p.lvl_off[p.row_level[c] + 1]++;
    for (int L = 0; L < nl; ++L) p.lvl_off[L + 1] += p.lvl_off[L];
    p.lvl_rows.resize(cm);
    {
        std::vector<int> pos(p.lvl_off.begin(), p.lvl_off.end() - 1);
        for (int c = 0; c < cm; ++c) p.lvl_rows[pos[p.row_level[c]]++] = c;  // ascending
    }

    // factor order per level: pivots (row order) then off-diagonal blocks (block-id order)
    p.lb_off.assign(nl + 1, 0);
    p.lb.resize(cnz);
    p.max_level_blocks = 0;
    p.max_level_rows = 0;
    {
        int o = 0;
        for (int L = 0; L < nl; ++L) {
            p.lb_off[L] = o;
            for (int t = p.lvl_off[L]; t < p.lvl_off[L + 1]; ++t) p.lb[o++] = p.cs_off[p.lvl_rows[t]];  // diagonal is first
            for (int t = p.lvl_off[L]; t < p.lvl_off[L + 1]; ++t) {
                const int r = p.lvl_rows[t];
                for (int q = p.cs_off[r] + 1; q < p.cs_off[r + 1]; ++q) p.lb[o++] = q;
            }
            p.max_level_blocks = std::max(p.max_level_blocks, o - p.lb_off[L]);
            p.max_level_rows = std::max(p.max_level_rows, p.lvl_off[L + 1] - p.lvl_off[L]);
        }
        p.lb_off[nl] = o;
        p.row_offdiag_start.resize(cm);
        for (int L = 0; L < nl; ++L) {
            int s = 0;
            for (int t = p.lvl_off[L]; t < p.lvl_off[L + 1]; ++t) {
                p.row_offdiag_start[t] = s;
                s += p.cs_off[p.lvl_rows[t] + 1] - p.cs_off[p.lvl_rows[t]] - 1;
            }
        }
    }
    // U' sweep order: per column level, pivots then off-diagonal blocks (block-id order)
    p.sb_off.assign(nl + 1, 0);
    p.sb.resize(cnz);
    {
        int o = 0;
        for (int L = 0; L < nl; ++L) {
            p.sb_off[L] = o;
            for (int t = p.lvl_off[L]; t < p.lvl_off[L + 1]; ++t) p.sb[o++] = p.cs_off[p.lvl_rows[t]];
            const int o0 = o;
            for (int t = p.lvl_off[L]; t < p.lvl_off[L + 1]; ++t) {
                const int c = p.lvl_rows[t];
                for (int q = p.csc_off[c]; q < p.csc_off[c + 1] - 1; ++q) p.sb[o++] = p.csc_blk[q];
            }
            std::sort(p.sb.begin() + o0, p.sb.begin() + o);
        }
        p.sb_off[nl] = o;
    }

    // formats and max_nnz
    p.fmt.resize(cnz);
    p.max_nnz.resize(cnz);
    const bool dbl = (precision == CULIPX_F64);
    for (int I = 0; I < cm; ++I) {
        int sum_nnz = 0, sum_blocks = 0;
        for (int q = p.cs_off[I]; q < p.cs_off[I + 1]; ++q) {
            sum_nnz += p.blk_nnzA[q];
            sum_blocks += (p.blk_nnzA[q] != 0);
        }
        // a block row without any A entry has no defined average in the
        // reference (0/0); such rows get 0 here
        const int avg = (sum_blocks == 0) ? 0
                        : dbl ? (int)std::ceil((double)sum_nnz / (double)sum_blocks)
                              : (int)std::ceil((float)sum_nnz / (float)sum_blocks);
        const int r = blk_size(p, I);
        for (int q = p.cs_off[I]; q < p.cs_off[I + 1]; ++q) {
            const int J = p.cs_col[q];
            const int c = blk_size(p, J);
            const int src = p.blk_nnzA[q] ? p.blk_nnzA[q] : avg;
            const int cap = dbl ? (int)std::ceil(fill_factor * (double)src)
                                : (int)std::ceil((float)fill_factor * (float)src);
            const int mx = std::min(r * c, cap);
            p.max_nnz[q] = mx;
            const size_t vb = dbl ? 8 : 4;
            const double lhs = (double)((4 + vb) * (size_t)(long long)mx);
            const double rhs = dbl ? 0.5 * 8.0 * (double)r * (double)c : (double)(0.5f * 4.0f * (float)r * (float)c);
            // the last 10 % of a system's block rows keep dense blocks
            const bool sparse = (I != J) && ((double)(I - sys_first[I]) < 0.9 * (double)sys_blocks[I]) && (lhs < rhs);
            p.fmt[q] = sparse ? kSparse : kDense;
            if (sparse) ++p.num_sparse; else ++p.num_dense;
        }
    }

    // value-store layout in factor order
    p.desc.resize(cnz);
    {
        long long o = 0;
        for (int t = 0; t < cnz; ++t) {
            const int q = p.lb[t];
            const int r = blk_size(p, p.blk_row[q]), c = blk_size(p, p.blk_col[q]);
            BlockDesc& d = p.desc[q];
            d.row = p.blk_row[q];
            d.col = p.blk_col[q];
            d.cap = (p.fmt[q] == kDense) ? r * c : std::max(p.max_nnz[q], p.blk_nnzA[q]);
            d.val_off = (int)o;
            o += d.cap;
            if (p.fmt[q] == kSparse) p.sparse_slots += d.cap;
            if (o > 0x7fffffffLL) { delete pp; return fail(CULIPX_NOT_SUPPORTED, "culipx_pattern_analyze: factor storage exceeds 2^31 slots"); }
        }
        p.val_slots = o;
    }

    // gather destinations of A's upper entries
    p.a_dst.assign(p.nnz, -1);
    p.idx_init.assign(p.val_slots, -1);
    p.nnz_init.assign(cnz, 0);
    for (int i = 0; i < n; ++i) {
        const int I = p.row_block[i];
        const int* cb = p.cs_col.data() + p.cs_off[I];
        const int clen = p.cs_off[I + 1] - p.cs_off[I];
        for (int q = rowptr[i]; q < rowptr[i + 1]; ++q) {
            const int c = colidx[q];
            if (c < i) continue;
            const int J = p.row_block[c];
            const int pos = (int)(std::lower_bound(cb, cb + clen, J) - cb);
            const int b = p.cs_off[I] + pos;
            const int w = blk_size(p, J);
            const int local = (i - p.bs[I]) * w + (c - p.bs[J]);
            const BlockDesc& d = p.desc[b];
            if (p.fmt[b] == kDense) {
                p.a_dst[q] = d.val_off + local;
            } else {
                const int slot = d.val_off + p.nnz_init[b]++;
                p.a_dst[q] = slot;
                p.idx_init[slot] = local;
            }
        }
    }

    // device mirror (not for a host-only handle)
    if (h->device < 0) {
        *out = pp;
        return CULIPX_OK;
    }
    int st = CULIPX_OK;
    auto up = [&](DeviceBuffer& buf, const void* src, size_t bytes) {
        if (st == CULIPX_OK) st = buf.upload(h, src, bytes);
    };
    up(p.d_cs_off, p.cs_off.data(), sizeof(int) * (cm + 1));
    up(p.d_row_offdiag_start, p.row_offdiag_start.data(), sizeof(int) * cm);
    up(p.d_lvl_off, p.lvl_off.data(), sizeof(int) * (p.num_levels + 1));
    up(p.d_desc, p.desc.data(), sizeof(BlockDesc) * cnz);
    up(p.d_bs, p.bs.data(), sizeof(int) * (cm + 1));
    up(p.d_csc_off, p.csc_off.data(), sizeof(int) * (cm + 1));
    up(p.d_csc_blk, p.csc_blk.data(), sizeof(int) * cnz);
    up(p.d_lb, p.lb.data(), sizeof(int) * cnz);
    up(p.d_lvl_rows, p.lvl_rows.data(), sizeof(int) * cm);
    up(p.d_a_dst, p.a_dst.data(), sizeof(int) * p.nnz);
    up(p.d_idx_init, p.idx_init.data(), sizeof(int) * p.val_slots);
    up(p.d_nnz_init, p.nnz_init.data(), sizeof(int) * cnz);
    up(p.d_fmt, p.fmt.data(), sizeof(int) * cnz);
    up(p.d_maxnnz, p.max_nnz.data(), sizeof(int) * cnz);
    up(p.d_row_block, p.row_block.data(), sizeof(int) * n);
    if (st != CULIPX_OK) { delete pp; return st; }
    p.device_bytes = (long long)(p.d_cs_off.bytes() + p.d_desc.bytes() + p.d_bs.bytes() + p.d_csc_off.bytes() + p.d_csc_blk.bytes() +
                                 p.d_lb.bytes() + p.d_lvl_rows.bytes() + p.d_a_dst.bytes() + p.d_idx_init.bytes() +
                                 p.d_nnz_init.bytes() + p.d_fmt.bytes() + p.d_maxnnz.bytes() + p.d_row_block.bytes());
    *out = pp;
    return CULIPX_OK;
}

}  // namespace culipx
