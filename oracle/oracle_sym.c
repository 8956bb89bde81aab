/*
 * oracle_sym.c -- CPU restatement of culip's block-iLDL^T symbolic phase.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the product's
 * symbolic analysis (culip_b200/csrc/symbolic.cpp); only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The
 * product library never links or calls it.
 *
 * Every function restates the reference function it cites (paths relative to
 * the culip repository):
 *   build_initial_coarse            libs/la/preconditioner/block_ildlt.impl.cuh:352-484
 *   determine_coarse_level_fill...  libs/la/preconditioner/block_ildlt.impl.cuh:492-728
 *   build_block_csc                 libs/la/preconditioner/block_ildlt.impl.cuh:732-762
 *   find_level_sets                 libs/la/preconditioner/block_ildlt.impl.cuh:766-1011
 *   build_blocks                    libs/la/preconditioner/block_ildlt.impl.cuh:1015-1280
 *   solve_analysis_block            libs/la/preconditioner/block_ildlt.impl.cuh:2050-2150
 *
 * The reference's host sorts use thrust's sequential (stable) backend, so the
 * per-level block lists are deterministic: pivot block first in row order,
 * then off-diagonal blocks in block-CSR order.  The only non-deterministic
 * output of the reference is the order of rows inside one level
 * (OpenMP atomic capture, block_ildlt.impl.cuh:841-856); this restatement
 * returns each level's rows sorted ascending (the canonical form).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static void *xmalloc(size_t n)
{
    void *p = malloc(n ? n : 1);
    if (!p) abort();
    return p;
}

static int cmp_int(const void *a, const void *b)
{
    const int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

void orc_sym_free(orc_sym *s)
{
    if (!s) return;
    free(s->bs); free(s->row_block);
    free(s->cs_off); free(s->cs_col); free(s->blk_nnzA);
    free(s->csc_off); free(s->csc_blk);
    free(s->lvl_off); free(s->lvl_rows); free(s->row_level);
    free(s->lb_off); free(s->lb);
    free(s->sb_off); free(s->sb);
    free(s->blk_row); free(s->blk_col); free(s->fmt); free(s->max_nnz);
    free(s->a_blk); free(s->a_idx);
    free(s);
}

/*
 * Coarse upper pattern: every entry (i, c) of the full symmetric CSR with
 * c >= i maps to block (rb[i], rb[c]); blocks are counted and emitted sorted
 * by (block row, block col).  Mirrors the remove_if / sort / reduce_by_key
 * chain of build_initial_coarse (block_ildlt.impl.cuh:380-483).
 */
static void build_initial_coarse(orc_sym *s, const int *rowptr, const int *colidx,
                                 int **out_off, int **out_col, int **out_cnt, int *out_nnz)
{
    const int cm = s->num_blocks;
    int *cnt = (int *)xmalloc(sizeof(int) * cm);
    int *touched = (int *)xmalloc(sizeof(int) * cm);
    memset(cnt, 0, sizeof(int) * cm);

    /* first pass: count coarse entries per block row */
    int *row_n = (int *)xmalloc(sizeof(int) * (cm + 1));
    long total = 0;
    for (int I = 0; I < cm; ++I) {
        int nt = 0;
        for (int i = s->bs[I]; i < s->bs[I + 1]; ++i)
            for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) {
                const int c = colidx[p];
                if (c < i) continue;
                const int bc = s->row_block[c];
                if (cnt[bc]++ == 0) touched[nt++] = bc;
            }
        row_n[I] = nt;
        total += nt;
        for (int t = 0; t < nt; ++t) cnt[touched[t]] = 0;
    }
    int *off = (int *)xmalloc(sizeof(int) * (cm + 1));
    off[0] = 0;
    for (int I = 0; I < cm; ++I) off[I + 1] = off[I] + row_n[I];
    int *col = (int *)xmalloc(sizeof(int) * (total ? total : 1));
    int *bn = (int *)xmalloc(sizeof(int) * (total ? total : 1));

    /* second pass: emit sorted columns with their counts */
    for (int I = 0; I < cm; ++I) {
        int nt = 0;
        for (int i = s->bs[I]; i < s->bs[I + 1]; ++i)
            for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) {
                const int c = colidx[p];
                if (c < i) continue;
                const int bc = s->row_block[c];
                if (cnt[bc]++ == 0) touched[nt++] = bc;
            }
        qsort(touched, nt, sizeof(int), cmp_int);
        for (int t = 0; t < nt; ++t) {
            col[off[I] + t] = touched[t];
            bn[off[I] + t] = cnt[touched[t]];
            cnt[touched[t]] = 0;
        }
    }
    free(cnt); free(touched); free(row_n);
    *out_off = off; *out_col = col; *out_cnt = bn; *out_nnz = (int)total;
}

/*
 * Level-of-fill on the coarse graph by a bounded BFS over the fine graph
 * (Hysom-Pothen), plus missing diagonal blocks.  Restates
 * determine_coarse_level_fill_and_diag (block_ildlt.impl.cuh:492-728): a
 * block k > i is fill iff it is first discovered from a node whose BFS length
 * is > 0; only blocks k < i are expanded, and only while length < max_level.
 * The diagonal test looks at the first entry of row i only (:560-567).
 * The result is the (row, col)-sorted union, as after the sort at :713-722.
 */
static void level_fill_and_diag(orc_sym *s, const int *rowptr, const int *colidx, int max_level,
                                int **p_off, int **p_col, int **p_cnt, int *p_nnz)
{
    const int cm = s->num_blocks;
    int *off = *p_off, *col = *p_col, *cnt = *p_cnt;
    const int nnz0 = *p_nnz;

    int *stamp = (int *)xmalloc(sizeof(int) * cm);
    int *length = (int *)xmalloc(sizeof(int) * cm);
    int *queue = (int *)xmalloc(sizeof(int) * cm);
    for (int i = 0; i < cm; ++i) stamp[i] = -1;

    int *fill_n = (int *)xmalloc(sizeof(int) * (cm + 1));
    int **fill_lists = (int **)xmalloc(sizeof(int *) * cm);
    long new_total = 0;

    for (int i = 0; i < cm; ++i) {
        int qh = 0, qt = 0, nf = 0, capf = 8;
        int *fl = (int *)xmalloc(sizeof(int) * capf);
        queue[qt++] = i;
        length[i] = 0;
        stamp[i] = i;
        while (qh < qt) {
            const int cur = queue[qh++];
            for (int j = s->bs[cur]; j < s->bs[cur + 1]; ++j)
                for (int p = rowptr[j]; p < rowptr[j + 1]; ++p) {
                    const int kc = s->row_block[colidx[p]];
                    if (stamp[kc] == i) continue;
                    stamp[kc] = i;
                    if (kc < i && length[cur] < max_level) {
                        queue[qt++] = kc;
                        length[kc] = length[cur] + 1;
                    }
                    if (kc > i && length[cur] > 0) {
                        if (nf == capf) { capf *= 2; fl = (int *)realloc(fl, sizeof(int) * capf); }
                        fl[nf++] = kc;
                    }
                }
        }
        /* diagonal check on the first entry of the row (reference :562-564) */
        const int has_diag = (off[i] < nnz0) && (col[off[i]] == i);
        if (!has_diag) {
            if (nf == capf) { capf *= 2; fl = (int *)realloc(fl, sizeof(int) * capf); }
            fl[nf++] = i;
        }
        fill_n[i] = nf;
        fill_lists[i] = fl;
        new_total += nf;
    }
    s->fill_nnz = (int)new_total;

    if (new_total > 0) {
        const long tot = nnz0 + new_total;
        int *noff = (int *)xmalloc(sizeof(int) * (cm + 1));
        int *ncol = (int *)xmalloc(sizeof(int) * tot);
        int *ncnt = (int *)xmalloc(sizeof(int) * tot);
        noff[0] = 0;
        for (int i = 0; i < cm; ++i) {
            /* merge the sorted original row with the sorted fill list */
            int *fl = fill_lists[i];
            qsort(fl, fill_n[i], sizeof(int), cmp_int);
            int a = off[i], ae = off[i + 1], b = 0, be = fill_n[i], o = noff[i];
            while (a < ae || b < be) {
                if (b >= be || (a < ae && col[a] < fl[b])) { ncol[o] = col[a]; ncnt[o] = cnt[a]; ++a; }
                else { ncol[o] = fl[b]; ncnt[o] = 0; ++b; }
                ++o;
            }
            noff[i + 1] = o;
        }
        free(off); free(col); free(cnt);
        *p_off = noff; *p_col = ncol; *p_cnt = ncnt; *p_nnz = (int)tot;
    }
    for (int i = 0; i < cm; ++i) free(fill_lists[i]);
    free(fill_lists); free(fill_n); free(stamp); free(length); free(queue);
}

orc_sym *orc_symbolic(int n, const int *rowptr, const int *colidx,
                      int num_blocks, const int *block_starts,
                      int fill_level, double fill_factor, int value_bytes)
{
    orc_sym *s = (orc_sym *)xmalloc(sizeof(orc_sym));
    memset(s, 0, sizeof(*s));
    s->n = n;
    s->nnz = rowptr[n];
    s->num_blocks = num_blocks;
    s->value_bytes = value_bytes;
    const int cm = num_blocks;

    s->bs = (int *)xmalloc(sizeof(int) * (cm + 1));
    memcpy(s->bs, block_starts, sizeof(int) * cm);
    s->bs[cm] = n; /* the constructor appends h_A->m (block_ildlt.impl.cuh:72-76) */
    s->row_block = (int *)xmalloc(sizeof(int) * (n ? n : 1));
    for (int I = 0; I < cm; ++I)
        for (int j = s->bs[I]; j < s->bs[I + 1]; ++j) s->row_block[j] = I;

    int *off, *col, *cnt, cnnz;
    build_initial_coarse(s, rowptr, colidx, &off, &col, &cnt, &cnnz);
    level_fill_and_diag(s, rowptr, colidx, fill_level, &off, &col, &cnt, &cnnz);
    s->cs_off = off; s->cs_col = col; s->blk_nnzA = cnt; s->coarse_nnz = cnnz;
    const int cnz = cnnz;

    s->blk_row = (int *)xmalloc(sizeof(int) * cnz);
    s->blk_col = (int *)xmalloc(sizeof(int) * cnz);
    for (int I = 0; I < cm; ++I)
        for (int p = off[I]; p < off[I + 1]; ++p) { s->blk_row[p] = I; s->blk_col[p] = col[p]; }

    /* block CSC (build_block_csc :732-762, with block ids as in :1268-1279) */
    s->csc_off = (int *)xmalloc(sizeof(int) * (cm + 1));
    s->csc_blk = (int *)xmalloc(sizeof(int) * cnz);
    memset(s->csc_off, 0, sizeof(int) * (cm + 1));
    for (int p = 0; p < cnz; ++p) s->csc_off[col[p] + 1]++;
    for (int c = 0; c < cm; ++c) s->csc_off[c + 1] += s->csc_off[c];
    {
        int *fillp = (int *)xmalloc(sizeof(int) * cm);
        memcpy(fillp, s->csc_off, sizeof(int) * cm);
        for (int p = 0; p < cnz; ++p) s->csc_blk[fillp[col[p]]++] = p; /* rows ascend */
        free(fillp);
    }

    /* level sets (find_level_sets :766-878) */
    int *dep = (int *)xmalloc(sizeof(int) * cm);
    for (int c = 0; c < cm; ++c) dep[c] = s->csc_off[c + 1] - s->csc_off[c];
    s->lvl_rows = (int *)xmalloc(sizeof(int) * (cm ? cm : 1));
    s->lvl_off = (int *)xmalloc(sizeof(int) * (cm + 2));
    s->row_level = (int *)xmalloc(sizeof(int) * (cm ? cm : 1));
    int nl = 0, wr = 0;
    s->lvl_off[0] = 0;
    for (int c = 0; c < cm; ++c)
        if (dep[c] == 1) { s->lvl_rows[wr++] = c; s->row_level[c] = 0; }
    s->lvl_off[1] = wr;
    int prev = 0;
    s->max_level_size = wr;
    long mlb = 0;
    for (int t = 0; t < wr; ++t) mlb += off[s->lvl_rows[t] + 1] - off[s->lvl_rows[t]];
    s->max_level_blocks = (int)mlb;
    while (prev < wr) {
        ++nl;
        const int cur_end = wr;
        long lvl_blocks = 0;
        for (int t = prev; t < cur_end; ++t) {
            const int cur = s->lvl_rows[t];
            for (int p = off[cur]; p < off[cur + 1]; ++p) {
                const int jc = col[p];
                if (--dep[jc] == 1) {
                    s->lvl_rows[wr++] = jc;
                    s->row_level[jc] = nl;
                    lvl_blocks += off[jc + 1] - off[jc];
                }
            }
        }
        /* canonical form: rows of a level ascending */
        qsort(s->lvl_rows + cur_end, wr - cur_end, sizeof(int), cmp_int);
        if (wr - cur_end > s->max_level_size) s->max_level_size = wr - cur_end;
        if (lvl_blocks > s->max_level_blocks) s->max_level_blocks = (int)lvl_blocks;
        s->lvl_off[nl + 1] = wr;
        prev = cur_end;
    }
    s->num_levels = nl;
    s->unleveled_rows = cm - wr;
    free(dep);

    /* level block lists: pivot blocks then off-diagonal blocks, CSR order (:916-967) */
    s->lb_off = (int *)xmalloc(sizeof(int) * (nl + 1));
    s->lb = (int *)xmalloc(sizeof(int) * cnz);
    {
        int o = 0;
        for (int L = 0; L < nl; ++L) {
            s->lb_off[L] = o;
            for (int t = s->lvl_off[L]; t < s->lvl_off[L + 1]; ++t) {
                const int r = s->lvl_rows[t];
                for (int p = off[r]; p < off[r + 1]; ++p)
                    if (col[p] == r) s->lb[o++] = p;
            }
            /* off-diagonal blocks in increasing block id: walk rows ascending */
            for (int t = s->lvl_off[L]; t < s->lvl_off[L + 1]; ++t) {
                const int r = s->lvl_rows[t];
                for (int p = off[r]; p < off[r + 1]; ++p)
                    if (col[p] != r) s->lb[o++] = p;
            }
        }
        s->lb_off[nl] = o;
        s->lb_count = o;
    }

    /* column-level lists for the U' sweep (solve_analysis_block :2050-2150) */
    s->sb_off = (int *)xmalloc(sizeof(int) * (nl + 1));
    s->sb = (int *)xmalloc(sizeof(int) * cnz);
    {
        int o = 0;
        for (int L = 0; L < nl; ++L) {
            s->sb_off[L] = o;
            for (int t = s->lvl_off[L]; t < s->lvl_off[L + 1]; ++t) {
                const int c = s->lvl_rows[t];
                const int p = s->csc_blk[s->csc_off[c + 1] - 1];
                if (s->blk_row[p] == c) s->sb[o++] = p;
            }
            /* off-diagonal blocks whose column lies in level L, block id order */
            const int o_start = o;
            for (int t = s->lvl_off[L]; t < s->lvl_off[L + 1]; ++t) {
                const int c = s->lvl_rows[t];
                for (int q = s->csc_off[c]; q < s->csc_off[c + 1]; ++q) {
                    const int p = s->csc_blk[q];
                    if (s->blk_row[p] != c) s->sb[o++] = p;
                }
            }
            qsort(s->sb + o_start, o - o_start, sizeof(int), cmp_int);
        }
        s->sb_off[nl] = o;
    }

    /* formats and max_nnz (build_blocks :1059-1153) */
    s->fmt = (int *)xmalloc(sizeof(int) * cnz);
    s->max_nnz = (int *)xmalloc(sizeof(int) * cnz);
    for (int I = 0; I < cm; ++I) {
        int sum_nnz = 0, sum_blocks = 0;
        for (int p = off[I]; p < off[I + 1]; ++p) { sum_nnz += cnt[p]; sum_blocks += (cnt[p] != 0); }
        int avg_nnz;
        if (sum_blocks == 0) avg_nnz = 0; /* 0/0 in the reference; pinned to 0 */
        else if (value_bytes == 8) avg_nnz = (int)ceil((double)sum_nnz / (double)sum_blocks);
        else avg_nnz = (int)ceilf((float)sum_nnz / (float)sum_blocks);
        for (int p = off[I]; p < off[I + 1]; ++p) {
            const int r = s->bs[I + 1] - s->bs[I];
            const int c = s->bs[col[p] + 1] - s->bs[col[p]];
            const int src = (cnt[p] == 0) ? avg_nnz : cnt[p];
            int cap;
            if (value_bytes == 8) cap = (int)ceil(fill_factor * (double)src);
            else cap = (int)ceilf((float)fill_factor * (float)src);
            const int mx = (r * c < cap) ? r * c : cap;
            s->max_nnz[p] = mx;
            const double lhs = (double)((size_t)(4 + value_bytes) * (size_t)mx);
            const double rhs = (value_bytes == 8)
                ? 0.5 * 8.0 * (double)r * (double)c
                : (double)(0.5f * 4.0f * (float)r * (float)c);
            const int sparse = (I != col[p]) && ((double)I < 0.9 * (double)cm) && (lhs < rhs);
            s->fmt[p] = sparse ? ORC_SPARSE : ORC_DENSE;
        }
    }

    /* gather map of A's upper entries into blocks (build_blocks :1214-1266) */
    s->a_blk = (int *)xmalloc(sizeof(int) * (s->nnz ? s->nnz : 1));
    s->a_idx = (int *)xmalloc(sizeof(int) * (s->nnz ? s->nnz : 1));
    for (int i = 0; i < n; ++i) {
        const int I = s->row_block[i];
        for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) {
            const int c = colidx[p];
            if (c < i) { s->a_blk[p] = -1; s->a_idx[p] = -1; continue; }
            const int C = s->row_block[c];
            /* find block (I, C) in the sorted coarse row */
            int lo = off[I], hi = off[I + 1] - 1, b = -1;
            while (lo <= hi) {
                const int mid = (lo + hi) >> 1;
                if (col[mid] == C) { b = mid; break; }
                if (col[mid] < C) lo = mid + 1; else hi = mid - 1;
            }
            const int csz = s->bs[C + 1] - s->bs[C];
            s->a_blk[p] = b;
            s->a_idx[p] = (i - s->bs[I]) * csz + (c - s->bs[C]);
        }
    }
    return s;
}
