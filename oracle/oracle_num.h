/*
 * oracle_num.h -- numeric part of the CPU restatement of culip's block-iLDL^T
 * solve path, instantiated twice by oracle.c (REAL = double / float).
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Arithmetic is written with explicit fma() where the reference's CUDA source
 * has a multiply feeding an add (nvcc contracts those by default) and the
 * file is compiled with -ffp-contract=off, so every rounding is spelled out.
 * nvcc's choices, as the reference's own sm_100a build computes them
 * (oracle/_ref, tests/test_ref_parity.py): a*b + c*d -> fma(a, b, c*d);
 * x - a*b -> fma(-a, b, x); -a*b + c*d (a negated product first) ->
 * fma(c, d, -(a*b)): the negation is moved out of the product, the sum
 * becomes c*d - a*b and the first product is the fused one;
 * d_multiply_block_by_block_diagonal's sup*l + dia*m + sub*r ->
 * fma(sub, r, fma(dia, m, sup*l)) (only rows next to a 2x2 pivot see a
 * difference: elsewhere sup = sub = 0).
 * Reference kernels followed (libs/la/preconditioner/block_ildlt_kernels.impl.cuh
 * unless noted):
 *   d_load_block                      :22-81
 *   d_multiply_block_by_block_diag.   :372-411
 *   d_apply_left_right_update         :415-456
 *   d_factor_pivot_apply_update       :465-534
 *   d_ldlt_1x1_step / d_ldlt_2x2_step :538-585 / :589-675
 *   d_dense_pivot_op                  :679-739
 *   d_select_pivot_bunch_kaufman      :743-834
 *   d_select_pivot_rook               :838-948
 *   d_factor_pivot_factorize          :956-1083
 *   k_factor_pivot_blocks             :1146-1283
 *   d_col_pivot_block / k_pivot_col.. :1287-1418
 *   d_apply_offdiagonal_update        :1422-1485
 *   d_left_solve_with_D_Ut            :1489-1570
 *   k_update_scale_offdiagonal_blocks :1628-1803
 *   k_apply_block_dual_dropping       :1866-2074 (+ d_save_block :85-173)
 *   d_left_solve_row_major            :2087-2113
 *   k_solve_blocks_{off,}diagonal_..  :2353-2606
 *   k_solve_D, k_permute_P/Pt         libs/la/helper_kernels.impl.cuh:720-816
 *   SQMR::solve                       libs/la/iterative_solvers/sqmr.impl.cuh:109-355
 *   k_sym_ortho                       libs/la/helper_kernels.impl.cuh:662-700
 *
 * Deterministic choices where the reference is racy:
 *   - dual dropping: a level's requests are served from the pool the earlier
 *     levels left, in level-list order, and the level's spare slots join the
 *     pool after the level (the reference's CTAs race on one leftover
 *     counter, :1949-2008: each takes before it returns its own spare slots);
 *   - row norms: off-diagonal contributions are added in level-list order
 *     (the reference uses atomicAdd, :1792);
 *   - triangular sweeps: each fine row subtracts its off-diagonal terms in
 *     increasing global column order (the reference uses atomicAdd, :2485).
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define F(name) CAT(name, SUFFIX)

#define NZ_EPS 1e-10

/* An FP32 factor inverts a 2x2 pivot in FP64 when
 * |d11 d22 - d12^2| < bound (|d11 d22| + d12^2) (the library's
 * kPivotFp64Default rule; not in the reference, whose float factor inverts
 * every pivot in float).  The products of two floats are exact in double. */
#ifndef ORC_WIDE_2X2
#define ORC_WIDE_2X2
static int orc_wide_2x2(int is_float, double d11, double d12, double d22, double bound)
{
    if (!is_float) return 0;
    const double p = d11 * d22, q = d12 * d12;
    return fabs(p - q) < bound * (fabs(p) + q);
}
#endif

/* per fine row: (global col, value) lists of the strictly off-diagonal
 * block part of U, and of U' (its columns), sorted by column */
typedef struct {
    int *off, *col;
    REAL *val;
} F(rowlist_t);

typedef struct CAT(orc_fac, SUFFIX) {
    const orc_sym *s;
    F(rowlist_t) U, Ut;
    int pivot;
    REAL threshold;
    int literal;
    int *nnz, *maxnnz, *got_extra;
    int **idx;
    REAL **val;
    REAL *tri;
    int *is_piv, *perm;
    REAL *row_norm;
    const int *forced_grants; /* per block: grants taken from another run, or NULL */
    double piv64;             /* FP32: 2x2 pivots below this ratio inverted in FP64 */
    long leftover;        /* pool the blocks of the current level draw from */
} F(fac_t);

static int F(bsize)(const orc_sym *s, int blockrow) { return s->bs[blockrow + 1] - s->bs[blockrow]; }
static void F(build_rowlists)(const F(fac_t) *f, F(rowlist_t) *U, F(rowlist_t) *Ut);

/* d_load_block: zero the tile, then place the block (optionally transposed) */
static void F(load_tile)(const F(fac_t) *f, int b, REAL T[32][32], int transpose)
{
    const orc_sym *s = f->s;
    memset(T, 0, sizeof(REAL) * 1024);
    const int h = F(bsize)(s, s->blk_row[b]);
    const int w = F(bsize)(s, s->blk_col[b]);
    if (s->fmt[b] == ORC_DENSE) {
        const REAL *v = f->val[b];
        for (int i = 0; i < h; ++i)
            for (int j = 0; j < w; ++j) {
                if (transpose) T[j][i] = v[i * w + j];
                else T[i][j] = v[i * w + j];
            }
    } else {
        for (int e = 0; e < f->nnz[b]; ++e) {
            const int r = f->idx[b][e] / w, c = f->idx[b][e] % w;
            if (transpose) T[c][r] = f->val[b][e];
            else T[r][c] = f->val[b][e];
        }
    }
}

/* d_multiply_block_by_block_diagonal: rows a < h of Lt times tridiagonal D
 * (lanes r < w), D given as [3*r + {0: coupling to r-1, 1: diag, 2: to r+1}] */
static void F(mult_tridiag)(REAL Lt[32][32], const REAL *D, int h, int w)
{
    for (int a = 0; a < h; ++a) {
        REAL old[34];
        old[0] = 0;
        old[33] = 0;
        for (int r = 0; r < 32; ++r) old[r + 1] = Lt[a][r];
        for (int r = 0; r < w; ++r) {
            const REAL sup = D[3 * r], dia = D[3 * r + 1], sub = D[3 * r + 2];
            /* sup*l + dia*m + sub*r as the reference's build rounds it */
            Lt[a][r] = FMA(sub, old[r + 2], FMA(dia, old[r + 1], sup * old[r]));
        }
    }
}

/* d_apply_left_right_update: P[a][b] -= sum_r R[r][b] * Lt[a][r], one
 * separately rounded product per (a, b) and update. */
static void F(left_right_update)(const F(fac_t) *f, REAL P[32][32], REAL Lt[32][32],
                                 REAL R[32][32], int lh, int bw, int rh)
{
    for (int a = 0; a < lh; ++a) {
        REAL prod[32];
        if (f->literal) {
            for (int b = 0; b < 32; ++b) {
                REAL p = 0;
                for (int r = 0; r < bw; ++r) p = FMA(R[r][b], Lt[a][r], p);
                prod[b] = p;
            }
        } else {
            /* exact zero skipping: fma(0, x, p) == p for finite x */
            for (int b = 0; b < 32; ++b) prod[b] = 0;
            for (int r = 0; r < bw; ++r) {
                const REAL la = Lt[a][r];
                if (la == 0) continue;
                for (int b = 0; b < rh; ++b)
                    if (R[r][b] != 0) prod[b] = FMA(R[r][b], la, prod[b]);
            }
        }
        for (int b = 0; b < rh; ++b) P[a][b] -= prod[b];
    }
}

/* d_ldlt_1x1_step */
static void F(step_1x1)(REAL T[32][32], REAL *D, int row, int len)
{
    int modified = 0;
    REAL d11 = T[row][row];
    if (FABS(d11) < 1e-8) { d11 = (REAL)1e-6; modified = 1; }
    REAL u[32], ru[32];
    for (int l = 0; l < 32; ++l) {
        const REAL a = (l < row) ? (REAL)0 : T[row][l];
        u[l] = a / d11;
    }
    for (int l = 0; l < 32; ++l) { T[row][l] = u[l]; ru[l] = u[l] * d11; }
    for (int i = row + 1; i < len; ++i) {
        const REAL lv = ru[i];
        for (int l = 0; l < len; ++l) T[i][l] = FMA(-lv, u[l], T[i][l]);
    }
    if (modified) T[row][row] = 1;
    D[3 * row] = 0; D[3 * row + 1] = d11; D[3 * row + 2] = 0;
}

/* d_ldlt_2x2_step (Givens-based 2x2 solve) */
static void F(step_2x2)(REAL T[32][32], REAL *D, int row, int len, double piv64)
{
    int modified = 0;
    REAL d11 = T[row][row], d12 = T[row][row + 1], d22 = T[row + 1][row + 1];
    if (FABS(FMA(d11, d22, -(d12 * d12))) < 1e-8) {
        d11 = (REAL)1e-6; d22 = (REAL)1e-6; modified = 1;
    }
    if (orc_wide_2x2(sizeof(REAL) == 4, d11, d12, d22, piv64)) {
        /* the same steps in double, each result rounded to REAL once */
        const double e11 = d11, e12 = d12, e22 = d22;
        const double gr = sqrt(fma(e11, e11, e12 * e12));
        const double gc = e11 / gr, gs = e12 / gr;
        const double td11 = fma(gc, e11, gs * e12);
        const double td12 = fma(gc, e12, gs * e22);
        const double td22 = fma(gc, e22, -(gs * e12));
        double u1[32], u2[32], r1[32], r2[32];
        for (int l = 0; l < 32; ++l) {
            const double a1 = (l < row) ? 0.0 : (double)T[row][l];
            const double a2 = (l < row) ? 0.0 : ((l == row) ? e12 : (double)T[row + 1][l]);
            double x1 = fma(gc, a1, gs * a2);
            double x2 = fma(gc, a2, -(gs * a1));
            x2 = x2 / td22;
            x1 = fma(-td12, x2, x1) / td11;
            u1[l] = x1; u2[l] = x2;
        }
        for (int l = 0; l < 32; ++l) {
            T[row][l] = (l < row) ? (REAL)0 : (REAL)u1[l];
            T[row + 1][l] = (l < row) ? (REAL)0 : (REAL)u2[l];
            r1[l] = fma(u1[l], e11, u2[l] * e12);
            r2[l] = fma(u1[l], e12, u2[l] * e22);
        }
        for (int i = row + 2; i < len; ++i) {
            const double l1 = r1[i], l2 = r2[i];
            for (int l = 0; l < 32; ++l) T[i][l] = (REAL)((double)T[i][l] - fma(l1, u1[l], l2 * u2[l]));
        }
        if (modified) { T[row][row] = 1; T[row][row + 1] = 0; T[row + 1][row + 1] = 1; }
        D[3 * row] = 0; D[3 * row + 1] = d11; D[3 * row + 2] = d12;
        D[3 * (row + 1)] = d12; D[3 * (row + 1) + 1] = d22; D[3 * (row + 1) + 2] = 0;
        return;
    }
    const REAL gr = SQRT(FMA(d11, d11, d12 * d12));
    const REAL gc = d11 / gr, gs = d12 / gr;
    const REAL td11 = FMA(gc, d11, gs * d12);
    const REAL td12 = FMA(gc, d12, gs * d22);
    const REAL td22 = FMA(gc, d22, -(gs * d12));
    REAL u1[32], u2[32], r1[32], r2[32];
    for (int l = 0; l < 32; ++l) {
        const REAL a1 = (l < row) ? (REAL)0 : T[row][l];
        const REAL a2 = (l < row) ? (REAL)0 : ((l == row) ? d12 : T[row + 1][l]);
        REAL x1 = FMA(gc, a1, gs * a2);
        REAL x2 = FMA(gc, a2, -(gs * a1));
        x2 = x2 / td22;
        x1 = FMA(-td12, x2, x1) / td11;
        u1[l] = x1; u2[l] = x2;
    }
    for (int l = 0; l < 32; ++l) {
        T[row][l] = (l < row) ? (REAL)0 : u1[l];
        T[row + 1][l] = (l < row) ? (REAL)0 : u2[l];
        r1[l] = FMA(u1[l], d11, u2[l] * d12);
        r2[l] = FMA(u1[l], d12, u2[l] * d22);
    }
    for (int i = row + 2; i < len; ++i) {
        const REAL l1 = r1[i], l2 = r2[i];
        for (int l = 0; l < 32; ++l) T[i][l] -= FMA(l1, u1[l], l2 * u2[l]);
    }
    if (modified) { T[row][row] = 1; T[row][row + 1] = 0; T[row + 1][row + 1] = 1; }
    D[3 * row] = 0; D[3 * row + 1] = d11; D[3 * row + 2] = d12;
    D[3 * (row + 1)] = d12; D[3 * (row + 1) + 1] = d22; D[3 * (row + 1) + 2] = 0;
}

/* d_dense_pivot_op: symmetric swap of positions p1 < p2 on the upper triangle,
 * emulating the warp's lockstep loads then stores. */
static void F(pivot_swap)(REAL T[32][32], int *perm, int p1, int p2, int len)
{
    int ia[32], ib[32];
    REAL va[32], vb[32];
    for (int l = 0; l < 32; ++l) {
        if (l < p1) { ia[l] = 32 * l + p1; ib[l] = 32 * l + p2; }
        else if (l == p1) { ia[l] = 32 * p1 + p1; ib[l] = 32 * p2 + p2; }
        else if (l < p2) { ia[l] = 32 * p1 + l; ib[l] = 32 * (p1 + (l - p1)) + p2; }
        else if (l == p2) { ia[l] = 32 * p1 + p2; ib[l] = 32 * p1 + p2; }
        else { ia[l] = 32 * p1 + l; ib[l] = 32 * p2 + l; }
    }
    REAL *flat = &T[0][0];
    for (int l = 0; l < len; ++l) { va[l] = flat[ia[l]]; vb[l] = flat[ib[l]]; }
    for (int l = 0; l < len; ++l) flat[ia[l]] = vb[l];
    for (int l = 0; l < len; ++l) flat[ib[l]] = va[l];
    const int t = perm[p1]; perm[p1] = perm[p2]; perm[p2] = t;
}

static REAL F(bk_alpha)(void) { return (REAL)((1.0f + sqrtf(17.0f)) / 8.0f); }

/* warp argmax of |T[p][l]| over p < l < len, lowest index on ties */
static void F(row_argmax)(REAL T[32][32], int p, int len, int *r_out, REAL *w_out)
{
    int r = p + 1;
    REAL w = 0;
    for (int l = p + 1; l < len; ++l) {
        const REAL v = FABS(T[p][l]);
        if (v > w) { w = v; r = l; }
    }
    *r_out = r; *w_out = w;
}

/* |T| of the Schur complement entry (a, b) read from the upper triangle */
static REAL F(upper_abs)(REAL T[32][32], int a, int b) { return (a < b) ? FABS(T[a][b]) : FABS(T[b][a]); }

static void F(select_bk)(REAL T[32][32], int p, int len, int *order, int *p0, int *p1)
{
    const REAL alpha = F(bk_alpha)();
    *order = 1;
    int r; REAL w1;
    F(row_argmax)(T, p, len, &r, &w1);
    if (w1 > 0) {
        if (FABS(T[p][p]) >= alpha * w1) { *p0 = p; return; }
        REAL wr = 0;
        for (int l = p; l < len; ++l) {
            if (l == r) continue;
            const REAL v = F(upper_abs)(T, l, r);
            wr = (v > wr) ? v : wr;
        }
        if (FABS(T[p][p]) * wr >= alpha * w1 * w1) *p0 = p;
        else if (FABS(T[r][r]) >= alpha * wr) *p0 = r;
        else { *order = 2; *p0 = p; *p1 = r; }
    } else {
        *p0 = p;
    }
}

static void F(select_rook)(REAL T[32][32], int p, int len, int *order, int *p0, int *p1)
{
    const REAL alpha = F(bk_alpha)();
    *order = 1;
    int r; REAL wi;
    F(row_argmax)(T, p, len, &r, &wi);
    if (!(wi > 0)) { *p0 = p; return; }
    int i = p;
    if (FABS(T[p][p]) >= alpha * wi) { *p0 = i; return; }
    for (;;) {
        int q = p; REAL wr = 0; int first = 1;
        for (int l = p; l < len; ++l) {
            REAL v = (l == r) ? (REAL)0 : F(upper_abs)(T, l, r);
            if (first) { q = l; wr = v; first = 0; }
            else if (v > wr) { q = l; wr = v; }
        }
        if (FABS(T[r][r]) >= alpha * wr) { *p0 = r; return; }
        else if (wi == wr) { *order = 2; *p0 = i; *p1 = r; return; }
        else { i = r; r = q; wi = wr; }
    }
}

/* d_factor_pivot_factorize */
static void F(factorize_tile)(REAL T[32][32], int len, int *is_piv, REAL *D, int *perm, int method,
                              double piv64)
{
    const int use_piv = (method != ORC_PIV_STATIC);
    int p = 0;
    while (p < len) {
        int order, p0 = p, p1 = p + 1;
        if (p < len - 1 && method == ORC_PIV_BK) F(select_bk)(T, p, len, &order, &p0, &p1);
        else if (p < len - 1 && method == ORC_PIV_ROOK) F(select_rook)(T, p, len, &order, &p0, &p1);
        else { order = (p < len - 1 && !is_piv[p + 1]) ? 2 : 1; p0 = p; p1 = p + 1; }
        if (order == 1) {
            if (use_piv && p != p0) F(pivot_swap)(T, perm, p, p0, len);
            F(step_1x1)(T, D, p, len);
            if (use_piv) is_piv[p] = 1;
        } else {
            if (use_piv) {
                if (p0 != p) F(pivot_swap)(T, perm, p, p0, len);
                F(pivot_swap)(T, perm, p + 1, p1, len);
            }
            F(step_2x2)(T, D, p, len, piv64);
            if (use_piv) { is_piv[p] = 1; is_piv[p + 1] = 0; }
        }
        p += order;
    }
}

/* d_left_solve_with_D_Ut: A <- D^-1 U^-T A for an h x w block; U is the
 * factored pivot tile (row-major, unit upper with stored diagonal). */
static void F(left_solve_D_Ut)(REAL U[32][32], const REAL *D, REAL A[32][32],
                               const int *is_piv, int h, int w, int literal, double piv64)
{
    /* an identity pivot tile makes the substitution a sequence of exact
     * no-ops (divide by 1, subtract 0 * x); an all-zero column stays zero */
    int ident = 1;
    for (int i = 0; i < h && ident; ++i)
        for (int l = i; l < h; ++l)
            if ((l == i) ? (U[i][l] != 1) : (U[i][l] != 0)) { ident = 0; break; }
    for (int j = 0; j < w; ++j) {
        if (!literal) {
            int any = 0;
            for (int l = 0; l < h; ++l) any |= (A[l][j] != 0);
            if (!any) continue;
        }
        REAL rhs[32];
        for (int l = 0; l < 32; ++l) rhs[l] = (l < h) ? A[l][j] : (REAL)0;
        if (!ident || literal)
            for (int i = 0; i < h; ++i) {
                const REAL piv = rhs[i] / U[i][i];
                for (int l = i + 1; l < h; ++l) rhs[l] = FMA(-U[i][l], piv, rhs[l]);
            }
        for (int l = h; l < 32; ++l) rhs[l] = 0;
        REAL x1v[32], x2v[32];
        for (int l = 0; l < 32; ++l) {
            const REAL right = rhs[(l < 31) ? l + 1 : 31];
            const REAL d11 = (l < h) ? D[3 * l + 1] : (REAL)0;
            const REAL d12 = (l < h) ? D[3 * l + 2] : (REAL)0;
            /* shfl_down(d_11, 1): lane 31 keeps its own value */
            const int ln = (l < 31) ? l + 1 : 31;
            REAL d22 = (ln < h) ? D[3 * ln + 1] : (REAL)0;
            if (l == h) d22 = 0;
            const int two = (l + 1) < h && !is_piv[l + 1];
            if (l >= h) { x1v[l] = 0; x2v[l] = 0; continue; }
            if (two && orc_wide_2x2(sizeof(REAL) == 4, d11, d12, d22, piv64)) {
                const double e11 = d11, e12 = d12, e22 = d22;
                const double wr = sqrt(fma(e11, e11, e12 * e12));
                const double wc = e11 / wr, ws = e12 / wr;
                double y1 = fma(wc, (double)rhs[l], ws * (double)right);
                double y2 = fma(wc, (double)right, -(ws * (double)rhs[l]));
                const double w11 = fma(wc, e11, ws * e12);
                const double w12 = fma(wc, e12, ws * e22);
                const double w22 = fma(wc, e22, -(ws * e12));
                y2 = y2 / w22;
                y1 = fma(-w12, y2, y1) / w11;
                x1v[l] = (REAL)y1; x2v[l] = (REAL)y2;
                continue;
            }
            const REAL gr = SQRT(FMA(d11, d11, d12 * d12));
            const REAL gc = d11 / gr, gs = d12 / gr;
            REAL x1 = FMA(gc, rhs[l], gs * right);
            REAL x2 = FMA(gc, right, -(gs * rhs[l]));
            const REAL td11 = FMA(gc, d11, gs * d12);
            const REAL td12 = FMA(gc, d12, gs * d22);
            const REAL td22 = FMA(gc, d22, -(gs * d12));
            x2 = two ? (x2 / td22) : (REAL)0;
            x1 = FMA(-td12, x2, x1) / td11;
            x1v[l] = x1; x2v[l] = x2;
        }
        for (int l = 0; l < h; ++l) {
            if (is_piv[l]) A[l][j] = x1v[l];
            if ((l + 1) < h && !is_piv[l + 1]) A[l + 1][j] = x2v[l];
        }
    }
}

/* k_apply_block_dual_dropping, first half: threshold dropping of a sparse
 * block's tile and the count of its remaining entries (|v| > NZ_EPS). */
static int F(drop_count)(const F(fac_t) *f, int b, REAL T[32][32])
{
    const orc_sym *s = f->s;
    const int I = s->blk_row[b];
    const int h = F(bsize)(s, I), w = F(bsize)(s, s->blk_col[b]);
    const int from = s->bs[I];
    int nnz = 0;
    for (int i = 0; i < h; ++i) {
        const REAL nrm = (REAL)sqrtf((float)f->row_norm[from + i]);
        for (int l = 0; l < w; ++l) {
            const REAL v = T[i][l];
            const int drop = FABS(v) < f->threshold * nrm;
            const int nz = FABS(v) > NZ_EPS;
            if (drop && nz) T[i][l] = 0;
            nnz += (!drop && nz);
        }
    }
    return nnz;
}

/* second half + d_save_block: store the tile in its final capacity mx
 * (sparse: its nnz entries, or the mx largest |v| when nnz > mx). */
static void F(save_block)(F(fac_t) *f, int b, REAL T[32][32], int nnz, int mx)
{
    const orc_sym *s = f->s;
    const int I = s->blk_row[b];
    const int h = F(bsize)(s, I), w = F(bsize)(s, s->blk_col[b]);
    if (s->fmt[b] == ORC_DENSE) {
        for (int i = 0; i < h; ++i)
            for (int j = 0; j < w; ++j) f->val[b][i * w + j] = T[i][j];
        f->nnz[b] = 0;
        return;
    }
    f->maxnnz[b] = mx;
    const int cap = (nnz < mx) ? nnz : mx;
    free(f->idx[b]); free(f->val[b]);
    f->idx[b] = (int *)malloc(sizeof(int) * (cap ? cap : 1));
    f->val[b] = (REAL *)malloc(sizeof(REAL) * (cap ? cap : 1));
    if (nnz > mx) {
        /* keep the mx largest |v|, ties to the lower tile index (stable
         * descending radix sort, :2016-2061); stored sorted by local index */
        char taken[1024];
        memset(taken, 0, sizeof(taken));
        for (int k = 0; k < mx; ++k) {
            int best = -1; REAL bv = -1;
            for (int t = 0; t < 1024; ++t) {
                if (taken[t]) continue;
                const int rr = t / 32, cc = t % 32;
                const REAL key = (rr < h && cc < w) ? FABS(T[rr][cc]) : (REAL)0;
                if (key > bv) { bv = key; best = t; }
            }
            taken[best] = 1;
        }
        int o = 0;
        for (int t = 0; t < 1024; ++t)
            if (taken[t]) { const int rr = t / 32, cc = t % 32; f->idx[b][o] = rr * w + cc; f->val[b][o] = T[rr][cc]; ++o; }
        f->nnz[b] = mx;
    } else {
        int o = 0;
        for (int i = 0; i < h; ++i)
            for (int l = 0; l < w; ++l)
                if (FABS(T[i][l]) > NZ_EPS) { f->idx[b][o] = i * w + l; f->val[b][o] = T[i][l]; ++o; }
        f->nnz[b] = o;
    }
}

/* a sparse block of a level; b >= 0 and tile set when it outgrew its
 * capacity and waits for the level's grants */
typedef struct {
    int b, nnz;
    REAL (*T)[32];
} F(pending_t);

F(fac_t) *F(orc_factor)(const orc_sym *s, const REAL *vals, const int *is_piv_init,
                        int pivot, REAL threshold, int literal)
{
    return F(orc_factor_forced)(s, vals, is_piv_init, pivot, threshold, literal, NULL, ORC_PIVOT_FP64_DEFAULT);
}

/* forced_grants (coarse_nnz entries, or NULL): the extra slots each block that
 * outgrows its capacity receives, taken from another run (the reference's
 * own grants race between a level's CTAs); NULL follows the pool */
F(fac_t) *F(orc_factor_forced)(const orc_sym *s, const REAL *vals, const int *is_piv_init,
                               int pivot, REAL threshold, int literal, const int *forced_grants, double piv64)
{
    F(fac_t) *f = (F(fac_t) *)calloc(1, sizeof(F(fac_t)));
    const int n = s->n, cnz = s->coarse_nnz;
    f->s = s; f->pivot = pivot; f->threshold = threshold; f->literal = literal;
    f->forced_grants = forced_grants;
    f->piv64 = piv64;
    f->nnz = (int *)calloc(cnz, sizeof(int));
    f->maxnnz = (int *)malloc(sizeof(int) * cnz);
    f->got_extra = (int *)calloc(cnz, sizeof(int));
    f->idx = (int **)calloc(cnz, sizeof(int *));
    f->val = (REAL **)calloc(cnz, sizeof(REAL *));
    f->tri = (REAL *)calloc(3 * (size_t)n + 96, sizeof(REAL));
    f->is_piv = (int *)malloc(sizeof(int) * (n + 1));
    f->perm = (int *)malloc(sizeof(int) * (n + 1));
    f->row_norm = (REAL *)calloc(n + 1, sizeof(REAL));
    for (int i = 0; i < n; ++i) { f->is_piv[i] = is_piv_init[i]; f->perm[i] = i; }
    f->is_piv[n] = 1; f->perm[n] = n;

    /* build_blocks gather of A (:1214-1266) */
    for (int b = 0; b < cnz; ++b) {
        f->maxnnz[b] = s->max_nnz[b];
        const int h = F(bsize)(s, s->blk_row[b]), w = F(bsize)(s, s->blk_col[b]);
        if (s->fmt[b] == ORC_DENSE) {
            f->val[b] = (REAL *)calloc((size_t)h * w, sizeof(REAL));
        } else {
            const int cap = s->max_nnz[b] > s->blk_nnzA[b] ? s->max_nnz[b] : s->blk_nnzA[b];
            f->idx[b] = (int *)malloc(sizeof(int) * (cap ? cap : 1));
            f->val[b] = (REAL *)malloc(sizeof(REAL) * (cap ? cap : 1));
        }
    }
    {
        const int nnzK = s->nnz;
        for (int p = 0; p < nnzK; ++p) {
            const int b = s->a_blk[p];
            if (b < 0) continue;
            if (s->fmt[b] == ORC_DENSE) f->val[b][s->a_idx[p]] = vals[p];
            else { f->idx[b][f->nnz[b]] = s->a_idx[p]; f->val[b][f->nnz[b]] = vals[p]; f->nnz[b]++; }
        }
    }

    /* the rows of a level are independent (each reads the levels before
     * it): steps 1-3 run over the level's block rows on all threads; only
     * the grants of the blocks that outgrow their capacity go in level-list
     * order, so the result does not depend on the thread count */
    int *row_first = (int *)malloc(sizeof(int) * (s->num_blocks + 1));
    F(pending_t) *pend = NULL;
    int pend_cap = 0;
    for (int L = 0; L < s->num_levels; ++L) {
        const int lb0 = s->lb_off[L], lb1 = s->lb_off[L + 1];
        const int npiv = s->lvl_off[L + 1] - s->lvl_off[L];
        /* step 1: pivot blocks (k_factor_pivot_blocks) */
#pragma omp parallel for schedule(dynamic, 4) if (npiv > 64)
        for (int t = lb0; t < lb0 + npiv; ++t) {
            REAL T[32][32], Lt[32][32], R[32][32];
            const int b = s->lb[t];
            const int I = s->blk_row[b];
            const int from = s->bs[I], len = F(bsize)(s, I);
            F(load_tile)(f, b, T, 0);
            for (int q = s->csc_off[I]; q < s->csc_off[I + 1] - 1; ++q) {
                const int kb = s->csc_blk[q];
                const int K = s->blk_row[kb];
                const int bw = F(bsize)(s, K);
                F(load_tile)(f, kb, R, 0);
                for (int a = 0; a < 32; ++a)
                    for (int r = 0; r < 32; ++r) Lt[a][r] = R[r][a];
                F(mult_tridiag)(Lt, f->tri + 3 * (size_t)s->bs[K], len, bw);
                F(left_right_update)(f, T, Lt, R, len, bw, len);
            }
            F(factorize_tile)(T, len, f->is_piv + from, f->tri + 3 * (size_t)from, f->perm + from, pivot,
                              f->piv64);
            for (int l = 0; l < len; ++l) {
                REAL rs = 0;
                for (int j = 0; j < len; ++j) rs = FMA(T[l][j], T[l][j], rs);
                f->row_norm[from + l] = rs;
            }
            F(save_block)(f, b, T, 0, 0); /* dense: exact copy */
        }
        /* steps 2-4 per block row (off-diagonal blocks are grouped by row) */
        int nrows = 0;
        for (int t = lb0 + npiv; t < lb1; ++t)
            if (t == lb0 + npiv || s->blk_row[s->lb[t]] != s->blk_row[s->lb[t - 1]]) row_first[nrows++] = t;
        row_first[nrows] = lb1;
        long spare = 0;
        int npend = 0;
        for (int t = lb0 + npiv; t < lb1; ++t) {
            const int b = s->lb[t];
            npend += (s->fmt[b] == ORC_SPARSE);
        }
        if (npend > pend_cap) {
            free(pend);
            pend_cap = npend;
            pend = (F(pending_t) *)malloc(sizeof(F(pending_t)) * (pend_cap ? pend_cap : 1));
        }
        /* pend[k] is the k-th sparse block of the level's list (b < 0: fits) */
        int *pend_base = (int *)malloc(sizeof(int) * (nrows + 1));
        pend_base[0] = 0;
        for (int r = 0; r < nrows; ++r) {
            int c = 0;
            for (int t = row_first[r]; t < row_first[r + 1]; ++t) c += (s->fmt[s->lb[t]] == ORC_SPARSE);
            pend_base[r + 1] = pend_base[r] + c;
        }
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : spare) if (nrows > 16)
        for (int r = 0; r < nrows; ++r) {
            REAL Lt[32][32], R[32][32], U[32][32];
            const int t = row_first[r], t_end = row_first[r + 1];
            const int I = s->blk_row[s->lb[t]];
            const int nb = t_end - t;
            REAL (*tiles)[32][32] = (REAL (*)[32][32])malloc(sizeof(REAL) * 1024 * (nb ? nb : 1));
            const int from = s->bs[I], h = F(bsize)(s, I);
            /* the row's pivot tile from final (dense) storage */
            const int pb = s->csc_blk[s->csc_off[I + 1] - 1];
            F(load_tile)(f, pb, U, 0);
            for (int k = 0; k < nb; ++k) {
                const int b = s->lb[t + k];
                const int J = s->blk_col[b];
                const int w = F(bsize)(s, J);
                REAL (*A)[32] = tiles[k];
                F(load_tile)(f, b, A, 0);
                int ip = s->csc_off[I], ie = s->csc_off[I + 1] - 1;
                int jp = s->csc_off[J], je = s->csc_off[J + 1] - 1;
                while (ip < ie && jp < je) {
                    const int ir = s->blk_row[s->csc_blk[ip]], jr = s->blk_row[s->csc_blk[jp]];
                    if (ir == jr) {
                        const int K = ir, bw = F(bsize)(s, K);
                        F(load_tile)(f, s->csc_blk[ip], Lt, 1);
                        F(mult_tridiag)(Lt, f->tri + 3 * (size_t)s->bs[K], h, bw);
                        F(load_tile)(f, s->csc_blk[jp], R, 0);
                        F(left_right_update)(f, A, Lt, R, h, bw, w);
                    }
                    ip += (ir <= jr);
                    jp += (ir >= jr);
                }
                if (pivot != ORC_PIV_STATIC) {
                    REAL tmp[32][32];
                    memcpy(tmp, A, sizeof(tmp));
                    for (int i = 0; i < h; ++i) {
                        const int pi = f->perm[from + i] - from;
                        for (int l = 0; l < 32; ++l) A[i][l] = tmp[pi][l];
                    }
                }
                F(left_solve_D_Ut)(U, f->tri + 3 * (size_t)from, A, f->is_piv + from, h, w, f->literal,
                                   f->piv64);
                if (f->threshold > 0 || f->literal)
                    for (int l = 0; l < h; ++l) {
                        REAL rs = 0;
                        for (int j = 0; j < w; ++j) rs = FMA(A[l][j], A[l][j], rs);
                        f->row_norm[from + l] += rs;
                    }
            }
            /* dropping: blocks within capacity are stored now, the others wait
             * for the level's grants */
            int pk = pend_base[r];
            for (int k = 0; k < nb; ++k) {
                const int b = s->lb[t + k];
                if (s->fmt[b] == ORC_DENSE) {
                    F(save_block)(f, b, tiles[k], 0, 0);
                    continue;
                }
                const int nnz = F(drop_count)(f, b, tiles[k]);
                const int mx = f->maxnnz[b];
                if (nnz > mx) {
                    pend[pk].b = b;
                    pend[pk].nnz = nnz;
                    pend[pk].T = (REAL (*)[32])malloc(sizeof(REAL) * 1024);
                    memcpy(pend[pk].T, tiles[k], sizeof(REAL) * 1024);
                } else {
                    pend[pk].b = -1;
                    F(save_block)(f, b, tiles[k], nnz, mx);
                    spare += mx - nnz;
                }
                ++pk;
            }
            free(tiles);
        }
        /* the level's requests, in level-list order, from the pool the earlier
         * levels left */
        for (int k = 0; k < pend_base[nrows]; ++k) {
            if (pend[k].b < 0) continue;
            const int b = pend[k].b, nnz = pend[k].nnz;
            int mx = f->maxnnz[b];
            const long req = nnz - mx;
            long granted = (req < f->leftover) ? req : f->leftover;
            if (granted < 0) granted = 0;
            if (f->forced_grants) granted = f->forced_grants[b];
            f->leftover -= granted;
            mx += (int)granted;
            f->got_extra[b] = (int)granted;
            spare += (mx - nnz > 0) ? (mx - nnz) : 0;
            F(save_block)(f, b, pend[k].T, nnz, mx);
            free(pend[k].T);
        }
        free(pend_base);
        /* step 3 (k_pivot_col_blocks): propagate pivot permutations upwards */
        if (pivot != ORC_PIV_STATIC) {
#pragma omp parallel for schedule(dynamic, 8) if (npiv > 64)
            for (int q = s->lvl_off[L]; q < s->lvl_off[L + 1]; ++q) {
                const int I = s->lvl_rows[q];
                const int from = s->bs[I], bw = F(bsize)(s, I);
                int lp[32], inv[32], same = 1;
                for (int l = 0; l < bw; ++l) { lp[l] = f->perm[from + l] - from; inv[lp[l]] = l; }
                for (int l = 0; l < bw; ++l) same &= (inv[l] == l);
                if (same) continue;
                for (int c = s->csc_off[I]; c < s->csc_off[I + 1] - 1; ++c) {
                    const int b = s->csc_blk[c];
                    const int hh = F(bsize)(s, s->blk_row[b]);
                    if (s->fmt[b] == ORC_SPARSE) {
                        for (int e = 0; e < f->nnz[b]; ++e) {
                            const int r = f->idx[b][e] / bw, cc = f->idx[b][e] % bw;
                            f->idx[b][e] = r * bw + inv[cc];
                        }
                    } else {
                        REAL *v = f->val[b];
                        for (int i = 0; i < hh; ++i) {
                            REAL row[32];
                            for (int l = 0; l < bw; ++l) row[l] = v[i * bw + l];
                            for (int l = 0; l < bw; ++l) v[i * bw + l] = row[lp[l]];
                        }
                    }
                }
            }
        }
        /* the level's spare slots join the pool for the later levels */
        f->leftover += spare;
    }
    free(row_first);
    free(pend);
    F(build_rowlists)(f, &f->U, &f->Ut);
    return f;
}

void F(orc_fac_free)(F(fac_t) *f)
{
    if (!f) return;
    free(f->U.off); free(f->U.col); free(f->U.val);
    free(f->Ut.off); free(f->Ut.col); free(f->Ut.val);
    for (int b = 0; b < f->s->coarse_nnz; ++b) { free(f->idx[b]); free(f->val[b]); }
    free(f->idx); free(f->val); free(f->nnz); free(f->maxnnz); free(f->got_extra);
    free(f->tri); free(f->is_piv); free(f->perm); free(f->row_norm);
    free(f);
}

long F(orc_fac_export_size)(const F(fac_t) *f)
{
    long tot = 0;
    const orc_sym *s = f->s;
    for (int b = 0; b < s->coarse_nnz; ++b)
        tot += (s->fmt[b] == ORC_DENSE) ? (long)F(bsize)(s, s->blk_row[b]) * F(bsize)(s, s->blk_col[b]) : f->nnz[b];
    return tot;
}

#ifndef ORACLE_NUM_CMP_IDX
#define ORACLE_NUM_CMP_IDX
static int cmp_idx_pair(const void *a, const void *b)
{
    const int x = ((const int *)a)[0], y = ((const int *)b)[0];
    return (x > y) - (x < y);
}
#endif

void F(orc_fac_export)(const F(fac_t) *f, int *blk_nnz, long *blk_off, int *idx, REAL *val,
                       REAL *tri, int *is_piv, int *perm, int *got_extra)
{
    const orc_sym *s = f->s;
    long o = 0;
    for (int b = 0; b < s->coarse_nnz; ++b) {
        blk_off[b] = o;
        blk_nnz[b] = f->nnz[b];
        got_extra[b] = f->got_extra[b];
        if (s->fmt[b] == ORC_DENSE) {
            const int cnt = F(bsize)(s, s->blk_row[b]) * F(bsize)(s, s->blk_col[b]);
            for (int e = 0; e < cnt; ++e) { idx[o + e] = e; val[o + e] = f->val[b][e]; }
            o += cnt;
        } else {
            const int cnt = f->nnz[b];
            /* canonical order: sorted by local index */
            int *tmp = (int *)malloc(sizeof(int) * 2 * (cnt ? cnt : 1));
            for (int e = 0; e < cnt; ++e) { tmp[2 * e] = f->idx[b][e]; tmp[2 * e + 1] = e; }
            qsort(tmp, cnt, 2 * sizeof(int), cmp_idx_pair);
            for (int e = 0; e < cnt; ++e) { idx[o + e] = tmp[2 * e]; val[o + e] = f->val[b][tmp[2 * e + 1]]; }
            free(tmp);
            o += cnt;
        }
    }
    blk_off[s->coarse_nnz] = o;
    memcpy(tri, f->tri, sizeof(REAL) * 3 * (size_t)s->n);
    memcpy(is_piv, f->is_piv, sizeof(int) * s->n);
    memcpy(perm, f->perm, sizeof(int) * s->n);
}

/* ------------------------------ solves ---------------------------------- */

#ifndef ORACLE_NUM_CMP_COL
#define ORACLE_NUM_CMP_COL
static int cmp_colval(const void *a, const void *b)
{
    const int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}
#endif

static void F(build_rowlists)(const F(fac_t) *f, F(rowlist_t) *U, F(rowlist_t) *Ut)
{
    const orc_sym *s = f->s;
    const int n = s->n;
    int *cu = (int *)calloc(n + 1, sizeof(int)), *ct = (int *)calloc(n + 1, sizeof(int));
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            U->off = (int *)malloc(sizeof(int) * (n + 1)); Ut->off = (int *)malloc(sizeof(int) * (n + 1));
            U->off[0] = 0; Ut->off[0] = 0;
            for (int i = 0; i < n; ++i) { U->off[i + 1] = U->off[i] + cu[i]; Ut->off[i + 1] = Ut->off[i] + ct[i]; }
            U->col = (int *)malloc(sizeof(int) * (U->off[n] + 1)); U->val = (REAL *)malloc(sizeof(REAL) * (U->off[n] + 1));
            Ut->col = (int *)malloc(sizeof(int) * (Ut->off[n] + 1)); Ut->val = (REAL *)malloc(sizeof(REAL) * (Ut->off[n] + 1));
            memset(cu, 0, sizeof(int) * (n + 1)); memset(ct, 0, sizeof(int) * (n + 1));
        }
        for (int b = 0; b < s->coarse_nnz; ++b) {
            const int I = s->blk_row[b], J = s->blk_col[b];
            if (I == J) continue;
            const int w = F(bsize)(s, J), h = F(bsize)(s, I);
            const int cnt = (s->fmt[b] == ORC_DENSE) ? h * w : f->nnz[b];
            for (int e = 0; e < cnt; ++e) {
                const int li = (s->fmt[b] == ORC_DENSE) ? e : f->idx[b][e];
                const REAL v = f->val[b][e];
                if (v == 0) continue;
                const int r = s->bs[I] + li / w, c = s->bs[J] + li % w;
                if (pass == 0) { cu[r]++; ct[c]++; }
                else {
                    U->col[U->off[r] + cu[r]] = c; U->val[U->off[r] + cu[r]] = v; cu[r]++;
                    Ut->col[Ut->off[c] + ct[c]] = r; Ut->val[Ut->off[c] + ct[c]] = v; ct[c]++;
                }
            }
        }
    }
    /* sort each row's entries by column */
    for (int pass = 0; pass < 2; ++pass) {
        F(rowlist_t) *L = pass ? Ut : U;
        for (int i = 0; i < n; ++i) {
            const int a = L->off[i], e = L->off[i + 1];
            if (e - a < 2) continue;
            struct { int c; int pad; REAL v; } *tmp = malloc(sizeof(*tmp) * (e - a));
            for (int k = a; k < e; ++k) { tmp[k - a].c = L->col[k]; tmp[k - a].v = L->val[k]; }
            qsort(tmp, e - a, sizeof(*tmp), cmp_colval);
            for (int k = a; k < e; ++k) { L->col[k] = tmp[k - a].c; L->val[k] = tmp[k - a].v; }
            free(tmp);
        }
    }
    free(cu); free(ct);
}

/* U^-1 in place (levels last to first), then U'^-1 variants */
static void F(solve_U)(const F(fac_t) *f, const F(rowlist_t) *U, REAL *x)
{
    const orc_sym *s = f->s;
    for (int L = s->num_levels - 1; L >= 0; --L) {
        /* block rows of a level are independent (each reads earlier levels only) */
#pragma omp parallel for schedule(dynamic, 16) if (s->lvl_off[L + 1] - s->lvl_off[L] > 256)
        for (int q = s->lvl_off[L]; q < s->lvl_off[L + 1]; ++q) {
            const int I = s->lvl_rows[q];
            const int from = s->bs[I], h = F(bsize)(s, I);
            REAL t[32];
            for (int r = 0; r < h; ++r) {
                REAL acc = x[from + r];
                for (int k = U->off[from + r]; k < U->off[from + r + 1]; ++k)
                    acc = FMA(-U->val[k], x[U->col[k]], acc);
                t[r] = acc;
            }
            const int pb = s->csc_blk[s->csc_off[I + 1] - 1];
            const REAL *P = f->val[pb];
            for (int c = h - 1; c >= 0; --c) {
                t[c] = t[c] / P[c * h + c];
                for (int r = 0; r < c; ++r) t[r] = FMA(-P[r * h + c], t[c], t[r]);
            }
            for (int r = 0; r < h; ++r) x[from + r] = t[r];
        }
    }
}

static void F(solve_Ut)(const F(fac_t) *f, const F(rowlist_t) *Ut, REAL *x)
{
    const orc_sym *s = f->s;
    for (int L = 0; L < s->num_levels; ++L) {
#pragma omp parallel for schedule(dynamic, 16) if (s->lvl_off[L + 1] - s->lvl_off[L] > 256)
        for (int q = s->lvl_off[L]; q < s->lvl_off[L + 1]; ++q) {
            const int I = s->lvl_rows[q];
            const int from = s->bs[I], h = F(bsize)(s, I);
            REAL t[32];
            for (int r = 0; r < h; ++r) {
                REAL acc = x[from + r];
                for (int k = Ut->off[from + r]; k < Ut->off[from + r + 1]; ++k)
                    acc = FMA(-Ut->val[k], x[Ut->col[k]], acc);
                t[r] = acc;
            }
            const int pb = s->csc_blk[s->csc_off[I + 1] - 1];
            const REAL *P = f->val[pb];
            for (int r = 0; r < h; ++r) {
                t[r] = t[r] / P[r * h + r];
                for (int c = r + 1; c < h; ++c) t[c] = FMA(-P[r * h + c], t[r], t[c]);
            }
            for (int r = 0; r < h; ++r) x[from + r] = t[r];
        }
    }
}

/* k_solve_D (Givens-based 1x1 / 2x2 block-diagonal solve), from a copy */
static void F(solve_D)(int n, const REAL *tri, const int *is_piv, const REAL *in, REAL *out, double piv64)
{
    /* every out entry is written by one g only, from the copy in */
#pragma omp parallel for schedule(static) if (n > 16384)
    for (int g = 0; g < n; ++g) {
        const int this_piv = is_piv[g];
        const int next_piv = (g < n - 1) ? is_piv[g + 1] : 1;
        const REAL p11 = tri[3 * g + 1], p12 = tri[3 * g + 2];
        const REAL p22 = !next_piv ? tri[3 * (g + 1) + 1] : (REAL)1;
        const REAL r1 = in[g], r2 = (g < n - 1) ? in[g + 1] : (REAL)0;
        if (!next_piv && orc_wide_2x2(sizeof(REAL) == 4, p11, p12, p22, piv64)) {
            const double e11 = p11, e12 = p12, e22 = p22;
            const double wr = sqrt(fma(e11, e11, e12 * e12));
            const double wc = e11 / wr, ws = e12 / wr;
            double y1 = fma(wc, (double)r1, ws * (double)r2);
            double y2 = fma(wc, (double)r2, -(ws * (double)r1));
            const double t12 = fma(wc, e12, ws * e22);
            const double t22 = fma(wc, e22, -(ws * e12));
            y2 = y2 / t22;
            y1 = fma(-t12, y2, y1) / wr;
            if (this_piv) out[g] = (REAL)y1;
            out[g + 1] = (REAL)y2;
            continue;
        }
        const REAL gr = SQRT(FMA(p11, p11, p12 * p12));
        const REAL gc = p11 / gr, gs = p12 / gr;
        REAL g1 = FMA(gc, r1, gs * r2);
        REAL g2 = FMA(gc, r2, -(gs * r1));
        const REAL tp12 = FMA(gc, p12, gs * p22);
        const REAL tp22 = FMA(gc, p22, -(gs * p12));
        g2 = g2 / tp22;
        g1 = FMA(-tp12, g2, g1) / gr;
        if (this_piv) out[g] = g1;
        if (!next_piv) out[g + 1] = g2;
    }
}

/* One block-Jacobi sweep of U x = b (UPPER) or U' x = b: every block row at
 * once from the previous iterate, x_out_I = U_II^-1 (b_I - U_I* x_in), with
 * the same per-row term order and pivot-tile substitution as solve_U /
 * solve_Ut; k_solve_block_stripe_level in solve_U_jacobi / solve_Ut_jacobi
 * (block_ildlt.impl.cuh:2455-2494, 2635-2674), starting from x = 0. */
static void F(jacobi_sweep)(const F(fac_t) *f, const F(rowlist_t) *R, int upper, const REAL *b,
                            const REAL *x_in, REAL *x_out)
{
    const orc_sym *s = f->s;
    for (int I = 0; I < s->num_blocks; ++I) {
        const int from = s->bs[I], h = F(bsize)(s, I);
        REAL t[32];
        for (int r = 0; r < h; ++r) {
            REAL acc = b[from + r];
            for (int k = R->off[from + r]; k < R->off[from + r + 1]; ++k)
                acc = FMA(-R->val[k], x_in[R->col[k]], acc);
            t[r] = acc;
        }
        const int pb = s->csc_blk[s->csc_off[I + 1] - 1];
        const REAL *P = f->val[pb];
        if (upper) {
            for (int c = h - 1; c >= 0; --c) {
                t[c] = t[c] / P[c * h + c];
                for (int r = 0; r < c; ++r) t[r] = FMA(-P[r * h + c], t[c], t[r]);
            }
        } else {
            for (int r = 0; r < h; ++r) {
                t[r] = t[r] / P[r * h + r];
                for (int c = r + 1; c < h; ++c) t[c] = FMA(-P[r * h + c], t[r], t[c]);
            }
        }
        for (int r = 0; r < h; ++r) x_out[from + r] = t[r];
    }
}

static void F(jacobi_solve)(const F(fac_t) *f, const F(rowlist_t) *R, int upper, int sweeps, const REAL *b,
                            REAL *x)
{
    const int n = f->s->n;
    REAL *a = (REAL *)calloc(n ? n : 1, sizeof(REAL));
    REAL *c = (REAL *)calloc(n ? n : 1, sizeof(REAL));
    for (int sw = 0; sw < sweeps; ++sw) {
        F(jacobi_sweep)(f, R, upper, b, a, c);
        REAL *t = a; a = c; c = t;
    }
    memcpy(x, a, sizeof(REAL) * n);
    free(a);
    free(c);
}

/* solve_left / solve_right with SOLVE_JACOBI (set_solve_algorithm,
 * block_ildlt.impl.cuh:253-258): the triangular solves replaced by `sweeps`
 * block-Jacobi sweeps; P, P' and D as in the exact applies. */
void F(orc_prec_apply_jacobi)(const F(fac_t) *f, int stage, int sweeps, const REAL *b, REAL *x)
{
    const int n = f->s->n;
    if (stage == 1) {
        F(orc_prec_apply)(f, 1, b, x);
        return;
    }
    REAL *t = (REAL *)malloc(sizeof(REAL) * (n ? n : 1));
    if (stage == 0) {
        for (int g = 0; g < n; ++g) t[g] = b[f->perm[g]];        /* k_permute_Pt */
        F(jacobi_solve)(f, &f->Ut, 0, sweeps, t, x);
    } else {
        REAL *u = (REAL *)malloc(sizeof(REAL) * (n ? n : 1));
        F(jacobi_solve)(f, &f->U, 1, sweeps, b, u);
        for (int g = 0; g < n; ++g) x[f->perm[g]] = u[g];        /* k_permute_P */
        free(u);
    }
    free(t);
}

/* solve_left (P' then U'^-1), solve_middle (D^-1, applied to a copy of b as in
 * block_ildlt.impl.cuh:216-219) and solve_right (U^-1 then P),
 * block_ildlt.impl.cuh:183-246. */
void F(orc_prec_apply)(const F(fac_t) *f, int stage, const REAL *b, REAL *x)
{
    const orc_sym *s = f->s;
    const int n = s->n;
    if (stage == 1) {
        REAL *t = (REAL *)malloc(sizeof(REAL) * (n ? n : 1));
#pragma omp parallel for schedule(static) if (n > 16384)
        for (int g = 0; g < n; ++g) { t[g] = b[g]; x[g] = b[g]; }
        F(solve_D)(n, f->tri, f->is_piv, t, x, f->piv64);
        free(t);
        return;
    }
    if (stage == 0) {
#pragma omp parallel for schedule(static) if (n > 16384)
        for (int g = 0; g < n; ++g) x[g] = b[f->perm[g]];        /* k_permute_Pt */
        F(solve_Ut)(f, &f->Ut, x);
    } else {
        REAL *t = (REAL *)malloc(sizeof(REAL) * (n ? n : 1));
#pragma omp parallel for schedule(static) if (n > 16384)
        for (int g = 0; g < n; ++g) t[g] = b[g];
        F(solve_U)(f, &f->U, t);
#pragma omp parallel for schedule(static) if (n > 16384)
        for (int g = 0; g < n; ++g) x[f->perm[g]] = t[g];        /* k_permute_P */
        free(t);
    }
}
