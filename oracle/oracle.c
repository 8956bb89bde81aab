/*
 * oracle.c -- CPU restatement (checker) of culip's block-iLDL^T + SQMR path.
 *
 * TEST INFRASTRUCTURE ONLY: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline / reference leg load liboracle.so.  The product
 * library (culip_b200/lib/libculipx.so) never links or calls it.
 *
 * Built by oracle/build.py:  gcc -O2 -ffp-contract=off -fPIC -shared
 * (contraction off: every fma in the restatement is explicit).
 */
#include "oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

/* ---- double instantiation ---- */
#define REAL double
#define SUFFIX _d
#define FMA fma
#define SQRT sqrt
#define FABS fabs
#include "oracle_num.h"
#undef REAL
#undef SUFFIX
#undef FMA
#undef SQRT
#undef FABS
#undef F
#undef CAT
#undef CAT_
#undef NZ_EPS

/* ---- float instantiation ---- */
#define REAL float
#define SUFFIX _s
#define FMA fmaf
#define SQRT sqrtf
#define FABS fabsf
#include "oracle_num.h"

/* ------------------------------------------------------------------------ */
/* CSR SpMV, b = alpha * A x + beta * b (T_csrmv, sparse_la_instances.cu:129-217;
 * the row sum is accumulated in column order) */
void orc_spmv_d(int m, const int *rowptr, const int *colidx, const double *val,
                const double *x, double *y, double alpha, double beta)
{
#pragma omp parallel for schedule(static) if (m > 16384)
    for (int i = 0; i < m; ++i) {
        double acc = 0;
        for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) acc = fma(val[p], x[colidx[p]], acc);
        y[i] = (beta == 0.0) ? alpha * acc : fma(alpha, acc, beta * y[i]);
    }
}

/* ------------------------------------------------------------------------ */
/* preconditioner dispatch used by the SQMR restatement */
typedef struct {
    int kind;                 /* 0 none, 1 block factor, 2 imported LDU */
    const orc_fac_d *fac;
    int sweeps;               /* kind 1: > 0 = block-Jacobi sweeps instead of exact solves */
    int n;
    const int *L_rowptr, *L_colidx;
    const double *L_val, *tri, *scale;
    const int *is_piv, *perm;
    double *t1, *t2;
} prec_t;

static void ldu_apply(const prec_t *P, int stage, const double *b, double *x)
{
    const int n = P->n;
    if (stage == 1) {
        /* ImportLDUPreconditioner::solve_middle -> k_solve_D on a copy */
        memcpy(x, b, sizeof(double) * n);
        for (int g = 0; g < n; ++g) {
            const int this_piv = P->is_piv[g];
            const int next_piv = (g < n - 1) ? P->is_piv[g + 1] : 1;
            const double p11 = P->tri[3 * g + 1], p12 = P->tri[3 * g + 2];
            const double p22 = !next_piv ? P->tri[3 * (g + 1) + 1] : 1.0;
            const double r1 = b[g], r2 = (g < n - 1) ? b[g + 1] : 0.0;
            const double gr = sqrt(fma(p11, p11, p12 * p12));
            const double gc = p11 / gr, gs = p12 / gr;
            double g1 = fma(gc, r1, gs * r2), g2 = fma(gc, r2, -(gs * r1));
            const double tp12 = fma(gc, p12, gs * p22), tp22 = fma(gc, p22, -(gs * p12));
            g2 = g2 / tp22;
            g1 = fma(-tp12, g2, g1) / gr;
            if (this_piv) x[g] = g1;
            if (!next_piv) x[g + 1] = g2;
        }
        return;
    }
    if (stage == 0) {
        /* solve_left: P' (S .* b), then L^-1 (forward substitution) */
        for (int g = 0; g < n; ++g) P->t1[g] = b[g] * P->scale[g];
        for (int g = 0; g < n; ++g) P->t2[g] = P->t1[P->perm[g]];
        for (int i = 0; i < n; ++i) {
            double acc = P->t2[i], diag = 1.0;
            for (int p = P->L_rowptr[i]; p < P->L_rowptr[i + 1]; ++p) {
                const int j = P->L_colidx[p];
                if (j < i) acc = fma(-P->L_val[p], x[j], acc);
                else if (j == i) diag = P->L_val[p];
            }
            x[i] = acc / diag;
        }
    } else {
        /* solve_right: L'^-1 b (column sweep), then S .* (P t) */
        memcpy(P->t1, b, sizeof(double) * n);
        for (int i = n - 1; i >= 0; --i) {
            double diag = 1.0;
            for (int p = P->L_rowptr[i]; p < P->L_rowptr[i + 1]; ++p)
                if (P->L_colidx[p] == i) diag = P->L_val[p];
            const double xi = P->t1[i] / diag;
            P->t1[i] = xi;
            for (int p = P->L_rowptr[i]; p < P->L_rowptr[i + 1]; ++p) {
                const int j = P->L_colidx[p];
                if (j < i) P->t1[j] = fma(-P->L_val[p], xi, P->t1[j]);
            }
        }
        for (int g = 0; g < n; ++g) P->t2[P->perm[g]] = P->t1[g];
        for (int g = 0; g < n; ++g) x[g] = P->t2[g] * P->scale[g];
    }
}

static void prec_apply(const prec_t *P, int stage, const double *b, double *x)
{
    if (P->kind == 1 && P->sweeps > 0) orc_prec_apply_jacobi_d(P->fac, stage, P->sweeps, b, x);
    else if (P->kind == 1) orc_prec_apply_d(P->fac, stage, b, x);
    else if (P->kind == 2) ldu_apply(P, stage, b, x);
    else memcpy(x, b, sizeof(double) * P->n);
}

/* Threads of the loops that are independent per element, per row or per
 * block row of a level (SpMV, vector updates, the level sweeps, D): the
 * results do not depend on the count.  Dot products stay serial (their
 * summation order is part of the restatement). */
void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int orc_get_threads(void) { return omp_get_max_threads(); }

/* a'b summed in DOT_CHUNKS fixed chunks (each in index order, the chunk sums
 * in chunk order): the same roundings for any number of threads */
#define DOT_CHUNKS 64
static double dot(int n, const double *a, const double *b)
{
    double part[DOT_CHUNKS];
    const int len = (n + DOT_CHUNKS - 1) / DOT_CHUNKS;
#pragma omp parallel for schedule(static) if (n > 16384)
    for (int c = 0; c < DOT_CHUNKS; ++c) {
        const int lo = c * len, hi = (lo + len < n) ? lo + len : n;
        double s = 0;
        for (int i = lo; i < hi; ++i) s = fma(a[i], b[i], s);
        part[c] = s;
    }
    double s = 0;
    for (int c = 0; c < DOT_CHUNKS; ++c) s += part[c];
    return s;
}

static double sgn(double v) { return v < 0 ? -1.0 : 1.0; }

/* k_sym_ortho (helper_kernels.impl.cuh:662-700) */
static void sym_ortho(double a, double b, double *c, double *s, double *r)
{
    if (b == 0) { *s = 0; *r = fabs(a); *c = (a == 0) ? 1 : sgn(a); }
    else if (a == 0) { *c = 0; *s = sgn(b); *r = fabs(b); }
    else if (fabs(b) >= fabs(a)) {
        const double tao = a / b;
        *s = sgn(b) / sqrt(fma(tao, tao, 1.0));
        *c = *s * tao;
        *r = b / *s;
    } else {
        const double tao = b / a;
        *c = sgn(a) / sqrt(fma(tao, tao, 1.0));
        *s = *c * tao;
        *r = a / *c;
    }
}

#define ACC(r) (((r) % 3) + (((r) < 0) ? 3 : 0))

/* SQMR::solve (sqmr.impl.cuh:109-355), including the lagged convergence
 * check: flags are copied at iterations = 3 (mod 4) and read at the next
 * iteration, so up to four iterations run after the test first passes. */
static int sqmr_core(int m, const int *rowptr, const int *colidx, const double *val,
                     const prec_t *P, const double *b, double *x, double tol, int max_it,
                     double *residual)
{
    double *v[3], *w[3], *p[3];
    for (int i = 0; i < 3; ++i) {
        v[i] = (double *)calloc(m, sizeof(double));
        w[i] = (double *)calloc(m, sizeof(double));
        p[i] = (double *)calloc(m, sizeof(double));
    }
    double *Av = (double *)calloc(m, sizeof(double));
    double *tmp = (double *)calloc(m, sizeof(double));
    double *ev = (double *)calloc(m, sizeof(double));
    double *ev2 = (double *)calloc(m, sizeof(double));
    double beta[3] = {0, 0, 0}, delta[3] = {0, 0, 0}, c[3] = {0, 0, 0}, s[3] = {0, 0, 0};
    double alpha = 0, norm_A = 0, epsilon = 0, beta_rot = 0, beta_rot_rot = 0, alpha_rot = 0;
    double tau = 0, rho = 0, gamma = 0, norm_pb = 0, norm_x = 0, eta = 0;
    int test0 = 0, test1 = 0, host0 = 0, host1 = 0;
    memset(x, 0, sizeof(double) * m);
    c[ACC(0)] = -1.0;

    prec_apply(P, 0, b, v[0]);
    norm_pb = sqrt(dot(m, v[0], v[0]));
    {
        const double t = 1.0 / norm_pb;
        #pragma omp parallel for schedule(static) if (m > 16384)
        for (int i = 0; i < m; ++i) v[0][i] *= t;
    }
    prec_apply(P, 1, v[0], w[0]);
    eta = sqrt(dot(m, w[0], w[0]));
    eta = 1.0 / eta;
    #pragma omp parallel for schedule(static) if (m > 16384)
    for (int i = 0; i < m; ++i) w[0][i] *= eta;
    gamma = norm_pb;
    prec_apply(P, 1, v[0], tmp);
    prec_apply(P, 2, tmp, ev);
    orc_spmv_d(m, rowptr, colidx, val, ev, ev2, 1.0, 0.0);
    prec_apply(P, 0, ev2, Av);

    int it = 0;
    while (it < max_it) {
        const int k0 = ACC(it), k1 = ACC(it + 1), km1 = ACC(it - 1), km2 = ACC(it - 2);
        prec_apply(P, 1, Av, tmp);
        alpha = dot(m, v[k0], tmp);
        prec_apply(P, 1, v[k0], tmp);
        double t = dot(m, v[k0], tmp);
        alpha = alpha / t;
#pragma omp parallel for schedule(static) if (m > 16384)
        for (int i = 0; i < m; ++i) {
            double vi = Av[i];
            vi = fma(-alpha, v[k0][i], vi);
            vi = fma(-beta[k0], v[km1][i], vi);
            v[k1][i] = vi;
        }
        delta[k1] = sqrt(dot(m, v[k1], v[k1]));
        t = 1.0 / delta[k1];
        #pragma omp parallel for schedule(static) if (m > 16384)
        for (int i = 0; i < m; ++i) v[k1][i] *= t;
        prec_apply(P, 1, v[k1], w[k1]);
        t = eta * delta[k1];
#pragma omp parallel for schedule(static) if (m > 16384)
        for (int i = 0; i < m; ++i) w[k1][i] *= t;
        prec_apply(P, 1, v[k1], tmp);
        prec_apply(P, 2, tmp, ev);
        orc_spmv_d(m, rowptr, colidx, val, ev, ev2, 1.0, 0.0);
        prec_apply(P, 0, ev2, Av);
        beta[k1] = dot(m, w[k0], Av);
        t = dot(m, w[k0], v[k0]);
        beta[k1] = beta[k1] / t;
        t = 1.0 / beta[k1];
#pragma omp parallel for schedule(static) if (m > 16384)
        for (int i = 0; i < m; ++i) w[k1][i] *= t;
        t = delta[k1] / beta[k1];
        eta = t * eta;
        t = sqrt(fma(delta[k1], delta[k1], fma(alpha, alpha, beta[k0] * beta[k0])));
        norm_A = (norm_A > t) ? norm_A : t;
        epsilon = s[km1] * beta[k0];
        beta_rot = (-c[km1]) * beta[k0];
        beta_rot_rot = fma(c[k0], beta_rot, s[k0] * alpha);
        alpha_rot = fma(s[k0], beta_rot, (-c[k0]) * alpha);
        sym_ortho(alpha_rot, delta[k1], &c[k1], &s[k1], &rho);
        tau = c[k1] * gamma;
#pragma omp parallel for schedule(static) if (m > 16384)
        for (int i = 0; i < m; ++i) {
            double pi = v[k0][i];
            pi = fma(-beta_rot_rot, p[km1][i], pi);
            pi = fma(-epsilon, p[km2][i], pi);
            p[k0][i] = pi * (1.0 / rho);
        }
        #pragma omp parallel for schedule(static) if (m > 16384)
        for (int i = 0; i < m; ++i) x[i] = fma(tau, p[k0][i], x[i]);
        norm_x = sqrt(dot(m, x, x));
        gamma = s[k1] * gamma;
        test0 |= (fabs(delta[k1]) <= tol);
        test1 |= (gamma / fma(norm_A, norm_x, norm_pb) <= tol);
        if (it > 0 && (it % 4) == 0) {
            if (host0 || host1) break;
        } else if (((it + 1) % 4) == 0) {
            host0 = test0; host1 = test1;
        }
        ++it;
    }
    *residual = gamma / norm_pb;
    memcpy(Av, x, sizeof(double) * m);
    prec_apply(P, 1, Av, tmp);
    prec_apply(P, 2, tmp, x);

    for (int i = 0; i < 3; ++i) { free(v[i]); free(w[i]); free(p[i]); }
    free(Av); free(tmp); free(ev); free(ev2);
    return it;
}

int orc_sqmr_d(int m, const int *rowptr, const int *colidx, const double *val,
               const orc_fac_d *f, const double *b, double *x, double tol, int max_it,
               double *residual)
{
    prec_t P;
    memset(&P, 0, sizeof(P));
    P.kind = f ? 1 : 0;
    P.fac = f;
    P.n = m;
    return sqmr_core(m, rowptr, colidx, val, &P, b, x, tol, max_it, residual);
}

int orc_sqmr_jacobi_d(int m, const int *rowptr, const int *colidx, const double *val, const orc_fac_d *f,
                      int sweeps, const double *b, double *x, double tol, int max_it, double *residual)
{
    prec_t P;
    memset(&P, 0, sizeof(P));
    P.kind = 1;
    P.fac = f;
    P.sweeps = sweeps;
    P.n = m;
    return sqmr_core(m, rowptr, colidx, val, &P, b, x, tol, max_it, residual);
}

void orc_ldu_apply_d(int n, const int *L_rowptr, const int *L_colidx, const double *L_val, const double *tri,
                     const int *is_piv, const int *perm, const double *scale, int stage, const double *b, double *x)
{
    prec_t P;
    memset(&P, 0, sizeof(P));
    P.kind = 2;
    P.n = n;
    P.L_rowptr = L_rowptr; P.L_colidx = L_colidx; P.L_val = L_val;
    P.tri = tri; P.is_piv = is_piv; P.perm = perm; P.scale = scale;
    P.t1 = (double *)calloc(n, sizeof(double));
    P.t2 = (double *)calloc(n, sizeof(double));
    ldu_apply(&P, stage, b, x);
    free(P.t1); free(P.t2);
}

int orc_sqmr_ldu_d(int m, const int *rowptr, const int *colidx, const double *val,
                   const int *L_rowptr, const int *L_colidx, const double *L_val,
                   const double *tri, const int *is_piv, const int *perm, const double *scale,
                   const double *b, double *x, double tol, int max_it, double *residual)
{
    prec_t P;
    memset(&P, 0, sizeof(P));
    P.kind = 2;
    P.n = m;
    P.L_rowptr = L_rowptr; P.L_colidx = L_colidx; P.L_val = L_val;
    P.tri = tri; P.is_piv = is_piv; P.perm = perm; P.scale = scale;
    P.t1 = (double *)calloc(m, sizeof(double));
    P.t2 = (double *)calloc(m, sizeof(double));
    const int it = sqmr_core(m, rowptr, colidx, val, &P, b, x, tol, max_it, residual);
    free(P.t1); free(P.t2);
    return it;
}
