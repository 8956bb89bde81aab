/*
 * oracle.h -- CPU restatement (checker) of culip's block-iLDL^T + SQMR solve
 * path.  TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg; never by the product library.
 */
#ifndef CULIPX_ORACLE_H
#define CULIPX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_SPARSE = 0, ORC_DENSE = 1 };      /* BLOCK_FORMAT, block_ildlt.cuh:17-21 */
enum { ORC_PIV_STATIC = 0, ORC_PIV_BK = 1, ORC_PIV_ROOK = 2 };

typedef struct orc_sym {
    int n, nnz;              /* fine order, nnz of the full symmetric CSR */
    int value_bytes;         /* 8 (double) or 4 (float): drives the format rule */
    int num_blocks;          /* coarse_m */
    int *bs;                 /* block_starts[num_blocks + 1] */
    int *row_block;          /* fine row -> block row */
    int coarse_nnz, fill_nnz;
    int *cs_off, *cs_col;    /* coarse CSR, sorted; block id = position */
    int *blk_nnzA;           /* A entries (upper part) per block */
    int *csc_off, *csc_blk;  /* block ids per block column, rows ascending */
    int num_levels, unleveled_rows;
    int *lvl_off, *lvl_rows, *row_level;
    int max_level_size, max_level_blocks;
    int lb_count;
    int *lb_off, *lb;        /* factor order: per level pivots then off-diag */
    int *sb_off, *sb;        /* U' sweep order: per column level */
    int *blk_row, *blk_col, *fmt, *max_nnz;
    int *a_blk, *a_idx;      /* per CSR entry: block and local index (-1: lower) */
} orc_sym;

orc_sym *orc_symbolic(int n, const int *rowptr, const int *colidx,
                      int num_blocks, const int *block_starts,
                      int fill_level, double fill_factor, int value_bytes);
void orc_sym_free(orc_sym *s);

/* numeric factorization, double and float instantiations */
typedef struct orc_fac_d orc_fac_d;
typedef struct orc_fac_s orc_fac_s;

orc_fac_d *orc_factor_d(const orc_sym *s, const double *vals, const int *is_piv_init,
                        int pivot, double threshold, int literal);
orc_fac_s *orc_factor_s(const orc_sym *s, const float *vals, const int *is_piv_init,
                        int pivot, float threshold, int literal);
/* the same with each outgrowing block's extra slots given (coarse_nnz ints,
 * or NULL for the pool) and the FP32 factor's FP64 2x2-pivot bound (the
 * plain entry points use ORC_PIVOT_FP64_DEFAULT; 0 = float throughout) */
#define ORC_PIVOT_FP64_DEFAULT 1e-3
orc_fac_d *orc_factor_forced_d(const orc_sym *s, const double *vals, const int *is_piv_init,
                               int pivot, double threshold, int literal, const int *forced_grants,
                               double piv64);
orc_fac_s *orc_factor_forced_s(const orc_sym *s, const float *vals, const int *is_piv_init,
                               int pivot, float threshold, int literal, const int *forced_grants,
                               double piv64);
void orc_fac_free_d(orc_fac_d *f);
void orc_fac_free_s(orc_fac_s *f);

/* export: sizes then flat arrays (blocks in block-id order; sparse entries
 * sorted by local index, dense blocks as all r*c entries) */
long orc_fac_export_size_d(const orc_fac_d *f);
long orc_fac_export_size_s(const orc_fac_s *f);
void orc_fac_export_d(const orc_fac_d *f, int *blk_nnz, long *blk_off, int *idx, double *val,
                      double *tri, int *is_piv, int *perm, int *got_extra);
void orc_fac_export_s(const orc_fac_s *f, int *blk_nnz, long *blk_off, int *idx, float *val,
                      float *tri, int *is_piv, int *perm, int *got_extra);

/* preconditioner applies: stage 0 = left (P' then U'), 1 = middle (D),
 * 2 = right (U then P) */
void orc_prec_apply_d(const orc_fac_d *f, int stage, const double *b, double *x);
void orc_prec_apply_s(const orc_fac_s *f, int stage, const float *b, float *x);
void orc_prec_apply_jacobi_d(const orc_fac_d *f, int stage, int sweeps, const double *b, double *x);
void orc_prec_apply_jacobi_s(const orc_fac_s *f, int stage, int sweeps, const float *b, float *x);
int orc_sqmr_jacobi_d(int m, const int *rowptr, const int *colidx, const double *val, const orc_fac_d *f,
                      int sweeps, const double *b, double *x, double tol, int max_it, double *residual);

/* y = alpha * A x + beta * y (beta == 0: y is not read) */
/* ImportLDUPreconditioner's solve_left (0) / middle (1) / right (2) */
void orc_ldu_apply_d(int n, const int *L_rowptr, const int *L_colidx, const double *L_val, const double *tri,
                     const int *is_piv, const int *perm, const double *scale, int stage, const double *b, double *x);

/* threads of the row-independent loops (results do not depend on it) */
void orc_set_threads(int n);
int orc_get_threads(void);

void orc_spmv_d(int m, const int *rowptr, const int *colidx, const double *val,
                const double *x, double *y, double alpha, double beta);

/* SQMR (sqmr.impl.cuh:109-355) with the factor as split preconditioner
 * (f may be NULL: no preconditioner).  Returns iterations. */
int orc_sqmr_d(int m, const int *rowptr, const int *colidx, const double *val,
               const orc_fac_d *f, const double *b, double *x, double tol, int max_it,
               double *residual);

/* SQMR with an imported L D L' preconditioner
 * (import_ldu_preconditioner.impl.cuh; used by tests/la/test_sqmr.cc). */
int orc_sqmr_ldu_d(int m, const int *rowptr, const int *colidx, const double *val,
                   const int *L_rowptr, const int *L_colidx, const double *L_val,
                   const double *tri, const int *is_piv, const int *perm, const double *scale,
                   const double *b, double *x, double tol, int max_it, double *residual);

#ifdef __cplusplus
}
#endif
#endif
