/*
 * culipx.h -- C ABI of the B200-native block-iLDL^T + SQMR KKT solve path.
 *
 * This boundary replaces the parts of culip's libs/la module that the
 * apps/block_ildlt driver calls (paths relative to the culip repository):
 *
 *   gpu_handle_t                 libs/utils/types.cuh:441-482, types.cu:343-430
 *   BlockiLDLt<T, BK, Rook>      libs/la/preconditioner/block_ildlt.cuh:188-401
 *     ctor + compute()           libs/la/preconditioner/block_ildlt.impl.cuh:44-146
 *     solve_analysis()           libs/la/preconditioner/block_ildlt.impl.cuh:1924-2150
 *     solve_left/middle/right    libs/la/preconditioner/block_ildlt.impl.cuh:183-246
 *     export_factorized()        libs/la/preconditioner/block_ildlt.impl.cuh:1700-1916
 *   CSRMatrixSPMV<T>             libs/la/spmv.cuh:19-66, spmv.impl.cuh:29-113
 *   SQMR<T>                      libs/la/iterative_solvers/sqmr.cuh:29-79,
 *                                sqmr.impl.cuh:109-369
 *
 * Conventions: every entry point returns a culipx status (0 = OK) instead of
 * raising SIGSEGV as the reference's CHECK_CUDA does (libs/utils/types.cuh:32);
 * culipx_last_error() describes the last failure of the calling thread.
 * Pointers named d_* are device pointers on the handle's device, h_* host
 * pointers.  Indices are 0-based int32 as the reference's mat_int_t
 * (libs/utils/defines.h:56-63).  Work is issued on the handle's stream.
 */
#ifndef CULIPX_H
#define CULIPX_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define CULIPX_OK            0
#define CULIPX_INVALID_ARG   1
#define CULIPX_OOM           2  /* device-memory budget or cudaMalloc exhausted */
#define CULIPX_BREAKDOWN     3  /* SQMR breakdown (division by zero / non-finite) */
#define CULIPX_MAXIT         4  /* SQMR hit max_it without passing its test */
#define CULIPX_TIMEOUT       5  /* a bounded device wait gave up */
#define CULIPX_CUDA_ERROR    6
#define CULIPX_NOT_SUPPORTED 7
#define CULIPX_PENDING       8  /* a server request has not finished yet */
#define CULIPX_STALLED       9  /* refinement: corrections stopped lowering the
                                   true residual; x is the best iterate reached */

/* ---- value precision (the reference's T = double / float) ---- */
#define CULIPX_F64 0
#define CULIPX_F32 1

/* ---- pivot method, as the driver's argument (apps/block_ildlt/block_ildlt.cc:33-35) ---- */
#define CULIPX_PIV_STATIC 0
#define CULIPX_PIV_BK     1
#define CULIPX_PIV_ROOK   2

/* ---- triangular-solve algorithm (SOLVE_ALGORITHM, libs/la/preconditioner/block_ildlt.cuh:24-30) ----
 * STRIPE, BLOCK and SCALAR are the reference's three schedules of the same
 * exact block triangular solves; here all three run the level-scheduled
 * sweeps.  JACOBI replaces each triangular solve by a number of block-Jacobi
 * sweeps from x = 0 (solve_U_jacobi / solve_Ut_jacobi, block_ildlt.impl.cuh:2455-2494). */
#define CULIPX_SOLVE_STRIPE 0
#define CULIPX_SOLVE_BLOCK  1
#define CULIPX_SOLVE_SCALAR 2
#define CULIPX_SOLVE_JACOBI 3

/* ---- preconditioner stage (Preconditioner<T>, libs/la/preconditioner.cuh:18-40) ---- */
#define CULIPX_LEFT   0   /* x = U'^-1 P' b   (solve_left)   */
#define CULIPX_MIDDLE 1   /* x = D^-1 b       (solve_middle) */
#define CULIPX_RIGHT  2   /* x = P U^-1 b     (solve_right)  */

typedef struct culipx_handle_t  *culipx_handle;
typedef struct culipx_pattern_t *culipx_pattern;
typedef struct culipx_factor_t  *culipx_factor;
typedef struct culipx_csr_t     *culipx_csr;

const char *culipx_last_error(void);
int culipx_version(void);

/* ------------------------------------------------------------------------ */
/* Seeded synthetic KKT systems (no counterpart in the reference, which reads
 * its inputs from files: apps/block_ildlt/block_ildlt.cc:29-35).           */
typedef struct culipx_kkt_spec {
    int n, m;             /* H is n x n, A is m x n; K has order n + m      */
    int nnz_per_col;      /* distinct nonzeros per column of A              */
    int band_half;        /* > 0: half of each column within +-band_half of floor(j m / n) */
    double hmin, hmax;    /* H diagonal, log-uniform                         */
    double delta, gamma;  /* K = [[H + delta I, A'], [A, -gamma I]]          */
    unsigned long long seed;
} culipx_kkt_spec;

int culipx_kkt_nnz(const culipx_kkt_spec *spec, long long *nnz_out);
/* full symmetric CSR with sorted columns and an explicit diagonal */
int culipx_kkt_generate(const culipx_kkt_spec *spec, int *h_rowptr, int *h_colidx, double *h_val);
/* contiguous blocking that never straddles row n; block_starts gets
 * num_blocks + 1 entries (NULL: only count) */
int culipx_kkt_blocking(int n, int m, int block, int *h_block_starts, int capacity, int *num_blocks);

/* Blocking generator for any symmetric pattern (host CSR, sorted columns; no
 * counterpart in the reference, whose driver reads the blocking from a file
 * it does not create, apps/block_ildlt/block_ildlt.cc:29-35; same output
 * contract: first rows of the blocks, then n).  Contiguous blocks of at most
 * max_size (<= 32) rows: runs of consecutive rows with equal column sets stay
 * together, a block closes once it holds min_size rows at the first run not
 * coupled to it, and a short last block is merged or split evenly with its
 * predecessor.  With h_block_starts NULL only num_blocks is returned. */
int culipx_blocking_generate(int n, const int *h_rowptr, const int *h_colidx, int min_size, int max_size,
                             int *h_block_starts, int capacity, int *num_blocks);
int culipx_normal_vector(unsigned long long seed, long long len, double *h_out);

/* ------------------------------------------------------------------------ */
/* Handle: device, stream, device-memory budget (replaces gpu_handle_t).    */
/* device = -1: host-only handle (symbolic analysis only, no CUDA calls) */
int culipx_handle_create(culipx_handle *out, int device, void *cuda_stream);
int culipx_handle_destroy(culipx_handle h);
int culipx_handle_set_stream(culipx_handle h, void *cuda_stream);
/* cap on the device bytes this handle's objects may hold (<= 0: unlimited) */
int culipx_handle_set_memory_budget(culipx_handle h, long long bytes);
int culipx_handle_memory_used(culipx_handle h, long long *bytes);
int culipx_handle_synchronize(culipx_handle h);
/* kernels this handle's objects launched (optionally reset to 0) */
int culipx_handle_launch_count(culipx_handle h, long long *count, int reset);

/* ------------------------------------------------------------------------ */
/* Symbolic analysis of one sparsity pattern (host; cacheable across IPM
 * iterations).  Replaces the BlockiLDLt constructor and the symbolic half of
 * compute(): build_initial_coarse, determine_coarse_level_fill_and_diag,
 * build_block_csc, find_level_sets, build_blocks
 * (libs/la/preconditioner/block_ildlt.impl.cuh:352-1280) and
 * solve_analysis_block (:2050-2150).
 *   h_rowptr/h_colidx : full symmetric CSR of K (n x n), sorted columns
 *   h_block_starts    : num_blocks entries (first row of each block), as the
 *                       reference's constructor; n is appended internally
 *   fill_level        : block level of fill (>= 0)
 *   fill_factor       : >= 1, fine fill allowed inside a block
 *   precision         : CULIPX_F64 / CULIPX_F32 (enters the block-format rule) */
int culipx_pattern_analyze(culipx_handle h, int n, const int *h_rowptr, const int *h_colidx,
                           int num_blocks, const int *h_block_starts, int fill_level,
                           double fill_factor, int precision, culipx_pattern *out);
/* The same for a block-diagonal union of independent systems (rows
 * h_row_offsets[k] .. h_row_offsets[k + 1], each on block boundaries): the
 * reference's rule that the last 10 % of block rows keep dense blocks
 * (build_blocks, block_ildlt.impl.cuh:1015-1280) is applied per system, so
 * block formats equal those of the separate analyses.  For culipx_batch_*. */
int culipx_pattern_analyze_systems(culipx_handle h, int n, const int *h_rowptr, const int *h_colidx,
                                   int num_blocks, const int *h_block_starts, int fill_level,
                                   double fill_factor, int precision, int num_systems,
                                   const int *h_row_offsets, culipx_pattern *out);
int culipx_pattern_destroy(culipx_pattern p);
/* info[0..15]: n, nnz, num_blocks, coarse_nnz, fill_nnz, num_levels, num_sparse,
 * num_dense, val_slots, idx_slots, max_level_blocks, max_level_rows,
 * device_bytes, precision, 0, 0 */
int culipx_pattern_info(culipx_pattern p, long long *info16);
/* canonical symbolic output for parity checks (host arrays sized by info):
 * coarse CSR (num_blocks+1, coarse_nnz), A nnz per block, level offsets
 * (num_levels+1) and rows (num_blocks, ascending per level), factor-order
 * block lists (num_levels+1, coarse_nnz), U'-sweep block lists (same),
 * format (0 sparse, 1 dense) and max_nnz per block.  Any pointer may be NULL. */
int culipx_pattern_export(culipx_pattern p, int *coarse_off, int *coarse_col, int *blk_nnzA,
                          int *lvl_off, int *lvl_rows, int *lb_off, int *lb, int *sb_off,
                          int *sb, int *fmt, int *max_nnz);

/* ------------------------------------------------------------------------ */
/* Numeric factorization (device).  Replaces BlockiLDLt::factorize
 * (block_ildlt.impl.cuh:1519-1671) and the kernels it launches.            */
int culipx_factor_create(culipx_pattern p, culipx_factor *out);
int culipx_factor_destroy(culipx_factor f);
/* d_vals: K's values in the pattern's CSR order, in the pattern's precision.
 * h_is_piv: n flags (1 = a pivot starts at this row), NULL = all ones; used
 * as given by CULIPX_PIV_STATIC and overwritten by BK / Rook.
 * threshold: relative dropping threshold (>= 0). */
int culipx_factor_compute(culipx_factor f, const void *d_vals, const int *h_is_piv, int pivot,
                          double threshold);
/* culipx_factor_compute (is_piv NULL) replayed from a CUDA graph; no
 * counterpart in the reference, which launches the factorization's kernels
 * one by one.  The first call for a given values pointer, pivot method and
 * threshold factors normally once, then captures the same launch sequence on
 * the handle's stream (which must not be capturing already); later calls with
 * that pointer launch the graph, one launch for the whole factorization, and
 * read whatever values the pointer then holds.  Another pointer, pivot or
 * threshold captures anew. */
int culipx_factor_compute_graph(culipx_factor f, const void *d_vals, int pivot, double threshold);
/* same, with K's values (double) in host memory; converts to the pattern's precision */
int culipx_factor_compute_host(culipx_factor f, const double *h_vals, const int *h_is_piv,
                               int pivot, double threshold);
/* factor export for parity (export_factorized, block_ildlt.impl.cuh:1700-1916):
 * total entry count, then per block (block-id order) nnz, offsets
 * (coarse_nnz + 1), entries (sparse: sorted local index row * width + col;
 * dense: all r * c entries row-major), D as tridiagonal[3n], is_piv[n],
 * permutation[n] and the extra slots granted by dual dropping.  Values are in
 * the pattern's precision. */
int culipx_factor_export_size(culipx_factor f, long long *entries);
int culipx_factor_export(culipx_factor f, int *h_blk_nnz, long long *h_blk_off, int *h_idx,
                         void *h_val, void *h_tri, int *h_is_piv, int *h_perm, int *h_got_extra);
/* timing of the last culipx_factor_compute on the device (ms), and launches */
int culipx_factor_stats(culipx_factor f, double *ms, int *launches);
/* sizes of the last computed factor's solve structures (no counterpart in
 * the reference; used for algorithmic-byte counts): info[0] stored strictly
 * off-diagonal entries of U, [1] block rows with a non-identity pivot tile,
 * [2] upper-triangle entries of those tiles, [3] fine rows of simple block
 * rows (identity tile, no swaps, 1x1 pivots), [4] block rows with a 2x2
 * pivot, [5] bytes per value, [6] blocks that drew extra capacity from the
 * dual-dropping pass's leftover pool (got_extra > 0), [7] 0 */
int culipx_factor_info(culipx_factor f, long long *info8);

/* set_solve_algorithm (block_ildlt.impl.cuh:253-258): algorithm one of
 * CULIPX_SOLVE_*, sweeps (>= 0) used by CULIPX_SOLVE_JACOBI.  Applies and
 * culipx_sqmr_solve follow it; SQMR with JACOBI needs an FP64 factor. */
int culipx_factor_set_solve_algorithm(culipx_factor f, int algorithm, int sweeps);

/* FP32 factors (no counterpart in the reference, whose float factor inverts
 * every pivot in float): a 2x2 pivot whose ratio
 * |d11 d22 - d12^2| / (|d11 d22| + d12^2) is below bound is inverted in FP64,
 * in the pivot-tile step (d_ldlt_2x2_step), the off-diagonal solve
 * (d_left_solve_with_D_Ut) and the D apply (k_solve_D); results are rounded
 * to FP32 once.  Default 1e-3; 0 keeps the reference's FP32 arithmetic.
 * Bunch-Kaufman and rook pivots have a ratio above 0.42, so the bound acts on
 * given (static) pivots.  No effect on FP64 factors; the next compute uses it. */
int culipx_factor_set_pivot_fp64(culipx_factor f, double bound);

/* Preconditioner applies; b and x are device vectors of n values in the
 * factor's precision (b == x allowed for MIDDLE). */
int culipx_prec_apply(culipx_factor f, int stage, const void *d_b, void *d_x);

/* ------------------------------------------------------------------------ */
/* Orderings (host functions; no handle, no device).
 * culipx_sprank replaces culip's sprank (libs/algorithms/sprank.cuh, an
 * UnweightedBipartiteMatching, libs/algorithms/matching.cuh:18-62): the
 * structural rank of the m x n CSR pattern by a maximum matching of rows to
 * columns; row_match[i] = the column matched to row i, col_match[j] = the row
 * matched to column j, INT_MAX where unmatched (either may be NULL).  Any
 * maximum matching may be returned; the rank is unique.
 * culipx_ordering_rcm (no counterpart in the reference, whose driver reads its
 * permutation from a file): reverse Cuthill-McKee of the symmetrized n x n
 * pattern, deterministic; perm[new] = old, i.e. pass perm_is_old_to_new = 0 to
 * culipx_permute_create. */
int culipx_sprank(int m, int n, const int *rowptr, const int *colidx, int *row_match, int *col_match, int *rank);
int culipx_ordering_rcm(int n, const int *rowptr, const int *colidx, int *perm);

/* ------------------------------------------------------------------------ */
/* KKT assembly for an interior-point iteration (no counterpart in culip's
 * libs/la, whose IPM caller forms K on the host): the explicit
 *   K = [[diag(d) + delta I, A'], [A, -gamma I]],  d_j = s_j / x_j
 * (the LP barrier Hessian X^-1 S; or d given directly), i.e. the matrix of
 * AugmentedMatrixSPMV<T> (libs/la/spmv.cuh:104-149) with the dual shift on
 * every row, as full symmetric CSR with sorted columns and an explicit
 * diagonal (N = n + m rows, nnz_K = 2 nnz_A + N).  create() plans K's
 * structure once per pattern of A (m x n CSR on the device, rows sorted, no
 * duplicates; invalid structure is rejected with CULIPX_INVALID_ARG);
 * assemble() writes one iteration's values with one gather on the handle's
 * stream (precision CULIPX_F64 or CULIPX_F32 output).  Pass d_d = NULL to
 * use x and s (all n entries > 0), else d_x / d_s may be NULL. */
typedef struct culipx_kkt_assembly_t *culipx_kkt_assembly;
int culipx_kkt_assembly_create(culipx_handle h, int m, int n, long long nnz_a, const int *d_rowptr,
                               const int *d_colidx, culipx_kkt_assembly *out);
int culipx_kkt_assembly_destroy(culipx_kkt_assembly K);
/* K's size and its device structure (owned by the plan) */
int culipx_kkt_assembly_size(culipx_kkt_assembly K, int *N, long long *nnz_k);
int culipx_kkt_assembly_structure(culipx_kkt_assembly K, const int **d_rowptr, const int **d_colidx);
/* K's structure copied to host arrays of N + 1 and nnz_k ints (culipx_pattern_analyze's input) */
int culipx_kkt_assembly_export(culipx_kkt_assembly K, int *h_rowptr, int *h_colidx);
int culipx_kkt_assemble(culipx_kkt_assembly K, const double *d_aval, const double *d_x, const double *d_s,
                        const double *d_d, double delta, double gamma, int precision, void *d_kval);

/* ------------------------------------------------------------------------ */
/* Permutation and scaling of K before the factorization: B = diag(1/r)
 * P_r K P_c' diag(1/c) with sorted rows and columns, as T_matrix_permute_scale
 * (libs/la/sparse_la.impl.cuh:599-657) called by the driver's host_permute
 * (apps/block_ildlt/block_ildlt_invariants.h:31-69).  The plan holds B's
 * structure and is built once per pattern; apply() maps each new set of
 * values with one gather.
 *   h_row_perm / h_col_perm : n entries each (h_col_perm NULL = h_row_perm);
 *     old -> new if perm_is_old_to_new, else new -> old (inverted first, as
 *     the reference's k_inv_perm)
 *   d_row_scale / d_col_scale : NULL for unit scaling, else both given; B's
 *     value is a / (r * c) with r, c taken at the old (row, column) when
 *     scale_before_match, else at the new ones.
 * d_rowptr / d_colidx are read during create only. */
typedef struct culipx_permute_t *culipx_permute;
int culipx_permute_create(culipx_handle h, int n, long long nnz, const int *d_rowptr, const int *d_colidx,
                          const int *h_row_perm, const int *h_col_perm, int perm_is_old_to_new,
                          culipx_permute *out);
int culipx_permute_destroy(culipx_permute p);
/* B's row offsets (n + 1) and columns (nnz), device arrays owned by the plan */
int culipx_permute_structure(culipx_permute p, const int **d_rowptr, const int **d_colidx);
/* the same copied to host arrays (n + 1 and nnz entries) */
int culipx_permute_export(culipx_permute p, int *h_rowptr, int *h_colidx);
int culipx_permute_apply(culipx_permute p, int precision, const void *d_val, const void *d_row_scale,
                         const void *d_col_scale, int scale_before_match, void *d_out);

/* ------------------------------------------------------------------------ */
/* CSR operator (CSRMatrixSPMV<T>).  Device arrays are borrowed, not copied:
 * they must outlive the operator, as the reference's raw pointer does. */
int culipx_csr_create(culipx_handle h, int m, int n, long long nnz, const int *d_rowptr,
                      const int *d_colidx, const void *d_val, int precision,
                      int explicit_transpose, culipx_csr *out);
int culipx_csr_destroy(culipx_csr A);
/* y = alpha op(A) x + beta y (beta == 0: y is not read) */
int culipx_spmv(culipx_csr A, const void *d_x, void *d_y, double alpha, double beta, int transpose);
/* Storage the non-transposed product reads (no counterpart in the
 * reference, which hands the CSR arrays to cuSPARSE each call).
 * CULIPX_FMT_CSR (default): the borrowed arrays.  CULIPX_FMT_SELL: a
 * SELL-32-sigma copy built now (rows of up to 64 entries in slices of 32,
 * sorted by length inside windows of 256 rows, entry j of a slice's rows
 * contiguous), so a warp's index and value loads coalesce; every row is
 * still summed serially in column order, so y is bit for bit the CSR
 * kernel's.  The copy holds the values of the time it was built: after
 * changing d_val call culipx_csr_refresh (one gather on the stream). */
#define CULIPX_FMT_CSR  0
#define CULIPX_FMT_SELL 1
int culipx_csr_set_format(culipx_csr A, int format);
int culipx_csr_refresh(culipx_csr A);

/* ------------------------------------------------------------------------ */
/* Vector operations on device vectors of n values in `precision`, on the
 * handle's stream: the BLAS-1 helpers T_doti / T_nrm2 / T_axpy / T_scal of
 * libs/la/dense_la.cuh:35-85 (cuBLAS calls there).  Reductions sum in FP64 in
 * a fixed order (deterministic) and return their result to host memory,
 * synchronizing the stream.  culipx_vec_convert copies between FP64 and FP32
 * (no counterpart; the class facade uses it for SQMR<float>). */
int culipx_vec_dot(culipx_handle h, int precision, long long n, const void *d_x, const void *d_y,
                   double *h_result);
int culipx_vec_nrm2(culipx_handle h, int precision, long long n, const void *d_x, double *h_result);
int culipx_vec_axpy(culipx_handle h, int precision, long long n, double alpha, const void *d_x, void *d_y);
int culipx_vec_scal(culipx_handle h, int precision, long long n, double alpha, void *d_x);
int culipx_vec_convert(culipx_handle h, long long n, int src_precision, const void *d_src, int dst_precision,
                       void *d_dst);

/* ------------------------------------------------------------------------ */
/* SQMR with the factor as split preconditioner M = (P U') D (U P')
 * (SQMR<double>::solve, sqmr.impl.cuh:109-355).  A must be FP64; M may be
 * FP64, FP32 (mixed precision: applies in FP32, recurrence in FP64) or NULL.
 * x is overwritten.  residual = the quasi-residual gamma / ||M_L^-1 b||, as
 * the reference returns; iterations as the reference counts them. */
int culipx_sqmr_solve(culipx_handle h, culipx_csr A, culipx_factor M, const double *d_b,
                      double *d_x, double tol, int max_it, double *residual, int *iterations);

/* Batched solves of independent systems (no counterpart in the reference,
 * which solves one system per SQMR object).  The systems are stored as one
 * block-diagonal union: consecutive row ranges h_row_offsets[k] ..
 * h_row_offsets[k + 1] of one pattern / factor / CSR / b / x, each range a
 * whole number of block rows and no block coupling two ranges (checked).
 * One launch solves them all, each system by one CTA with its own SQMR
 * scalars and stopping test (tol, max_it as culipx_sqmr_solve); a system's
 * result does not depend on which other systems share the batch.  Per
 * system: h_residual (gamma / ||M_L^-1 b||), h_iterations, h_status (OK,
 * MAXIT or BREAKDOWN); any of the three may be NULL.  The factor of a union
 * equals the systems' separate factors when no block draws extra capacity
 * from the dual-dropping pass's leftover pool, which is one pool per
 * factorization as in the reference (culipx_factor_info[6] == 0; always the
 * case at level-0 fill of natural-order KKT systems, whose off-diagonal
 * blocks keep K's pattern). */
typedef struct culipx_batch_t *culipx_batch;
int culipx_batch_create(culipx_pattern p, int num_systems, const int *h_row_offsets, culipx_batch *out);
int culipx_batch_destroy(culipx_batch b);
int culipx_batch_sqmr_solve(culipx_batch b, culipx_csr A, culipx_factor M, const double *d_b, double *d_x,
                            double tol, int max_it, double *h_residual, int *h_iterations, int *h_status);
/* The numeric factorization of the batch's union (values d_vals, in M's
 * precision) and the batched SQMR solve of all its systems as ONE CUDA-graph
 * launch (no counterpart in the reference).  The first call for a set of
 * buffers (d_vals, A, M, d_b, d_x) and settings runs both as ordinary launches,
 * which sizes every buffer (the batch keeps its own solver workspace), and
 * captures them; later calls replay the graph, so the buffers' contents may
 * change between calls but not their addresses.  Results as
 * culipx_batch_sqmr_solve. */
int culipx_batch_factor_solve_graph(culipx_batch b, culipx_csr A, culipx_factor M, const void *d_vals, int pivot,
                                    double threshold, const double *d_b, double *d_x, double tol, int max_it,
                                    double *h_residual, int *h_iterations, int *h_status);

/* Several right-hand sides of one system (no counterpart in the reference,
 * whose SQMR takes one): d_B and d_X are n x nrhs column-major.  Up to four
 * right-hand sides share one launch, in which every work item reads the
 * factor and K once for all of them; each has its own SQMR scalars and
 * stopping test (tol, max_it as culipx_sqmr_solve) and its x is final once
 * it stops.  Per right-hand side: quasi-residual, iterations, status (OK,
 * MAXIT, BREAKDOWN); any of the three may be NULL. */
int culipx_sqmr_solve_multi(culipx_handle h, culipx_csr A, culipx_factor M, int nrhs, const double *d_B,
                            double *d_X, double tol, int max_it, double *h_residual, int *h_iterations,
                            int *h_status);

/* culipx_sqmr_refine for several right-hand sides (d_B, d_X n x nrhs
 * column-major): per right-hand side its own true residual, corrections and
 * stopping test; every step solves the corrections of the right-hand sides
 * still above tol together (culipx_sqmr_solve_multi).  Per right-hand side:
 * relres = ||b - K x|| / ||b||, SQMR iterations summed, corrections, status
 * (OK, MAXIT, STALLED, BREAKDOWN), each as culipx_sqmr_refine defines them;
 * any output array may be NULL. */
int culipx_sqmr_refine_multi(culipx_handle h, culipx_csr A, culipx_factor M, int nrhs, const double *d_B,
                             double *d_X, double tol, double inner_tol, int inner_max_it, int max_refine,
                             double *h_relres, int *h_iterations, int *h_steps, int *h_status);

/* Many independent systems, each with its own pattern, factor, matrix and
 * vectors (no union), solved in one launch, one CTA per system; all factors
 * of one call share a precision.  Same per-system outputs as
 * culipx_batch_sqmr_solve.  No counterpart in the reference. */
int culipx_sqmr_solve_many(culipx_handle h, int num, const culipx_csr *A, const culipx_factor *M,
                           const double *const *d_b, double *const *d_x, double tol, int max_it,
                           double *h_residual, int *h_iterations, int *h_status);

/* ------------------------------------------------------------------------ */
/* Request server for streams of KKT solves (no counterpart in the reference).
 * Patterns are analysed once; each request brings K's values (host FP64, the
 * pattern's CSR order) and nrhs right-hand sides (host, n x nrhs column-major),
 * copied at submit.  progress() completes finished batches and admits queued
 * requests, in arrival order and within memory_budget device bytes (<= 0:
 * unlimited), into free slots: per request the values' upload and the numeric
 * factor (BK, level-0 fill), then the SQMR(tol, max_it) solves.  A batch
 * holds requests of one class, in arrival order.  Patterns with n below the
 * large-row threshold (culipx_server_set_large_rows, default 131072): one CTA
 * per request and group of up to 4 of its right-hand sides (the group shares
 * every factor and K load); up to `slots` such batches run concurrently on
 * their own streams, at most max_batch requests each.  Larger patterns: per request the whole-GPU
 * solver of culipx_sqmr_solve_multi (right-hand sides in groups of up to 4),
 * at most 4 requests per batch, and such a batch runs alone on the device.
 * A request's results do not depend on the other requests.
 * result() returns CULIPX_PENDING until the request is done; latency_ms runs
 * from submit to the progress() call that saw it finish. */
typedef struct culipx_server_t *culipx_server;
int culipx_server_create(int device, long long memory_budget, int slots, int max_batch, double tol, int max_it,
                         culipx_server *out);
int culipx_server_destroy(culipx_server s);
int culipx_server_add_pattern(culipx_server s, int n, const int *h_rowptr, const int *h_colidx, int num_blocks,
                              const int *h_block_starts, int precision, int *pattern_id);
int culipx_server_submit(culipx_server s, int pattern_id, const double *h_vals, int nrhs, const double *h_b,
                         int *request_id);
/* wait != 0: block until at least one request finishes (or nothing runs) */
int culipx_server_progress(culipx_server s, int wait, int *completed);
int culipx_server_result(culipx_server s, int request_id, double *h_x, int *h_iterations, int *h_status,
                         double *latency_ms);
/* forget a finished request */
int culipx_server_release(culipx_server s, int request_id);
/* stats[0..7]: queued, running, done, batches launched, device bytes of
 * running requests, device bytes held by patterns and factor pools, patterns,
 * large (whole-GPU) batches launched */
int culipx_server_stats(culipx_server s, long long *stats8);
/* requests on patterns with n >= rows use the whole-GPU solver (rows >= 1;
 * default 131072); applies to batches admitted afterwards */
int culipx_server_set_large_rows(culipx_server s, int rows);
/* Imported L D L' preconditioner (ImportLDUPreconditioner<T>,
 * libs/la/preconditioner/import_ldu_preconditioner.impl.cuh, as the
 * reference's tests/la/test_sqmr.cc:192-293 use it): L lower-triangular CSR
 * (n rows, device, FP64; its diagonal divides, 1 where absent), D as
 * tri[3n] / is_piv[n] (the block factor's storage), perm[n] (P) and scale[n]
 * (S), all device arrays, copied at create (which synchronizes).
 *   LEFT   x = L^-1 P' (S .* b)
 *   MIDDLE x = D^-1 b
 *   RIGHT  x = S .* P (L'^-1 b)
 * Both substitutions run level by level; each row sums its terms in the order
 * of a serial sweep.  b and x must not overlap. */
typedef struct culipx_ldu_t *culipx_ldu;
int culipx_ldu_create(culipx_handle h, int n, const int *d_rowptr, const int *d_colidx, const double *d_val,
                      const double *d_tri, const int *d_is_piv, const int *d_perm, const double *d_scale,
                      culipx_ldu *out);
int culipx_ldu_apply(culipx_ldu P, int stage, const double *d_b, double *d_x);
/* SQMR (as culipx_sqmr_solve) with the imported preconditioner */
int culipx_sqmr_solve_ldu(culipx_handle h, culipx_csr A, culipx_ldu P, const double *d_b, double *d_x, double tol,
                          int max_it, double *residual, int *iterations);
int culipx_ldu_destroy(culipx_ldu P);

/* Matrix-free KKT operators over a constraint matrix A (m x n, FP64 CSR on
 * the device, borrowed) and a diagonal D (n, borrowed); they replace
 * AugmentedMatrixSPMV<T> and NormalMatrixSPMV<T> (libs/la/spmv.cuh:75-149,
 * spmv.impl.cuh:122-430), FP64:
 *   CULIPX_OP_AUGMENTED  y = alpha [D x1 + A' x2 ; A x1 + (delta I)(ix) x2] + beta y,
 *                        x = [x1; x2], n + m rows
 *   CULIPX_OP_NORMAL     y = alpha (A D^-1 A' x + (delta I)(ix) x) + beta y, m rows
 * (delta I)(ix) adds delta * x[ix[i]] at row ix[i] (ix: num_ix row indices of
 * the constraint block, device, may be NULL with num_ix = 0).  Two
 * differences from the reference on purpose: its augmented product adds
 * A' x1 where A' x2 belongs (spmv.impl.cuh:416-420), and its shift multiplies
 * x[i] instead of x[ix[i]] (k_add_app, helper_kernels.impl.cuh:361-374).
 * create copies A to the host once to build A' (the reference's
 * explicit_At) and synchronizes; multiply is asynchronous on the handle's
 * stream. */
#define CULIPX_OP_AUGMENTED 0
#define CULIPX_OP_NORMAL 1
typedef struct culipx_kkt_operator_t *culipx_kkt_operator;
int culipx_kkt_operator_create(culipx_handle h, int kind, int m, int n, long long nnz, const int *d_rowptr,
                               const int *d_colidx, const double *d_val, const double *d_d, double delta,
                               int num_ix, const int *d_ix, culipx_kkt_operator *out);
int culipx_kkt_operator_multiply(culipx_kkt_operator op, const double *d_x, double *d_y, double alpha, double beta);
int culipx_kkt_operator_destroy(culipx_kkt_operator op);

/* Block-size tuner for a KKT pattern (n H rows, m constraint rows; no
 * counterpart in the reference, whose driver reads a fixed blocking from a
 * file, apps/block_ildlt/block_ildlt.cc:29-35): for each candidate size the
 * contiguous KKT blocking (culipx_kkt_blocking), symbolic analysis, numeric
 * factor (precision F64 or F32, BK, level-0 fill) and one SQMR solve of d_b
 * (tol, max_it), timed with CUDA events on the handle's stream after one
 * warm-up run.  best_block = the fastest candidate whose solve met tol, else
 * the one with the smallest final SQMR residual estimate.  Per candidate: the
 * factor + solve time in ms, iterations, status (OK, MAXIT, BREAKDOWN) and
 * the residual estimate; each output array may be NULL.  Synchronizes the
 * stream. */
int culipx_tune_kkt_block(culipx_handle h, int n, int m, const int *h_rowptr, const int *h_colidx,
                          const double *d_vals, const double *d_b, int precision, const int *candidates,
                          int num_candidates, double tol, int max_it, int *best_block, double *h_ms,
                          int *h_iterations, int *h_status, double *h_residual);

/* FP64 iterative refinement of every request (the mixed-precision serving
 * path, meant for FP32 patterns; no counterpart in the reference): after the
 * solve, r = b - K x in FP64 per right-hand side; while ||r|| > tol ||b|| and
 * fewer than max_refine corrections: d = SQMR(K, M, r, inner_tol), x += d,
 * new r; two corrections in a row without a new smallest ||r|| stop the
 * right-hand side (STALLED).  Corrections of a batch's right-hand sides run
 * together.  Every right-hand side returns its iterate of smallest ||r||, the
 * request's iterations are the SQMR iterations summed and its status OK when
 * ||b - K x|| <= tol ||b||, else STALLED or MAXIT (BREAKDOWN if a solve broke
 * down).
 * max_refine 0 (the default) turns it off; applies to batches admitted
 * afterwards. */
int culipx_server_set_refine(culipx_server s, int max_refine, double inner_tol);
/* kernels the server has launched so far (all slots) */
int culipx_server_launch_count(culipx_server s, long long *count);

/* culipx_sqmr_refine per system of a batch: every step solves all systems
 * still above tol in one batched launch (the others get a zero right-hand
 * side); per system the true relative residual, the SQMR iterations summed,
 * the corrections computed and a status (OK, MAXIT, STALLED, BREAKDOWN), as
 * culipx_sqmr_refine defines them. */
int culipx_batch_sqmr_refine(culipx_batch b, culipx_csr A, culipx_factor M, const double *d_b, double *d_x,
                             double tol, double inner_tol, int inner_max_it, int max_refine, double *h_relres,
                             int *h_iterations, int *h_steps, int *h_status);

/* FP64 iterative refinement around SQMR (no counterpart in the reference,
 * whose SQMR solves once in the factor's precision): x = 0, r = b; while
 * ||r|| > tol ||b|| and fewer than max_refine corrections: d = SQMR(K, M, r,
 * inner_tol, inner_max_it), x += d, r = b - K x (FP64).  With an FP32 factor
 * the preconditioner applies are single precision and everything else FP64.
 * The iterate of smallest ||r|| is kept and returned; two corrections in a
 * row that do not lower it end the loop with CULIPX_STALLED (the inner solves
 * no longer help: raise inner_max_it or use an FP64 factor).  relres =
 * ||b - K x|| / ||b|| of the returned x, iterations = SQMR iterations summed,
 * steps = corrections computed.  Returns CULIPX_MAXIT if tol was not reached
 * in max_refine corrections. */
int culipx_sqmr_refine(culipx_handle h, culipx_csr A, culipx_factor M, const double *d_b, double *d_x,
                       double tol, double inner_tol, int inner_max_it, int max_refine, double *relres,
                       int *iterations, int *steps);

/* Per-phase device timing of the persistent solver (no counterpart in the
 * reference, which has wall-clock timers only, libs/utils/defines.h:65-85):
 * enable, solve, then read for each of the first min(iterations, 64)
 * iterations six values in microseconds: phase 1 (v+, its norm and the
 * first U-sweep level), the other U-sweep levels, the first U'-sweep level
 * (with the fused SpMV, the dots and the p / x update), the other U'-sweep
 * levels with the final reduction, an unused slot (0), and the whole
 * iteration. */
int culipx_sqmr_profile(culipx_handle h, int enable);
/* Fault injection for tests (no counterpart in the reference).  In the
 * persistent solver's iteration the level-0 rows of a two-level system wait
 * on a device counter for the level-1 rows of every CTA (a bounded wait:
 * 200 ms); skew > 0 raises the count they wait for beyond reach, so the wait
 * gives up and the solve returns CULIPX_TIMEOUT (results invalid) instead of
 * hanging.  0 (the default) for normal operation. */
int culipx_sqmr_set_wait_skew(culipx_handle h, unsigned long long skew);
int culipx_sqmr_phase_times(culipx_handle h, double *out_us, int iterations);

/* The same solve (same kernel, same results) without any device allocation;
 * no counterpart in the reference.  For callers that cannot allocate device
 * memory while they solve: processes whose GPU memory is already owned by
 * another allocator (a caching allocator such as PyTorch's, or an
 * application-wide pool), and latency-critical request loops in which
 * cudaMalloc / cudaFree could synchronize the device.  M must be a computed
 * factor (FP64 or FP32); n must not exceed 65536 (larger n is rejected with
 * CULIPX_INVALID_ARG).  The work vectors live in a fixed scratch array
 * compiled into the library (about 4.3 MB, held by every GPU that loads the
 * library until the process exits); it is shared by all calls and keeps the
 * last call's contents, so calls whose work overlaps on the GPU race.  The
 * first call on a device looks up the scratch's device address; make it
 * before any stream capture. */
int culipx_sqmr_solve_noalloc(culipx_handle h, culipx_csr A, culipx_factor M, const double *d_b,
                              double *d_x, double tol, int max_it, double *residual, int *iterations);

#ifdef __cplusplus
}
#endif
#endif /* CULIPX_H */
