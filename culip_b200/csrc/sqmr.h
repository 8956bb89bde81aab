// SQMR workspace and solver entry.
#pragma once

#include "device.h"
#include "spmv.h"

#include <vector>

namespace culipx {

struct Factor;

// Work vectors (13 x n doubles), per-CTA partials and the device scalar block.
struct Sqmr {
    int n = -1;
    bool force_multi_kernel = false;  // use the per-phase kernels instead of the persistent solver
    bool profile = false;             // record per-phase device timestamps of the persistent solver
    unsigned long long wait_skew = 0; // added to the persistent solver's level-wait target (tests; 0)
    DeviceBuffer ts;                  // 64 iterations x 8 phase stamps (ns, %globaltimer)
    DeviceBuffer vecs, partials, scal;
    DeviceBuffer ref_r, ref_d, ref_part;  // iterative refinement: residual, correction, norm partials
    DeviceBuffer ref_best;                // its best iterate so far
    DeviceBuffer many;                    // sqmr_solve_many: vectors, argument blocks, counter
    void* host_flags = nullptr;  // pinned
    ~Sqmr()
    {
        if (host_flags) cudaFreeHost(host_flags);
    }
};

// Independent systems stored as one block-diagonal union pattern: row ranges
// and, per system and level, the positions of its block rows in the level lists.
struct Pattern;
struct Batch {
    culipx_handle_t* h = nullptr;
    const Pattern* pat = nullptr;
    Pattern* pat_ref = nullptr;               // the C ABI's reference on pat (released with the batch)
    int num = 0, nl = 0;
    std::vector<int> row_off;                 // num + 1
    DeviceBuffer d_row_off, d_qb, d_qe;       // num + 1, num x nl, num x nl
    DeviceBuffer d_out, d_next;               // num x 8 results, system counter
    // batch_factor_solve_graph: the factorization and the batched solve as one
    // CUDA graph, its own workspace (the graph holds its addresses), and what
    // the graph was captured for
    Sqmr* gw = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaStream_t capture_stream = nullptr;
    struct Key {
        const void* vals = nullptr;
        unsigned long long A = 0, M = 0;  // serial numbers: host addresses can be reused
        const double* b = nullptr;
        double* x = nullptr;
        int pivot = -1, max_it = -1;
        double threshold = -1.0, tol = -1.0, piv64 = -1.0;
        bool operator==(const Key& o) const
        {
            return vals == o.vals && A == o.A && M == o.M && b == o.b && x == o.x && pivot == o.pivot &&
                   max_it == o.max_it && threshold == o.threshold && tol == o.tol && piv64 == o.piv64;
        }
    } graph_key;
    int graph_launches = 0;
    ~Batch();
};

int batch_create(culipx_handle_t* h, const Pattern* p, int num, const int* h_row_off, Batch** out);
int batch_sqmr_solve(Batch* bt, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                     double* h_res, int* h_its, int* h_status, Sqmr* w);

int batch_factor_solve_graph(Batch* bt, Csr* A, Factor* M, const void* d_vals, int pivot, double threshold,
                             const double* b, double* x, double tol, int max_it, double* h_res, int* h_its,
                             int* h_status);

int batch_sqmr_refine(Batch* bt, Csr* A, Factor* M, const double* b, double* x, double tol, double inner_tol,
                      int inner_max_it, int max_refine, double* h_relres, int* h_its, int* h_steps, int* h_status,
                      Sqmr* w);

int sqmr_solve_many(culipx_handle_t* h, int num, Csr* const* A, Factor* const* M, const double* const* b,
                    double* const* x, double tol, int max_it, double* h_res, int* h_its, int* h_status, Sqmr* w);

int sqmr_solve_many_async(culipx_handle_t* h, int num, Csr* const* A, Factor* const* M, const double* const* b,
                          double* const* x, double tol, int max_it, Sqmr* w, double* out_host);
int sqmr_solve_many_nr_async(culipx_handle_t* h, int num, Csr* const* A, Factor* const* M, const double* const* b,
                             double* const* x, const int* nr, double tol, int max_it, Sqmr* w, double* out_host);
void many_results(int num, int max_it, const double* out, double* h_res, int* h_its, int* h_status);

int sqmr_solve_multi(culipx_handle_t* h, Csr* A, Factor* M, int nrhs, const double* B, double* X, double tol,
                     int max_it, double* h_res, int* h_its, int* h_status, Sqmr* w);
int sqmr_solve_multi_async(culipx_handle_t* h, Csr* A, Factor* M, int nrhs, const double* B, double* X, double tol,
                           int max_it, Sqmr* w, double* out_host);

int sqmr_refine_multi(culipx_handle_t* h, Csr* A, Factor* M, int nrhs, const double* B, double* X, double tol,
                      double inner_tol, int inner_max_it, int max_refine, double* h_relres, int* h_its, int* h_steps,
                      int* h_status, Sqmr* w);

int sqmr_workspace(Sqmr* w, culipx_handle_t* h, int n);

struct Ldu;
int sqmr_solve_ldu(culipx_handle_t* h, Csr* A, Ldu* P, const double* b, double* x, double tol, int max_it,
                   double* residual, int* iterations, Sqmr* w);

int tune_kkt_block(culipx_handle_t* h, int n, int m, const int* rowptr, const int* colidx, const double* d_vals,
                   const double* d_b, int precision, const int* candidates, int num_candidates, double tol, int max_it,
                   int* best_block, double* h_ms, int* h_iterations, int* h_status, double* h_residual);
int sqmr_solve(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
               double* residual, int* iterations, Sqmr* w);
int sqmr_solve_persistent(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                          double* residual, int* iterations, Sqmr* w);
int sqmr_refine(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, double inner_tol,
                int inner_max_it, int max_refine, double* relres, int* iterations, int* steps, Sqmr* w);
int sqmr_solve_noalloc(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                       double* residual, int* iterations);

}  // namespace culipx

struct culipx_batch_t : culipx::Batch {};
