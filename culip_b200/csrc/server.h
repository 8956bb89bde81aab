// Request server over the batched solver (see server.cu).
#pragma once

#include "device.h"
#include "spmv.h"
#include "sqmr.h"

#include <deque>
#include <unordered_map>
#include <vector>

namespace culipx {

struct Pattern;
struct Factor;

struct ServerPattern {
    Pattern* pat = nullptr;
    int n = 0;
    long long nnz = 0;
    int precision = CULIPX_F64;
    DeviceBuffer d_rowptr, d_colidx;       // K's structure on the device
    std::vector<Factor*> free_factors;     // pool, reused across requests
    long long pool_bytes = 0;              // device bytes held by the pool
    long long factor_bytes_estimate() const;
};

struct ServerRequest {
    int id = 0, pid = 0, nrhs = 1;
    int state = 0;                         // 0 queued, 1 running, 2 done
    std::vector<double> vals, b;           // host copies until the batch launches
    std::vector<double> x;                 // result, n x nrhs column-major
    std::vector<int> its, status;
    double t_submit = 0.0, t_done = 0.0;   // ms, steady clock
    long long bytes = 0;                   // device bytes while running
    Factor* F = nullptr;
    void *d_vals = nullptr, *d_vals32 = nullptr, *d_b = nullptr, *d_x = nullptr;
    // FP64 refinement (Server::max_refine > 0): residuals, corrections, best
    // iterates, and per right-hand side ||b||, the smallest relative residual,
    // corrections computed, corrections in a row without a smaller residual,
    // SQMR iterations summed, breakdown seen, stalled
    void *d_r = nullptr, *d_d = nullptr, *d_best = nullptr;
    int q = -1;                            // position in the running batch
    std::vector<double> bnorm, rel;
    std::vector<int> steps, fails, its_acc;
    std::vector<char> broke, stalled;
};

struct ServerSlot {
    culipx_handle_t* h = nullptr;          // own stream and SQMR workspace
    cudaEvent_t done = nullptr;
    bool busy = false;
    bool large = false;                    // the running batch is of whole-GPU solves
    std::vector<int> reqs;
    std::vector<Csr> csrs;
    double* out_host = nullptr;            // pinned: 8 values per system
    int out_cap = 0;
    double* x_host = nullptr;              // pinned: the batch's solutions
    size_t x_cap = 0;
    int phase = 0;                         // 0: solving or ending; 1: residuals in flight (refinement)
    std::vector<std::pair<int, int>> cols; // (request, column) of the last solves, in result-slot order
    double* res_host = nullptr;            // pinned: their residuals' sums of squares
    size_t res_cap = 0;
    DeviceBuffer jobs;                     // device descriptors of the refinement kernels
};

struct Server {
    int device = 0;
    long long budget = 0, in_use = 0;
    int max_batch = 0, max_it = 0;
    int large_rows = 131072;               // patterns with n >= this get the whole-GPU solver
    int max_refine = 0;                    // FP64 refinement corrections per right-hand side (0: none)
    double inner_tol = 1e-6;               // SQMR tolerance of the corrections
    long long large_batches = 0;
    double tol = 0.0;
    culipx_handle_t* base = nullptr;       // owns the patterns' device mirrors
    std::vector<ServerPattern> patterns;
    std::vector<ServerSlot> slots;
    std::deque<int> queue;
    std::unordered_map<int, ServerRequest> requests;
    int next_id = 0;
    long long done = 0, batches = 0;
    long long fixed_bytes() const;
    int running_slots() const;
    ~Server();
};

int server_create(int device, long long budget, int slots, int max_batch, double tol, int max_it, Server** out);
int server_add_pattern(Server* s, int n, const int* rowptr, const int* colidx, int num_blocks, const int* block_starts,
                       int precision, int* pattern_id);
int server_submit(Server* s, int pid, const double* vals, int nrhs, const double* b, int* request_id);
int server_progress(Server* s, int wait, int* completed);
int server_result(Server* s, int id, double* x, int* its, int* status, double* latency_ms);
int server_release(Server* s, int id);
int server_stats(Server* s, long long* st8);
int server_set_large_rows(Server* s, int rows);
int server_launch_count(Server* s, long long* out);
int server_set_refine(Server* s, int max_refine, double inner_tol);
int factor_compute(Factor* f, const void* d_vals, const int* h_is_piv, int pivot, double threshold);
int factor_create(Pattern* p, Factor** out);

}  // namespace culipx

struct culipx_server_t : culipx::Server {};
