// SQMR workspace and solver entry.
#pragma once

#include "device.h"
#include "spmv.h"

namespace culipx {

struct Factor;

// Work vectors (13 x n doubles), per-CTA partials and the device scalar block.
struct Sqmr {
    int n = -1;
    bool force_multi_kernel = false;  // use the per-phase kernels instead of the persistent solver
    bool profile = false;             // record per-phase device timestamps of the persistent solver
    DeviceBuffer ts;                  // 64 iterations x 8 phase stamps (ns, %globaltimer)
    DeviceBuffer vecs, partials, scal;
    DeviceBuffer ref_r, ref_d, ref_part;  // iterative refinement: residual, correction, norm partials
    void* host_flags = nullptr;  // pinned
    ~Sqmr()
    {
        if (host_flags) cudaFreeHost(host_flags);
    }
};

int sqmr_workspace(Sqmr* w, culipx_handle_t* h, int n);
int sqmr_solve(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
               double* residual, int* iterations, Sqmr* w);
int sqmr_solve_persistent(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                          double* residual, int* iterations, Sqmr* w);
int sqmr_refine(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, double inner_tol,
                int inner_max_it, int max_refine, double* relres, int* iterations, int* steps, Sqmr* w);
int sqmr_solve_noalloc(culipx_handle_t* h, Csr* A, Factor* M, const double* b, double* x, double tol, int max_it,
                       double* residual, int* iterations);

}  // namespace culipx
