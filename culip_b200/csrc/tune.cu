// Block-size tuner for KKT patterns (no counterpart in the reference, whose
// driver reads a fixed blocking from a file, apps/block_ildlt/block_ildlt.cc:29-35).
//
// For each candidate size c the pattern gets the contiguous KKT blocking of
// c-row blocks (culipx_kkt_blocking), the symbolic analysis, the numeric
// factor in the requested precision and one preconditioned SQMR solve of the
// caller's right-hand side; the factor + solve of a second, timed run is
// measured with CUDA events on the handle's stream (the first run warms the
// workspaces up).  The best size is the fastest among the candidates whose
// solve met tol; when none did, the one whose solve got furthest (the
// smallest final SQMR residual estimate), the better start for refinement.
#include "factor.h"
#include "pattern.h"
#include "spmv.h"
#include "sqmr.h"
#include "kernels_common.cuh"

#include <vector>

extern "C" int culipx_kkt_blocking(int n, int m, int block, int* block_starts, int capacity, int* num_blocks);

namespace culipx {

namespace {

__global__ void k_f64_to_f32(const double* __restrict__ in, float* __restrict__ out, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) out[i] = (float)in[i];
}

}  // namespace

int tune_kkt_block(culipx_handle_t* h, int n, int m, const int* rowptr, const int* colidx, const double* d_vals,
                   const double* d_b, int precision, const int* candidates, int num_candidates, double tol, int max_it,
                   int* best_block, double* h_ms, int* h_iterations, int* h_status, double* h_residual)
{
    if (!h || !rowptr || !colidx || !d_vals || !d_b || !candidates || num_candidates < 1 || !best_block ||
        n < 1 || m < 0 || max_it < 0 || !(tol >= 0.0))
        return fail(CULIPX_INVALID_ARG, "culipx_tune_kkt_block: bad argument");
    if (precision != CULIPX_F64 && precision != CULIPX_F32)
        return fail(CULIPX_INVALID_ARG, "culipx_tune_kkt_block: bad precision");
    const int N = n + m;
    const long long nnz = rowptr[N];
    cudaStream_t s = h->stream;
    DeviceBuffer d_rp, d_ci, d_x, d_v32;
    CULIPX_TRY(d_rp.upload(h, rowptr, (size_t)(N + 1) * sizeof(int)));
    CULIPX_TRY(d_ci.upload(h, colidx, (size_t)std::max<long long>(nnz, 1) * sizeof(int)));
    CULIPX_TRY(d_x.alloc(h, (size_t)N * sizeof(double)));
    const void* fv = d_vals;
    if (precision == CULIPX_F32) {
        CULIPX_TRY(d_v32.alloc(h, (size_t)std::max<long long>(nnz, 1) * sizeof(float)));
        k_f64_to_f32<<<148 * 4, 256, 0, s>>>(d_vals, d_v32.as<float>(), nnz);
        h->launches += 1;
        CULIPX_TRY(launch_check("k_f64_to_f32"));
        fv = d_v32.get();
    }
    Csr A;
    A.h = h;
    A.m = A.n = N;
    A.nnz = nnz;
    A.rowptr = d_rp.as<int>();
    A.colidx = d_ci.as<int>();
    A.val = d_vals;
    A.precision = CULIPX_F64;
    cudaEvent_t e0, e1;
    CULIPX_CUDA(cudaEventCreate(&e0));
    CULIPX_CUDA(cudaEventCreate(&e1));
    int best = -1;
    double best_ms = 0.0, best_res = 0.0;
    bool best_ok = false;
    int st = CULIPX_OK;
    for (int c = 0; c < num_candidates && st == CULIPX_OK; ++c) {
        int nb = 0;
        st = culipx_kkt_blocking(n, m, candidates[c], nullptr, 0, &nb);
        if (st != CULIPX_OK) break;
        std::vector<int> bs(nb + 1);
        st = culipx_kkt_blocking(n, m, candidates[c], bs.data(), nb + 1, &nb);
        if (st != CULIPX_OK) break;
        Pattern* p = nullptr;
        st = analyze_pattern(h, N, rowptr, colidx, nb, bs.data(), 0, 1.0, precision, &p);
        if (st != CULIPX_OK) break;
        Factor* f = nullptr;
        st = factor_create(p, &f);
        double ms = 0.0, res = 0.0;
        int its = 0, sst = CULIPX_OK;
        for (int run = 0; run < 2 && st == CULIPX_OK; ++run) {
            if (run == 1 && cudaEventRecord(e0, s) != cudaSuccess) st = fail(CULIPX_CUDA_ERROR, "event record failed");
            if (st == CULIPX_OK) st = factor_compute(f, fv, nullptr, CULIPX_PIV_BK, 0.0);
            if (st == CULIPX_OK) {
                sst = sqmr_solve(h, &A, f, d_b, d_x.as<double>(), tol, max_it, &res, &its, h->sqmr);
                if (sst != CULIPX_OK && sst != CULIPX_MAXIT && sst != CULIPX_BREAKDOWN) st = sst;
            }
            if (run == 1 && st == CULIPX_OK) {
                float t = 0.0f;
                if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                    cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)
                    st = fail(CULIPX_CUDA_ERROR, "culipx_tune_kkt_block: event timing failed");
                ms = t;
            }
        }
        delete static_cast<culipx_factor_t*>(f);
        delete static_cast<culipx_pattern_t*>(p);
        if (st != CULIPX_OK) break;
        if (h_ms) h_ms[c] = ms;
        if (h_iterations) h_iterations[c] = its;
        if (h_status) h_status[c] = sst;
        if (h_residual) h_residual[c] = res;
        const bool ok = sst == CULIPX_OK;
        const bool better = best < 0 || (ok && !best_ok) || (ok && best_ok && ms < best_ms) ||
                            (!ok && !best_ok && res < best_res);
        if (better) {
            best = c;
            best_ms = ms;
            best_res = res;
            best_ok = ok;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != CULIPX_OK) return st;
    *best_block = candidates[best];
    return CULIPX_OK;
}

}  // namespace culipx
