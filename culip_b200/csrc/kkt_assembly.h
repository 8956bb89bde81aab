// KKT assembly of an interior-point iteration: the explicit K of the
// augmented system from the constraint matrix A and the iterate.
#pragma once

#include "device.h"

namespace culipx {

struct KktAssembly {
    culipx_handle_t* handle = nullptr;
    int m = 0, n = 0;
    long long nnz_a = 0, nnz_k = 0;
    DeviceBuffer rowptr, colidx;  // K's structure: N + 1 offsets, nnz_k columns (sorted)
    DeviceBuffer src;             // per entry of K: its entry of A (>= 0) or -1 - row for a diagonal
};

int kkt_assembly_create(culipx_handle_t* h, int m, int n, long long nnz_a, const int* d_rowptr, const int* d_colidx,
                        KktAssembly** out);
int kkt_assembly_values(KktAssembly* K, const double* d_aval, const double* d_x, const double* d_s,
                        const double* d_d, double delta, double gamma, int precision, void* d_kval);

}  // namespace culipx

struct culipx_kkt_assembly_t : culipx::KktAssembly {};
