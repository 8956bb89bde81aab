// Matrix-free KKT operators (augmented and normal-equations products).
#pragma once

#include "device.h"

namespace culipx {

struct KktOperator {
    culipx_handle_t* h = nullptr;
    int kind = 0;                         // 0 augmented (n + m rows), 1 normal (m rows)
    int m = 0, n = 0;
    long long nnz = 0;
    const int* rowptr = nullptr;          // A, borrowed
    const int* colidx = nullptr;
    const double* val = nullptr;
    const double* d = nullptr;            // diagonal D (n), borrowed
    DeviceBuffer t_rowptr, t_colidx, t_val;  // A' (owned)
    DeviceBuffer shift;                   // delta at the rows listed in ix, 0 elsewhere (m)
    DeviceBuffer tmp;                     // normal product: D^-1 A' x (n)
};

int kkt_operator_create(culipx_handle_t* h, int kind, int m, int n, long long nnz, const int* d_rowptr,
                        const int* d_colidx, const double* d_val, const double* d_d, double delta, int num_ix,
                        const int* d_ix, KktOperator** out);
int kkt_operator_multiply(KktOperator* op, const double* x, double* y, double alpha, double beta);

}  // namespace culipx

struct culipx_kkt_operator_t : culipx::KktOperator {};
