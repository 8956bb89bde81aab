// CSR operator (borrowed device arrays) and its SpMV.
#pragma once

#include "device.h"

namespace culipx {

struct Csr {
    culipx_handle_t* h = nullptr;
    int m = 0, n = 0;
    long long nnz = 0;
    const int* rowptr = nullptr;
    const int* colidx = nullptr;
    const void* val = nullptr;
    int precision = CULIPX_F64;
    bool has_t = false;
    DeviceBuffer t_rowptr, t_colidx, t_val;  // explicit transpose (owned)
};

int csr_build_transpose(Csr* A);
int csr_spmv(Csr* A, const void* x, void* y, double alpha, double beta, int transpose, cudaStream_t s);

}  // namespace culipx

struct culipx_csr_t : culipx::Csr {};
