// Imported L D L' preconditioner (see ldu.cu).
#pragma once

#include "device.h"

#include <vector>

namespace culipx {

struct Ldu {
    culipx_handle_t* h = nullptr;
    int n = 0;
    DeviceBuffer rp, ci, val, diag;      // L (rows), its diagonal (1 where absent)
    DeviceBuffer trp, tci, tval;         // L' rows, columns descending
    DeviceBuffer fwd_rows, bwd_rows;     // rows by level of the two substitutions
    std::vector<int> fwd_rows_h, bwd_rows_h, fwd_off, bwd_off;
    DeviceBuffer tri, is_piv, perm, scale;  // D (tridiagonal storage), P, S
    DeviceBuffer t1, t2;                 // scratch
};

int ldu_create(culipx_handle_t* h, int n, const int* d_rowptr, const int* d_colidx, const double* d_val,
               const double* d_tri, const int* d_is_piv, const int* d_perm, const double* d_scale, Ldu** out);
int ldu_apply(Ldu* P, int stage, const double* b, double* x, cudaStream_t s);

}  // namespace culipx

struct culipx_ldu_t : culipx::Ldu {};
