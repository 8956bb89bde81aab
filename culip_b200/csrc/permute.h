// Permutation plan of a CSR pattern (B = P_r A P_c' with sorted rows and
// columns) and the per-call value gather with optional scaling.
#pragma once

#include "device.h"

namespace culipx {

struct PermutePlan {
    culipx_handle_t* handle = nullptr;
    int n = 0;
    long long nnz = 0;
    DeviceBuffer col_perm, inv_row;          // old -> new columns, new -> old rows
    DeviceBuffer rowptr, colidx;             // B's structure
    DeviceBuffer src;                        // per entry of B: its entry in A
    DeviceBuffer new_row_of, old_row_of, old_col_of;
    DeviceBuffer scan_tmp;
    DeviceBuffer bad;                        // create: invalid input seen
};

int permute_plan_create(culipx_handle_t* h, int n, long long nnz, const int* d_rowptr, const int* d_colidx,
                        const int* h_row_perm, const int* h_col_perm, int perm_is_old_to_new, PermutePlan** out);
int permute_plan_apply(PermutePlan* p, int precision, const void* d_val, const void* d_row_scale,
                       const void* d_col_scale, int scale_before_match, void* d_out);

}  // namespace culipx

struct culipx_permute_t : culipx::PermutePlan {};
