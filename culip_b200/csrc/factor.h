// Numeric block-iLDL^T factor on the device and the solve structures built
// from it.
#pragma once

#include "pattern.h"

namespace culipx {

// per block row flags written by the factor's pivot kernel
enum RowFlags : int {
    kRowIdentity = 1,      // the factored pivot tile is exactly the identity
    kRowHas2x2 = 2,        // D has a 2x2 pivot in this block row
    kRowPermIdentity = 4,  // no pivot swaps inside the tile
    kRowNoUpdates = 8,     // the pivot block received no Schur updates
};

// A pivot-tile block row as a work item of the sweeps: everything the item
// needs before its data, read with two 16-byte loads (block row, first row,
// rows, row flags; packed-tile offset, non-unit diagonal mask)
struct alignas(16) CItem {
    int I, fr, h, flags;
    long long pk_off;
    unsigned nd;
    int pad;
};
static_assert(sizeof(CItem) == 32, "CItem is two 16-byte words");

struct Factor {
    Pattern* pat = nullptr;
    unsigned long long serial = next_serial();
    int precision = CULIPX_F64;
    size_t vbytes = 8;
    bool computed = false;
    int pivot = CULIPX_PIV_BK;
    double threshold = 0.0;
    int solve_algorithm = CULIPX_SOLVE_BLOCK;  // set_solve_algorithm
    int jacobi_sweeps = 0;
    double pivot_fp64 = kPivotFp64Default;     // FP32 factors: FP64 inversion of 2x2 pivots below this ratio

    // block storage (pattern layout + relocation arena for blocks that were
    // granted extra slots by dual dropping)
    DeviceBuffer val, idx;       // val_cap slots
    long long val_cap = 0;
    DeviceBuffer boff;           // per block: slot offset (int64)
    DeviceBuffer nnz, cap;       // per block: stored entries (sparse), capacity after grants
    DeviceBuffer got_extra;      // per block
    DeviceBuffer tri;            // 3n values
    DeviceBuffer is_piv, perm;   // n ints
    DeviceBuffer rowflags;       // per block row: bit0 pivot tile is identity, bit1 D has a 2x2
    DeviceBuffer state;          // device scalars (see factor.cu)
    DeviceBuffer deferred;       // per level list of deferred blocks
    DeviceBuffer slowlist;       // per level list of blocks for the tiled off-diagonal kernel
    DeviceBuffer norm_part;      // threshold > 0: row-norm partials
    DeviceBuffer row_norm;       // n values

    // sweep structures (fine-row CSR of the strictly off-diagonal block part)
    DeviceBuffer u_off, u_col, u_val;    // rows of U
    DeviceBuffer ut_off, ut_col, ut_val; // rows of U' (columns of U)
    DeviceBuffer piv_off;                // per block row: value slot of its pivot tile
    // the persistent solver's copies: upper triangles of the non-identity
    // pivot tiles packed column by column (U sweep) and row by row (U'
    // sweep), h(h+1)/2 slots per block row at pk_off; the U columns mapped
    // through the pivot permutation; the diagonal of D
    DeviceBuffer pk_col, pk_row, pk_off;
    DeviceBuffer ndmask;  // per block row: bit r set if U_rr != 1 in its pivot tile
    DeviceBuffer u_colp;
    DeviceBuffer dg;
    // each level's block rows split in level-list order into simple ones
    // (identity pivot tile, no swaps, 1x1 pivots: every fine row is
    // independent) and the others; scan_s / scan_c (num_blocks + 1) are the
    // running counts of simple fine rows / other block rows, so level L owns
    // simple_rows[scan_s[lvl_off[L]] ..) and cplx[scan_c[lvl_off[L]] ..)
    DeviceBuffer scan_s, scan_c, simple_rows, cplx;
    // per entry of cplx: its block row's metadata in one 32-byte record (CItem)
    DeviceBuffer citem;
    DeviceBuffer work;                   // n values of apply scratch
    DeviceBuffer jac_a, jac_b;           // SOLVE_JACOBI iterates (n values each, allocated on first use)
    DeviceBuffer scan_tmp;               // scan partial sums
    long long u_nnz = 0;

    float last_ms = 0.f;
    int last_launches = 0;
    // the numeric factorization as a CUDA graph (factor_compute_graph)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    const void* graph_vals = nullptr;
    int graph_pivot = -1;
    double graph_threshold = -1.0;
    double graph_piv64 = -1.0;
    int graph_launches = 0;
    bool capturing = false;
    cudaStream_t capture_stream = nullptr;
    Factor() = default;
    Factor(const Factor&) = delete;
    Factor& operator=(const Factor&) = delete;
    ~Factor();
};

int factor_create(Pattern* p, Factor** out);
int factor_compute(Factor* f, const void* d_vals, const int* h_is_piv, int pivot, double threshold);
int factor_compute_graph(Factor* f, const void* d_vals, int pivot, double threshold);
int factor_export(Factor* f, int* blk_nnz, long long* blk_off, int* idx, void* val, void* tri,
                  int* is_piv, int* perm, int* got_extra, long long* total);
int prec_apply(Factor* f, int stage, const void* d_b, void* d_x, cudaStream_t stream);

}  // namespace culipx

struct culipx_factor_t : culipx::Factor {};
