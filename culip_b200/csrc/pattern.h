// Host-side symbolic analysis of one KKT sparsity pattern and the device
// mirror that the numeric kernels read.
#pragma once

#include "common.h"
#include "device.h"

#include <vector>

namespace culipx {

enum BlockFormat : int { kSparse = 0, kDense = 1 };  // BLOCK_FORMAT, block_ildlt.cuh:17-21

// Per-block descriptor as the kernels read it (16 bytes, one load).
struct BlockDesc {
    int row;      // block row
    int col;      // block column
    int val_off;  // first value slot in the value store (dense: r*c, sparse: capacity)
    int cap;      // sparse: capacity in entries (max_nnz); dense: r*c
};

struct Pattern {
    culipx_handle_t* handle = nullptr;
    // the creator's reference plus one per factor / batch made from it through
    // the C ABI; the last release frees the pattern (and releases the handle)
    std::atomic<int> refs{1};
    int n = 0;
    long long nnz = 0;
    int precision = CULIPX_F64;
    int fill_level = 0;
    double fill_factor = 1.0;

    int num_blocks = 0;
    std::vector<int> bs;         // num_blocks + 1
    std::vector<int> row_block;  // n

    int coarse_nnz = 0, fill_nnz = 0;
    std::vector<int> cs_off, cs_col, blk_nnzA;
    std::vector<int> blk_row, blk_col, fmt, max_nnz;
    std::vector<int> csc_off, csc_blk;

    int num_levels = 0;
    std::vector<int> lvl_off, lvl_rows, row_level;
    // every level-0 block row's diagonal block of K is diagonal (no entry
    // between two rows of the same level-0 block row): a level-0 row's K row
    // then reads only itself and rows of later levels
    bool l0_diagonal = false;
    std::vector<int> lb_off, lb;  // factor order per level: pivots, then off-diagonal (CSR order)
    // per row position t of lvl_rows: index of the row's first off-diagonal
    // block inside its level's off-diagonal list
    std::vector<int> row_offdiag_start;
    long long sparse_slots = 0;   // sum of the sparse blocks' capacities
    std::vector<int> sb_off, sb;  // U' sweep order per column level
    int max_level_blocks = 0, max_level_rows = 0;
    int num_sparse = 0, num_dense = 0;

    // value-store layout (level-list order)
    std::vector<BlockDesc> desc;
    long long val_slots = 0;
    // K entry -> value slot (dense: val_off + local; sparse: val_off + running count); -1: lower
    std::vector<int> a_dst;
    std::vector<int> idx_init;   // val_slots entries: sparse local indices of A's entries (-1 unused)
    std::vector<int> nnz_init;   // per block

    DeviceBuffer d_row_offdiag_start, d_lvl_off;
    DeviceBuffer d_cs_off, d_desc, d_bs, d_csc_off, d_csc_blk, d_lb, d_lvl_rows, d_a_dst, d_idx_init,
        d_nnz_init, d_fmt, d_maxnnz, d_row_block;
    long long device_bytes = 0;
};

// Builds the analysis on the host and uploads the device mirror.
int analyze_pattern(culipx_handle_t* h, int n, const int* rowptr, const int* colidx,
                    int num_blocks, const int* block_starts, int fill_level, double fill_factor,
                    int precision, Pattern** out, int num_systems = 1, const int* system_row_offsets = nullptr);

}  // namespace culipx

struct culipx_pattern_t : culipx::Pattern {};
