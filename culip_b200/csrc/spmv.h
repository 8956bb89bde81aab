// CSR operator (borrowed device arrays) and its SpMV.
#pragma once

#include "device.h"

namespace culipx {

// SELL-32-sigma copy of a CSR matrix: the rows of at most kSellMaxRow
// entries, sorted by decreasing length inside windows of kSellWindow rows,
// form slices of 32; entry j of a slice's 32 rows is stored contiguously
// (slot slice_off[s] + 32 j + lane), each row's entries in column order,
// padded with col = -1 to the slice's longest row.  A thread still sums its
// own row serially in column order (bit-identical to the CSR loop) while a
// warp's index and value loads are contiguous.  Longer rows follow the slices
// in CSR order (a warp each; long_off[i] is the first slot of long row i), so
// the copy holds every value it reads.
struct Sell {
    bool built = false;
    int nslices = 0, nrows = 0, nlong = 0;
    long long slots = 0;     // slice slots, then the long rows' entries
    DeviceBuffer rows;       // nslices * 32 row ids (-1 past the end)
    DeviceBuffer slice_off;  // long long per slice
    DeviceBuffer slice_len;  // int per slice
    DeviceBuffer col;        // int per slot (-1: padding)
    DeviceBuffer map;        // long long per slot: position in the CSR arrays (-1: padding)
    DeviceBuffer val;        // value per slot (the matrix precision)
    DeviceBuffer long_rows;  // rows of more than kSellMaxRow entries
    DeviceBuffer long_off;   // long long per long row + 1: their first slots
};

constexpr int kSellMaxRow = 64;
constexpr int kSellWindow = 256;

struct Csr {
    culipx_handle_t* h = nullptr;
    unsigned long long serial = next_serial();
    int m = 0, n = 0;
    long long nnz = 0;
    const int* rowptr = nullptr;
    const int* colidx = nullptr;
    const void* val = nullptr;
    int precision = CULIPX_F64;
    bool has_t = false;
    DeviceBuffer t_rowptr, t_colidx, t_val;  // explicit transpose (owned)
    Sell sell;                               // culipx_csr_set_format(CULIPX_FMT_SELL)
};

int csr_build_transpose(Csr* A);
// builds the SELL-32 copy (structure from the CSR arrays, values gathered)
int csr_build_sell(Csr* A);
// re-gathers the SELL copy's values from the CSR value array
int csr_refresh_sell(Csr* A, cudaStream_t s);
int csr_spmv(Csr* A, const void* x, void* y, double alpha, double beta, int transpose, cudaStream_t s);

}  // namespace culipx

struct culipx_csr_t : culipx::Csr {};
