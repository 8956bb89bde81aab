// Blocking generator for a symmetric sparse pattern (no counterpart in the
// reference, whose driver reads the blocking from a file it does not create:
// apps/block_ildlt/block_ildlt.cc:29-35, "list of first rows in a block and
// number of rows as last element").  Same output contract: block_starts with
// num_blocks + 1 entries, the last one n.
//
// Contiguous blocks, built in one pass over the rows:
//   1. supervariables: maximal runs of consecutive rows whose column sets are
//      equal (rows that a factorization treats alike) are never split unless
//      a run is longer than max_size;
//   2. a block grows run by run up to max_size; once it holds min_size rows it
//      is closed at the first run that has no entry in the block's columns
//      (no coupling the dense diagonal block would capture);
//   3. a last block shorter than min_size is merged into its predecessor when
//      both fit in max_size, else the two are split evenly.
#include "common.h"

#include <algorithm>
#include <vector>

namespace {

bool same_columns(const int* rowptr, const int* colidx, int a, int b)
{
    const int la = rowptr[a + 1] - rowptr[a], lb = rowptr[b + 1] - rowptr[b];
    if (la != lb) return false;
    return std::equal(colidx + rowptr[a], colidx + rowptr[a + 1], colidx + rowptr[b]);
}

// does any row of [r0, r1) have an entry in columns [c0, c1)?
bool coupled(const int* rowptr, const int* colidx, int r0, int r1, int c0, int c1)
{
    for (int r = r0; r < r1; ++r)
        for (int k = rowptr[r]; k < rowptr[r + 1]; ++k)
            if (colidx[k] >= c0 && colidx[k] < c1) return true;
    return false;
}

}  // namespace

extern "C" CULIPX_API int culipx_blocking_generate(int n, const int* h_rowptr, const int* h_colidx, int min_size,
                                                   int max_size, int* h_block_starts, int capacity, int* num_blocks)
{
    using culipx::fail;
    if (n < 0 || (n > 0 && (!h_rowptr || !h_colidx)) || !num_blocks || min_size < 1 || max_size > 32 ||
        min_size > max_size)
        return fail(CULIPX_INVALID_ARG, "culipx_blocking_generate: bad arguments");
    if (n > 0 && h_rowptr[0] != 0) return fail(CULIPX_INVALID_ARG, "culipx_blocking_generate: rowptr[0] != 0");
    for (int r = 0; r < n; ++r) {
        if (h_rowptr[r + 1] < h_rowptr[r]) return fail(CULIPX_INVALID_ARG, "culipx_blocking_generate: rowptr decreases");
        for (int k = h_rowptr[r]; k < h_rowptr[r + 1]; ++k)
            if (h_colidx[k] < 0 || h_colidx[k] >= n || (k > h_rowptr[r] && h_colidx[k] <= h_colidx[k - 1]))
                return fail(CULIPX_INVALID_ARG, "culipx_blocking_generate: columns out of range or unsorted");
    }
    // supervariable runs, split at max_size
    std::vector<int> run_start;
    for (int r = 0; r < n;) {
        int e = r + 1;
        while (e < n && e - r < max_size && same_columns(h_rowptr, h_colidx, e - 1, e)) ++e;
        run_start.push_back(r);
        r = e;
    }
    run_start.push_back(n);
    std::vector<int> starts;
    int b0 = 0, b1 = 0;  // current block [b0, b1)
    for (size_t s = 0; s + 1 < run_start.size(); ++s) {
        const int r0 = run_start[s], r1 = run_start[s + 1];
        if (b1 > b0) {
            const bool full = (b1 - b0) + (r1 - r0) > max_size;
            const bool loose = (b1 - b0) >= min_size && !coupled(h_rowptr, h_colidx, r0, r1, b0, b1);
            if (full || loose) {
                starts.push_back(b0);
                b0 = b1;
            }
        }
        b1 = r1;
    }
    if (b1 > b0) starts.push_back(b0);
    // a short last block: merged or split evenly with its predecessor
    const int nb = (int)starts.size();
    if (nb >= 2) {
        const int last = n - starts[nb - 1], prev = starts[nb - 1] - starts[nb - 2];
        if (last < min_size) {
            if (prev + last <= max_size) {
                starts.pop_back();
            } else {
                starts[nb - 1] = starts[nb - 2] + (prev + last + 1) / 2;
            }
        }
    }
    *num_blocks = (int)starts.size();
    if (!h_block_starts) return CULIPX_OK;
    if (capacity < *num_blocks + 1) return fail(CULIPX_INVALID_ARG, "culipx_blocking_generate: capacity too small");
    std::copy(starts.begin(), starts.end(), h_block_starts);
    h_block_starts[*num_blocks] = n;
    return CULIPX_OK;
}
