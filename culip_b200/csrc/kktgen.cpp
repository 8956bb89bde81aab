// Seeded synthetic KKT systems K = [[H + delta I, A'], [A, -gamma I]] from
// interior-point steps, the blocking that feeds the block-iLDL^T analysis, and
// N(0,1) right-hand sides.  The reference ships no generator (its driver
// reads matrix, permutation, blocking and pivot files,
// apps/block_ildlt/block_ildlt.cc:29-35); this module defines the inputs all
// measurements use.
//
// RNG: std::mt19937_64; uniforms are the top 53 bits scaled to [0, 1);
// normals come from a Box-Muller transform written here (std::normal_distribution
// is implementation-defined), consumed in pairs.
#include "common.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

namespace {

struct Rng {
    std::mt19937_64 eng;
    bool have_spare = false;
    double spare = 0.0;
    explicit Rng(uint64_t seed) : eng(seed) {}
    double uniform() { return (double)(eng() >> 11) * (1.0 / 9007199254740992.0); }
    double normal()
    {
        if (have_spare) { have_spare = false; return spare; }
        double u1;
        do { u1 = uniform(); } while (u1 <= 0.0);
        const double u2 = uniform();
        const double rad = std::sqrt(-2.0 * std::log(u1));
        const double ang = 6.283185307179586476925286766559 * u2;
        spare = rad * std::sin(ang);
        have_spare = true;
        return rad * std::cos(ang);
    }
    int below(int n) { return (int)(uniform() * (double)n); }
};

}  // namespace

extern "C" {

CULIPX_API int culipx_kkt_nnz(const culipx_kkt_spec* spec, long long* nnz_out)
{
    if (!spec || !nnz_out || spec->n <= 0 || spec->m < 0 || spec->nnz_per_col < 0 ||
        spec->nnz_per_col > spec->m)
        return culipx::fail(CULIPX_INVALID_ARG, "culipx_kkt_nnz: bad spec");
    *nnz_out = (long long)spec->n + spec->m + 2LL * spec->n * spec->nnz_per_col;
    return CULIPX_OK;
}

// A (m x n): per column j, nnz_per_col distinct rows.  band_half > 0: the first
// ceil(k/2) rows come from [floor(j*m/n) - band_half, floor(j*m/n) + band_half - 1]
// clipped to [0, m), the rest uniform; duplicates are rejected and redrawn.
// H diagonal log-uniform in [hmin, hmax]; values of A are N(0,1).
// Draw order: H (n uniforms), then per column its rows, then its values.
CULIPX_API int culipx_kkt_generate(const culipx_kkt_spec* spec, int* rowptr, int* colidx,
                                   double* val)
{
    long long nnz = 0;
    int st = culipx_kkt_nnz(spec, &nnz);
    if (st) return st;
    if (!rowptr || !colidx || !val) return culipx::fail(CULIPX_INVALID_ARG, "culipx_kkt_generate: null output");
    if (nnz > 0x7fffffffLL) return culipx::fail(CULIPX_INVALID_ARG, "culipx_kkt_generate: nnz exceeds int32");
    const int n = spec->n, m = spec->m, k = spec->nnz_per_col;
    const int N = n + m;
    Rng rng(spec->seed);

    std::vector<double> h(n);
    const double la = std::log10(spec->hmin), lb = std::log10(spec->hmax);
    for (int j = 0; j < n; ++j) h[j] = std::pow(10.0, la + (lb - la) * rng.uniform());

    // columns of A: (row, value) sorted by row
    std::vector<int> acol_ptr(n + 1, 0);
    std::vector<int> arow((size_t)n * k);
    std::vector<double> aval((size_t)n * k);
    std::vector<int> rows(k);
    const int nband = (spec->band_half > 0) ? (k + 1) / 2 : 0;
    for (int j = 0; j < n; ++j) {
        int got = 0;
        const long long center = (long long)j * m / n;
        const int lo = (int)std::max<long long>(0, center - spec->band_half);
        const int hi = (int)std::min<long long>(m, center + spec->band_half);  // exclusive
        while (got < k) {
            int r;
            if (got < nband && hi > lo) r = lo + rng.below(hi - lo);
            else r = rng.below(m);
            bool dup = false;
            for (int t = 0; t < got; ++t) dup |= (rows[t] == r);
            if (!dup) rows[got++] = r;
        }
        std::sort(rows.begin(), rows.end());
        for (int t = 0; t < k; ++t) {
            arow[(size_t)j * k + t] = rows[t];
            aval[(size_t)j * k + t] = rng.normal();
        }
    }

    // full symmetric CSR: rows 0..n-1: [H+delta]_jj then A(:,j)' at columns n + r;
    // rows n..N-1: A(r,:) at columns j, then -gamma on the diagonal.
    std::vector<int> rcount(m, 0);
    for (size_t t = 0; t < arow.size(); ++t) rcount[arow[t]]++;
    rowptr[0] = 0;
    for (int j = 0; j < n; ++j) rowptr[j + 1] = rowptr[j] + 1 + k;
    for (int r = 0; r < m; ++r) rowptr[n + r + 1] = rowptr[n + r] + rcount[r] + 1;
    for (int j = 0; j < n; ++j) {
        int p = rowptr[j];
        colidx[p] = j;
        val[p] = h[j] + spec->delta;
        ++p;
        for (int t = 0; t < k; ++t) {
            colidx[p] = n + arow[(size_t)j * k + t];
            val[p] = aval[(size_t)j * k + t];
            ++p;
        }
    }
    std::vector<int> fillp(m);
    for (int r = 0; r < m; ++r) fillp[r] = rowptr[n + r];
    for (int j = 0; j < n; ++j)  // columns ascending -> each A row's entries sorted
        for (int t = 0; t < k; ++t) {
            const int r = arow[(size_t)j * k + t];
            colidx[fillp[r]] = j;
            val[fillp[r]] = aval[(size_t)j * k + t];
            fillp[r]++;
        }
    for (int r = 0; r < m; ++r) {
        colidx[fillp[r]] = n + r;
        val[fillp[r]] = -spec->gamma;
    }
    (void)N;
    return CULIPX_OK;
}

// Contiguous diagonal blocks of size `block` over [0, n) and [n, n+m) that never
// straddle row n.  A part whose last block would be shorter than min(8, block)
// splits its last two blocks evenly instead (sizes stay in [8, 32] for block 32).
// Writes block_starts[0..num_blocks] (last entry n + m).
CULIPX_API int culipx_kkt_blocking(int n, int m, int block, int* block_starts, int capacity,
                                   int* num_blocks)
{
    if (n < 0 || m < 0 || block < 1 || block > 32 || !num_blocks)
        return culipx::fail(CULIPX_INVALID_ARG, "culipx_kkt_blocking: bad arguments");
    std::vector<int> starts;
    auto part = [&](int from, int len) {
        if (len <= 0) return;
        const int nb = (len + block - 1) / block;
        const int last = len - (nb - 1) * block;
        const int minsz = std::min(8, block);
        if (nb >= 2 && last < minsz) {
            for (int b = 0; b < nb - 2; ++b) starts.push_back(from + b * block);
            const int rest = block + last;
            const int first = (rest + 1) / 2;
            starts.push_back(from + (nb - 2) * block);
            starts.push_back(from + (nb - 2) * block + first);
        } else {
            for (int b = 0; b < nb; ++b) starts.push_back(from + b * block);
        }
    };
    part(0, n);
    part(n, m);
    const int nbk = (int)starts.size();
    *num_blocks = nbk;
    if (!block_starts) return CULIPX_OK;
    if (capacity < nbk + 1) return culipx::fail(CULIPX_INVALID_ARG, "culipx_kkt_blocking: capacity too small");
    for (int b = 0; b < nbk; ++b) block_starts[b] = starts[b];
    block_starts[nbk] = n + m;
    return CULIPX_OK;
}

CULIPX_API int culipx_normal_vector(unsigned long long seed, long long len, double* out)
{
    if (len < 0 || (len > 0 && !out)) return culipx::fail(CULIPX_INVALID_ARG, "culipx_normal_vector: bad arguments");
    Rng rng(seed);
    for (long long i = 0; i < len; ++i) out[i] = rng.normal();
    return CULIPX_OK;
}

}  // extern "C"
