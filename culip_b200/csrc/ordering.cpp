// Orderings for the block-iLDL' path (host code): the structural rank by a
// maximum bipartite matching, and a reverse Cuthill-McKee ordering.
//
// culipx_sprank mirrors culip's sprank (libs/algorithms/sprank.cuh,
// sprank_instances.cu: an UnweightedBipartiteMatching of rows to columns,
// libs/algorithms/matching.cuh:18-62) -- same arguments, same outputs: the
// number of matched pairs, and per row its matched column / per column its
// matched row, INT_MAX where unmatched (the reference's m_inv_label).  The
// matching here is Hopcroft-Karp (breadth-first layering from the free rows,
// then vertex-disjoint shortest augmenting paths found depth-first with an
// explicit stack), started from a greedy matching; its size is the maximum,
// so the rank equals the reference's, while the pairs themselves may differ
// where several maximum matchings exist.
//
// culipx_ordering_rcm: reverse Cuthill-McKee on the symmetrized pattern
// (i ~ j if A_ij or A_ji is stored, the diagonal ignored).  Each connected
// component starts from a pseudo-peripheral vertex (George-Liu: repeated
// breadth-first searches from the last level's vertex of least degree until
// the eccentricity stops growing, starting at the component's vertex of least
// degree, ties to the lower index); neighbours are visited by increasing
// degree, ties by index; components in order of their lowest vertex; the
// whole order is reversed.  Deterministic.  perm[new] = old (pass
// perm_is_old_to_new = 0 to culipx_permute_create).
#include "common.h"

#include <algorithm>
#include <climits>
#include <vector>

namespace culipx {

namespace {

bool valid_csr(int m, int n, const int* rowptr, const int* colidx)
{
    if (m < 0 || n < 0 || !rowptr || rowptr[0] != 0) return false;
    for (int i = 0; i < m; ++i) {
        if (rowptr[i + 1] < rowptr[i]) return false;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (colidx[k] < 0 || colidx[k] >= n) return false;
    }
    return true;
}

}  // namespace

int sprank(int m, int n, const int* rowptr, const int* colidx, int* row_match, int* col_match, int* rank)
{
    if (!rank || !valid_csr(m, n, rowptr, colidx)) return fail(CULIPX_INVALID_ARG, "culipx_sprank: bad matrix");
    constexpr int kFree = -1;
    std::vector<int> rm(m, kFree), cm(n, kFree);
    int matched = 0;
    // greedy start: the first free column of each row
    for (int i = 0; i < m; ++i)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (cm[colidx[k]] == kFree) {
                rm[i] = colidx[k];
                cm[colidx[k]] = i;
                ++matched;
                break;
            }
    std::vector<int> dist(m), queue(m), it(m), stack;
    stack.reserve(64);
    for (;;) {
        // layers of rows by alternating-path distance from the free rows
        int qh = 0, qt = 0;
        bool found = false;
        for (int i = 0; i < m; ++i) {
            if (rm[i] == kFree) {
                dist[i] = 0;
                queue[qt++] = i;
            } else {
                dist[i] = INT_MAX;
            }
        }
        while (qh < qt) {
            const int i = queue[qh++];
            for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
                const int r = cm[colidx[k]];
                if (r == kFree) found = true;
                else if (dist[r] == INT_MAX) {
                    dist[r] = dist[i] + 1;
                    queue[qt++] = r;
                }
            }
        }
        if (!found) break;
        // vertex-disjoint shortest augmenting paths, depth-first along the layers
        for (int i = 0; i < m; ++i) it[i] = rowptr[i];
        for (int s = 0; s < m; ++s) {
            if (rm[s] != kFree) continue;
            stack.clear();
            stack.push_back(s);
            while (!stack.empty()) {
                const int i = stack.back();
                bool advanced = false;
                while (it[i] < rowptr[i + 1]) {
                    const int c = colidx[it[i]];
                    const int r = cm[c];
                    if (r == kFree) {
                        // augment along the stack: each row takes the column its successor left
                        int col = c;
                        for (int d = (int)stack.size() - 1; d >= 0; --d) {
                            const int row = stack[d];
                            const int prev = rm[row];
                            rm[row] = col;
                            cm[col] = row;
                            col = prev;
                        }
                        ++matched;
                        for (int row : stack) dist[row] = INT_MAX;  // used: off the layers
                        stack.clear();
                        advanced = true;
                        break;
                    }
                    if (dist[r] == dist[i] + 1) {
                        ++it[i];
                        stack.push_back(r);
                        advanced = true;
                        break;
                    }
                    ++it[i];
                }
                if (!advanced) {
                    dist[i] = INT_MAX;  // dead end
                    stack.pop_back();
                }
            }
        }
    }
    if (row_match)
        for (int i = 0; i < m; ++i) row_match[i] = rm[i] == kFree ? INT_MAX : rm[i];
    if (col_match)
        for (int j = 0; j < n; ++j) col_match[j] = cm[j] == kFree ? INT_MAX : cm[j];
    *rank = matched;
    return CULIPX_OK;
}

int ordering_rcm(int n, const int* rowptr, const int* colidx, int* perm)
{
    if (!perm || !valid_csr(n, n, rowptr, colidx)) return fail(CULIPX_INVALID_ARG, "culipx_ordering_rcm: bad matrix");
    // symmetrized adjacency without the diagonal, neighbours sorted and unique
    std::vector<int> deg(n + 1, 0);
    for (int i = 0; i < n; ++i)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (colidx[k] != i) {
                ++deg[i + 1];
                ++deg[colidx[k] + 1];
            }
    for (int i = 0; i < n; ++i) deg[i + 1] += deg[i];
    std::vector<int> adj(deg[n]);
    {
        std::vector<int> pos(deg.begin(), deg.end() - 1);
        for (int i = 0; i < n; ++i)
            for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
                if (colidx[k] != i) {
                    adj[pos[i]++] = colidx[k];
                    adj[pos[colidx[k]]++] = i;
                }
    }
    std::vector<int> off(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        auto b = adj.begin() + deg[i], e = adj.begin() + deg[i + 1];
        std::sort(b, e);
        off[i + 1] = off[i] + (int)(std::unique(b, e) - b);
    }
    {
        std::vector<int> packed(off[n]);
        for (int i = 0; i < n; ++i) std::copy(adj.begin() + deg[i], adj.begin() + deg[i] + (off[i + 1] - off[i]),
                                              packed.begin() + off[i]);
        adj.swap(packed);
    }
    auto degree = [&](int v) { return off[v + 1] - off[v]; };
    // neighbours by increasing degree, ties by index
    for (int i = 0; i < n; ++i)
        std::stable_sort(adj.begin() + off[i], adj.begin() + off[i + 1],
                         [&](int a, int b) { return degree(a) < degree(b); });

    std::vector<int> order, level(n, -1), comp(n, 0);
    order.reserve(n);
    std::vector<int> bfs;
    bfs.reserve(n);
    // breadth-first levels from root inside the unnumbered part; returns the
    // eccentricity and leaves the visit order in bfs
    auto levels = [&](int root, int stamp) {
        bfs.clear();
        bfs.push_back(root);
        comp[root] = stamp;
        level[root] = 0;
        int ecc = 0;
        for (size_t h = 0; h < bfs.size(); ++h) {
            const int v = bfs[h];
            for (int k = off[v]; k < off[v + 1]; ++k) {
                const int w = adj[k];
                if (comp[w] == stamp || comp[w] < 0) continue;  // seen this round / already numbered
                comp[w] = stamp;
                level[w] = level[v] + 1;
                ecc = std::max(ecc, level[w]);
                bfs.push_back(w);
            }
        }
        return ecc;
    };
    int stamp = 0;
    for (int s = 0; s < n; ++s) {
        if (comp[s] < 0) continue;  // numbered
        // the component's vertex of least degree
        int root = s;
        int ecc = levels(s, ++stamp);
        for (int v : bfs)
            if (degree(v) < degree(root) || (degree(v) == degree(root) && v < root)) root = v;
        ecc = levels(root, ++stamp);
        for (;;) {
            int cand = -1;
            for (int v : bfs)
                if (level[v] == ecc &&
                    (cand < 0 || degree(v) < degree(cand) || (degree(v) == degree(cand) && v < cand)))
                    cand = v;
            const int e2 = levels(cand, ++stamp);
            if (e2 <= ecc) break;
            root = cand;
            ecc = e2;
        }
        // Cuthill-McKee from root
        const size_t first = order.size();
        order.push_back(root);
        comp[root] = -1;
        for (size_t h = first; h < order.size(); ++h) {
            const int v = order[h];
            for (int k = off[v]; k < off[v + 1]; ++k) {
                const int w = adj[k];
                if (comp[w] < 0) continue;
                comp[w] = -1;
                order.push_back(w);
            }
        }
    }
    for (int i = 0; i < n; ++i) perm[i] = order[n - 1 - i];
    return CULIPX_OK;
}

}  // namespace culipx

extern "C" {

CULIPX_API int culipx_sprank(int m, int n, const int* rowptr, const int* colidx, int* row_match, int* col_match,
                             int* rank)
{
    try {
        return culipx::sprank(m, n, rowptr, colidx, row_match, col_match, rank);
    } catch (...) {
        return culipx::fail(CULIPX_OOM, "culipx_sprank: host allocation failed");
    }
}

CULIPX_API int culipx_ordering_rcm(int n, const int* rowptr, const int* colidx, int* perm)
{
    try {
        return culipx::ordering_rcm(n, rowptr, colidx, perm);
    } catch (...) {
        return culipx::fail(CULIPX_OOM, "culipx_ordering_rcm: host allocation failed");
    }
}

}  // extern "C"
