"""Seeded test problems shared by the CPU and GPU tests."""
from __future__ import annotations

import numpy as np

import culip_b200 as cb


def kkt(name: str = "small", seed: int = cb.SEED, **over):
    cfg = dict(cb.KKT_CONFIGS[name])
    cfg.update(over)
    rp, ci, v = cb.kkt_generate(cfg["n"], cfg["m"], cfg["nnz_per_col"], cfg["band_half"], cfg["hmin"], cfg["hmax"],
                                seed=seed)
    bs = cb.kkt_blocking(cfg["n"], cfg["m"], cfg["block"])
    return rp, ci, v, bs


def permute_sym(rp, ci, v, perm):
    """B = P K P' with B[i, j] = K[perm[i], perm[j]] (perm: new -> old), rows sorted."""
    n = len(rp) - 1
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    rows = np.repeat(np.arange(n), np.diff(rp))
    nr, nc = inv[rows], inv[ci]
    order = np.lexsort((nc, nr))
    nr, nc, nv = nr[order], nc[order], v[order]
    nrp = np.zeros(n + 1, np.int32)
    np.add.at(nrp, nr + 1, 1)
    return np.cumsum(nrp).astype(np.int32), nc.astype(np.int32), nv


def random_blocking(n, rng, lo=1, hi=32):
    starts = [0]
    while starts[-1] < n:
        starts.append(min(n, starts[-1] + int(rng.integers(lo, hi + 1))))
    return np.array(starts, np.int32)


def scrambled_kkt(n=300, m=150, k=3, seed=7, block_lo=2, block_hi=12):
    """A small KKT under a random symmetric permutation and random blocking:
    mixed H/A blocks give 2x2 pivots and swaps, deep level schedules and fill."""
    rng = np.random.default_rng(seed)
    rp, ci, v = cb.kkt_generate(n, m, k, 0, 1e-2, 1e2, seed=seed)
    perm = rng.permutation(n + m)
    rp, ci, v = permute_sym(rp, ci, v, perm)
    bs = random_blocking(n + m, rng, block_lo, block_hi)
    return rp, ci, v, bs


def random_spd_ish(n=200, density=0.03, seed=3, indefinite=True):
    """Random symmetric matrix with explicit diagonal (for SpMV / SQMR checks)."""
    rng = np.random.default_rng(seed)
    import scipy.sparse as sp

    A = sp.random(n, n, density=density, random_state=seed, format="csr")
    A = A + A.T
    d = rng.uniform(1, 4, n) * (np.where(rng.random(n) < 0.5, -1, 1) if indefinite else 1)
    A = (A + sp.diags(d * (1 + abs(A).sum(axis=1).A1))).tocsr()
    A.sort_indices()
    return A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)


def planted_pairs(nblocks=20, block=8, eps=1e-5, coupling=1e-3, density=0.05, seed=17):
    """A symmetric matrix whose first nblocks diagonal blocks hold 2x2 pairs
    with d11 d22 = d12^2 (1 - eps) (ratio |det| / (|d11 d22| + d12^2) about
    eps / 2), coupled (entries of size coupling) only to nblocks further
    blocks with a dominant diagonal of 10; is_piv marks the pairs for static
    pivoting.  The paired blocks are level 0 (their pivots see the planted
    values), the others level 1.  Float32-representable values, so an FP32 and
    an FP64 factor see the same matrix."""
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    half = nblocks * block
    n = 2 * half
    rows, cols, vals = [], [], []
    for p in range(0, half, 2):
        a = rng.uniform(0.5, 2.0) * rng.choice([-1.0, 1.0])
        b = rng.uniform(0.5, 2.0) * np.sign(a)
        c = np.sqrt(a * b * (1.0 - eps * rng.uniform(0.5, 1.5))) * rng.choice([-1.0, 1.0])
        rows += [p, p, p + 1, p + 1]
        cols += [p, p + 1, p, p + 1]
        vals += [a, c, c, b]
    for p in range(half, n):
        rows.append(p)
        cols.append(p)
        vals.append(10.0 * rng.choice([-1.0, 1.0]))
    C = sp.random(half, half, density=density, random_state=seed, format="coo")
    r, c, v = C.row, C.col + half, coupling * (2 * C.data - 1)
    rows += list(r) + list(c)
    cols += list(c) + list(r)
    vals += list(v) + list(v)
    K = sp.csr_matrix((np.array(vals, np.float32).astype(np.float64), (rows, cols)), shape=(n, n))
    K.sum_duplicates()
    K.sort_indices()
    bs = np.arange(0, n + 1, block, dtype=np.int32)
    is_piv = np.ones(n, np.int32)
    is_piv[1:half:2] = 0
    return K.indptr.astype(np.int32), K.indices.astype(np.int32), K.data, bs, is_piv
