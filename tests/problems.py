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
