"""bench.schur_update_stats: the sparsity analysis behind the decision not to
put the factorization's Schur updates on tensor cores.  Checked on the C
restatement's factor of the small KKT system (32-row blocks, fill 0 and 1)
against a brute-force count over dense copies of the blocks."""
import os
import sys

import numpy as np
import pytest

import culip_b200 as cb
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
import bench  # noqa: E402


class _P:
    def __init__(self, off, col):
        self._e = {"coarse_off": off, "coarse_col": col}

    def export(self):
        return self._e


class _F:
    def __init__(self, e):
        self._e = e

    def export(self):
        return self._e


@pytest.mark.parametrize("fill", [0, 1])
def test_schur_stats_against_dense_blocks(fill):
    cfg = cb.KKT_CONFIGS["small"]
    n, m = cfg["n"], cfg["m"]
    rp, ci, v = cb.kkt_generate(n, m, cfg["nnz_per_col"], cfg["band_half"], cfg["hmin"], cfg["hmax"])
    N = n + m
    bs = cb.kkt_blocking(n, m, 32)
    bsn = np.asarray(bs) if bs[-1] == N else np.concatenate([bs, [N]])
    S = oracle.Sym(rp, ci, bs, fill, 1.0)
    E = S.factor(v).export()
    rows, cols = np.asarray(S.blk_row), np.asarray(S.blk_col)
    cm = len(bsn) - 1
    off = np.zeros(cm + 1, np.int64)
    np.add.at(off, rows + 1, 1)
    off = np.cumsum(off)
    st = bench.schur_update_stats(_P(off, cols), _F(E), bsn)
    # brute force: dense nonzero masks of the upper off-diagonal blocks
    mask = {}
    for q in range(len(rows)):
        I, J = int(rows[q]), int(cols[q])
        if J <= I:
            continue
        h, w = bsn[I + 1] - bsn[I], bsn[J + 1] - bsn[J]
        M = np.zeros((h, w), bool)
        s0, s1 = E["blk_off"][q], E["blk_off"][q + 1]
        idx, val = E["idx"][s0:s1], E["val"][s0:s1]
        keep = val != 0
        M[idx[keep] // w, idx[keep] % w] = True
        mask[(I, J)] = M
    exists = set(zip(rows.tolist(), cols.tolist()))
    f_alg = f_tile = 0.0
    upd = 0
    for k in range(cm):
        js = sorted(J for (I, J) in mask if I == k)
        for a, i in enumerate(js):
            for j in js[a:]:
                if (i, j) not in exists:
                    continue
                Mi, Mj = mask[(k, i)].astype(float), mask[(k, j)].astype(float)
                f_alg += 2.0 * float((Mi.T @ Mj).sum())
                f_tile += 2.0 * Mi.shape[0] * Mi.shape[1] * Mj.shape[1]
                upd += 1
    assert st["updates"] == upd
    assert st["F_alg"] == f_alg and st["F_tile"] == f_tile
    assert 0.0 < st["F_alg_over_F_tile"] < 0.05
