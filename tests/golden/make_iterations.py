"""Writes sqmr_iterations_<config>.txt: the iteration count of the full FP64
block-iLDLt (BK, fill 0) + SQMR (tol 1e-8, max_it 1000) solve of a seeded
KKT workload, computed by the CPU oracle.  The benchmark's reference arm
times a bounded number of oracle iterations per step and scales them to this
count, so the committed count must come from the full solve.
Run:  python tests/golden/make_iterations.py [small|scale ...]   (scale: minutes)
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main(names):
    import culip_b200 as cb
    import oracle

    for name in names:
        cfg = cb.KKT_CONFIGS[name]
        rp, ci, v = cb.kkt_generate(cfg["n"], cfg["m"], cfg["nnz_per_col"], cfg["band_half"], cfg["hmin"],
                                    cfg["hmax"])
        bs = cb.kkt_blocking(cfg["n"], cfg["m"], cfg["block"])
        b = cb.normal_vector(cb.SEED + 1, len(rp) - 1)
        S = oracle.Sym(rp, ci, bs, 0, 1.0)
        F = S.factor(v)
        _, res, its = oracle.sqmr(rp, ci, v, b, F, 1e-8, 1000)
        with open(os.path.join(HERE, f"sqmr_iterations_{name}.txt"), "w") as f:
            f.write(f"{its}\n")
        print(name, "iterations", its, "residual", res)


if __name__ == "__main__":
    main(sys.argv[1:] or ["small", "scale"])
