"""Converts the reference's own test fixtures into compact .npz golden files.

Source: culip's tests/la/data/*.mtx (read from the reference checkout, which
exists only where the fixtures are generated; the .npz files are committed).
  sqmr_{small,big}_{A,prec_L,prec_D,prec_p,prec_s}   tests/la/test_sqmr.cc:192-293
  spmv_{A,K}                                          tests/la/test_spmv.cc:150-210
  bound_rank_*  (patterns and rank bounds)            tests/algorithms/test_bound_rank.cc:55-86
MatrixMarket semantics follow libs/test/test.impl.h: 1-based coordinates,
symmetric files expanded to both triangles (:73-89), rows sorted; dense
"array" vectors read as written (shift 0, :233-290).
Run:  python tests/golden/make_fixtures.py /path/to/culip
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_mtx(path):
    with open(path) as f:
        header = f.readline().lower().split()
        lines = [ln for ln in f if not ln.startswith("%") and ln.strip()]
    if header[2] == "array":
        m, n = map(int, lines[0].split())
        vals = np.array([float(x) for x in lines[1:1 + m * n]])
        return vals
    symmetric = header[4] == "symmetric"
    m, n, nnz = map(int, lines[0].split())
    ii, jj, vv = [], [], []
    for ln in lines[1:1 + nnz]:
        a, b, c = ln.split()[:3]
        ii.append(int(a) - 1)
        jj.append(int(b) - 1)
        vv.append(float(c))
    ii, jj, vv = np.array(ii), np.array(jj), np.array(vv)
    if symmetric:
        off = ii != jj
        ii, jj, vv = np.concatenate([ii, jj[off]]), np.concatenate([jj, ii[off]]), np.concatenate([vv, vv[off]])
    order = np.lexsort((jj, ii))
    ii, jj, vv = ii[order], jj[order], vv[order]
    rowptr = np.zeros(m + 1, np.int64)
    np.add.at(rowptr, ii + 1, 1)
    rowptr = np.cumsum(rowptr)
    return dict(m=m, n=n, rowptr=rowptr.astype(np.int32), colidx=jj.astype(np.int32), val=vv)


def main(root):
    data = os.path.join(root, "tests", "la", "data")
    for case in ("small", "big"):
        A = read_mtx(os.path.join(data, f"sqmr_{case}_A.mtx"))
        L = read_mtx(os.path.join(data, f"sqmr_{case}_prec_L.mtx"))
        D = read_mtx(os.path.join(data, f"sqmr_{case}_prec_D.mtx"))
        p = read_mtx(os.path.join(data, f"sqmr_{case}_prec_p.mtx"))
        s = read_mtx(os.path.join(data, f"sqmr_{case}_prec_s.mtx"))
        np.savez_compressed(os.path.join(HERE, f"sqmr_{case}.npz"),
                            A_rowptr=A["rowptr"], A_colidx=A["colidx"], A_val=A["val"],
                            L_rowptr=L["rowptr"], L_colidx=L["colidx"], L_val=L["val"],
                            D_rowptr=D["rowptr"], D_colidx=D["colidx"], D_val=D["val"],
                            perm=p.astype(np.int32), scale=s)
    for name in ("A", "K"):
        M = read_mtx(os.path.join(data, f"spmv_{name}.mtx"))
        np.savez_compressed(os.path.join(HERE, f"spmv_{name}.npz"), m=M["m"], n=M["n"], rowptr=M["rowptr"],
                            colidx=M["colidx"], val=M["val"])
    # tests/algorithms/test_bound_rank.cc:84-86: the patterns (values are not read) and
    # their rank bounds (BTF lower bound, sprank upper bound)
    for fname, lb, ub in (("bound_rank_51_800", 51, 800), ("bound_rank_920_930", 920, 930),
                          ("bound_rank_4380_4380", 4380, 4380)):
        M = read_mtx(os.path.join(root, "tests", "algorithms", "data", fname + ".mtx"))
        np.savez_compressed(os.path.join(HERE, f"{fname}.npz"), m=M["m"], n=M["n"], rowptr=M["rowptr"],
                            colidx=M["colidx"], lb=lb, ub=ub)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <path to the culip checkout>")
    main(sys.argv[1])
