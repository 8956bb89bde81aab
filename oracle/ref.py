"""The culip reference's own solve path, run as a checker.

TEST INFRASTRUCTURE ONLY: tests (and nothing in the product) call this to run
oracle/_ref/ref_dump -- culip's BlockiLDLt / CSRMatrixSPMV / SQMR compiled
from the reference sources by oracle/build_ref.py -- on one system, and read
back the factor, the preconditioner applies and the SQMR result it computed
on the GPU.  The binary exists only where build_ref.py ran (it travels with
the tree); `available()` says whether it is there.

Factor blocks come back in the reference's own storage (block descriptors,
value and index stores: libs/la/preconditioner/block_ildlt.cuh:32-86,
block_ildlt_kernels.impl.cuh:21-173).  `canonical_blocks` turns them into
{(block_row, block_col): (format, nnz, got_extra, idx, val)} with sparse
entries sorted by local index (row * width + col) and dense blocks as all
rows * width values, the form culip_b200's factor export uses.
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DUMP = os.path.join(HERE, "_ref", "ref_dump")
REF_DRIVER = os.path.join(HERE, "_ref", "culip-block-ildlt")

SOLVE_STRIPE, SOLVE_BLOCK, SOLVE_SCALAR, SOLVE_JACOBI = 0, 1, 2, 3
_KINDS = {0: np.int32, 1: np.float32, 2: np.float64, 3: np.int64}


def available() -> bool:
    return os.path.exists(REF_DUMP) and os.access(REF_DUMP, os.X_OK)


def write_input(path, rowptr, colidx, val, block_starts, is_piv, b):
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    n = len(rowptr) - 1
    bs = np.ascontiguousarray(block_starts, np.int32)
    if bs[-1] != n:
        bs = np.concatenate([bs, [n]]).astype(np.int32)
    with open(path, "wb") as f:
        f.write(np.array([n, len(bs) - 1], np.int32).tobytes())
        f.write(np.array([rowptr[-1]], np.int64).tobytes())
        f.write(rowptr.tobytes())
        f.write(np.ascontiguousarray(colidx, np.int32).tobytes())
        f.write(np.ascontiguousarray(val, np.float64).tobytes())
        f.write(bs.tobytes())
        f.write(np.ascontiguousarray(is_piv, np.int32).tobytes())
        f.write(np.ascontiguousarray(b, np.float64).tobytes())


def read_output(path) -> dict:
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    o = 0
    while o < len(data):
        name = data[o:o + 16].split(b"\0", 1)[0].decode()
        kind = int(np.frombuffer(data, np.int32, 1, o + 16)[0])
        cnt = int(np.frombuffer(data, np.int64, 1, o + 20)[0])
        dt = np.dtype(_KINDS[kind])
        out[name] = np.frombuffer(data, dt, cnt, o + 28).copy()
        o += 28 + cnt * dt.itemsize
    for k in ("residual", "iterations", "true_relres", "symbolic_s", "upload_s", "factor_s", "analysis_s", "sqmr_s",
              "max_level_blks"):
        if k in out:
            out[k] = out[k][0].item()
    out["blocks"] = out["blocks"].reshape(-1, 9)
    return out


def run(rowptr, colidx, val, block_starts, b, is_piv=None, precision=1, pivot=1, fill_level=0, fill_factor=1.0,
        threshold=0.0, tol=1e-8, max_it=1000, algorithm=SOLVE_BLOCK, sweeps=0, repeats=1, timeout=900) -> dict:
    """Runs the reference on one system; precision 1 = double, 0 = float;
    pivot 0 = static, 1 = Bunch-Kaufman (Rook is not run: its search loop has
    no iteration bound)."""
    if not available():
        raise FileNotFoundError(f"{REF_DUMP} is missing (python oracle/build_ref.py --culip <checkout>)")
    n = len(rowptr) - 1
    ip = np.ones(n, np.int32) if is_piv is None else is_piv
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        write_input(fin, rowptr, colidx, val, block_starts, ip, b)
        cmd = [REF_DUMP, fin, fout, str(precision), str(pivot), str(fill_level), repr(float(fill_factor)),
               repr(float(threshold)), repr(float(tol)), str(max_it), str(algorithm), str(sweeps), str(repeats)]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_dump failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        out = read_output(fout)
    out["stdout"] = r.stdout
    return out


def canonical_blocks(ref: dict) -> dict:
    """{(block_row, block_col): (format, nnz, got_extra, idx, val)} of the reference's factor."""
    bs = ref["block_starts"]
    vs, ix = ref["val_store"], ref["ix_store"]
    out = {}
    for bid, fmt, nnz, _max_nnz, got_extra, br, bc, col_ptr, val_ptr in ref["blocks"]:
        h = int(bs[br + 1] - bs[br])
        w = int(bs[bc + 1] - bs[bc])
        if fmt == 1:  # BLOCK_DENSE: rows x width, row-major
            idx = np.arange(h * w, dtype=np.int32)
            val = vs[val_ptr:val_ptr + h * w]
        else:  # BLOCK_SPARSE: nnz (index, value) pairs in any order
            i = ix[col_ptr:col_ptr + nnz]
            v = vs[val_ptr:val_ptr + nnz]
            o = np.argsort(i, kind="stable")
            idx, val = i[o].astype(np.int32), v[o]
        out[(int(br), int(bc))] = (int(fmt), int(nnz), int(got_extra), idx, val)
    return out


def canonical_export(export: dict, blk_row, blk_col, fmt) -> dict:
    """The same form for a culip_b200 (or oracle restatement) factor export,
    whose blocks are listed in block-id order with rows / cols / formats
    given by the pattern."""
    out = {}
    off = export["blk_off"]
    for b in range(len(blk_row)):
        s, e = int(off[b]), int(off[b + 1])
        out[(int(blk_row[b]), int(blk_col[b]))] = (int(fmt[b]), int(export["blk_nnz"][b]),
                                                   int(export["got_extra"][b]), export["idx"][s:e],
                                                   export["val"][s:e])
    return out
