"""Builds the CPU oracle (checker) liboracle.so from oracle.c / oracle_sym.c.

Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's CPU
baseline load it; the product library never does.
gcc -O2 -ffp-contract=off keeps every rounding of the restatement explicit.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRCS = [os.path.join(HERE, f) for f in ("oracle.c", "oracle_sym.c")]
DEPS = SRCS + [os.path.join(HERE, f) for f in ("oracle.h", "oracle_num.h")]


def build(verbose: bool = False) -> str:
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in DEPS):
        return LIB
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-fopenmp", "-o", LIB, *SRCS, "-lm"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
