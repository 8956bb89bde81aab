"""Builds the culip reference's own solve path from its sources, for sm_100a,
into oracle/_ref/ (git-ignored; the binaries travel to the GPU box with the
tree, the reference sources do not).

TEST INFRASTRUCTURE ONLY: the outputs are the checker of culip_b200 (and of
the C restatement in this folder), never part of the product.

    python oracle/build_ref.py --culip <path to the culip checkout>

Compiled from the culip checkout, unchanged:
  libs/utils/{types.cu, mem_pool.cu, defines.cc}, libs/test/test_instances.cc,
  libs/data_structures/b_kvheap_instances.cc (the memory pool's heap),
  libs/la/{helper_kernels,dense_la,sparse_la,spmv}_instances.cu,
  libs/la/iterative_solvers/sqmr_instances.cu,
  libs/la/preconditioner/block_ildlt_instances.cu,
  apps/block_ildlt/block_ildlt.cc (the reference's own driver).
With the reference's flags (build_parameters_device.cmake: -O3 -lineinfo
-prec-div=true -prec-sqrt=true -rdc=true, OpenMP) plus -std=c++17 (CUDA
12.9's Thrust needs it) and the shim under oracle/ref_shim/ force-included
(legacy cuSPARSE csrmv / csr2csc on the generic API, BLAS/LAPACKE
prototypes, a Matrix Market reader, helper_cuda.h).

Outputs:
  oracle/_ref/ref_dump               the dump driver (oracle/ref_dump.cu)
  oracle/_ref/culip-block-ildlt      apps/block_ildlt as the reference ships it
  oracle/_ref/culip-block-ildlt-b200 the same unmodified driver source compiled
                                     against culip_b200's class facade
                                     (include/culip_la.hpp through
                                     include/culip_compat/) and linked to
                                     culip_b200/lib/libculipx.so: the drop-in
                                     check; nothing of the reference's libs/
                                     is on its include path
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "ref_shim")
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-prec-div=true", "-prec-sqrt=true", "-rdc=true",
         "-Xcompiler", "-fPIC,-fopenmp", "-w"]

REF_SOURCES = [
    "libs/utils/types.cu",
    "libs/utils/mem_pool.cu",
    "libs/utils/defines.cc",
    "libs/data_structures/b_kvheap_instances.cc",
    "libs/test/test_instances.cc",
    "libs/la/helper_kernels_instances.cu",
    "libs/la/dense_la_instances.cu",
    "libs/la/sparse_la_instances.cu",
    "libs/la/spmv_instances.cu",
    "libs/la/iterative_solvers/sqmr_instances.cu",
    "libs/la/preconditioner/block_ildlt_instances.cu",
]
DRIVER = "apps/block_ildlt/block_ildlt.cc"
LIBS = ["-lcublas", "-lcusparse", "-lcusolver", "-lgomp"]


# where the culip checkout sits on the build machine; CULIP_REFERENCE overrides it
_DEFAULT_CHECKOUT = "/root/reference"


def default_checkout() -> str | None:
    """The culip checkout to build from, or None when there is none here."""
    src = os.environ.get("CULIP_REFERENCE", _DEFAULT_CHECKOUT)
    return src if os.path.isfile(os.path.join(src, REF_SOURCES[-1])) else None


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _shim_mtime() -> float:
    return max(os.path.getmtime(os.path.join(SHIM, f)) for f in os.listdir(SHIM))


def _compile(src: str, obj: str, culip: str, dep_m: float) -> str:
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), dep_m):
        return obj
    cmd = [_nvcc(), *ARCH, *FLAGS, "-I", culip, "-I", SHIM, "-include", "culip_ref_shim.h"]
    if src.endswith((".cc", ".cpp")):
        cmd += ["-x", "cu"]
    if src.endswith(".c"):
        cmd = [_nvcc(), "-O2", "-Xcompiler", "-fPIC", "-I", SHIM]
    cmd += ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference build: {os.path.basename(src)} failed:\n{r.stdout}\n{r.stderr[-4000:]}")
    return obj


def build(culip: str, jobs: int | None = None) -> dict:
    culip = os.path.abspath(culip)
    if not os.path.isfile(os.path.join(culip, REF_SOURCES[-1])):
        raise FileNotFoundError(f"{culip} is not a culip checkout")
    os.makedirs(OBJ, exist_ok=True)
    dep_m = _shim_mtime()
    units = [(os.path.join(culip, s), os.path.join(OBJ, s.replace("/", "_") + ".o")) for s in REF_SOURCES]
    units += [(os.path.join(SHIM, "ref_shim.cu"), os.path.join(OBJ, "ref_shim.o")),
              (os.path.join(SHIM, "mmio.c"), os.path.join(OBJ, "mmio.o"))]
    dump = (os.path.join(HERE, "ref_dump.cu"), os.path.join(OBJ, "ref_dump.o"))
    drv = (os.path.join(culip, DRIVER), os.path.join(OBJ, "block_ildlt.o"))
    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda u: _compile(u[0], u[1], culip, dep_m), units + [dump, drv]))
    lib_objs = objs[:len(units)]
    outs = {}
    for name, main_obj in (("ref_dump", objs[-2]), ("culip-block-ildlt", objs[-1])):
        exe = os.path.join(OUT, name)
        newest = max(os.path.getmtime(o) for o in lib_objs + [main_obj])
        if not os.path.exists(exe) or os.path.getmtime(exe) < newest:
            cmd = [_nvcc(), *ARCH, "-rdc=true", "-o", exe, main_obj, *lib_objs, *LIBS]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"reference build: linking {name} failed:\n{r.stdout}\n{r.stderr[-4000:]}")
        outs[name] = exe
    outs["culip-block-ildlt-b200"] = build_facade_driver(culip)
    return outs


def build_facade_driver(culip: str) -> str:
    """apps/block_ildlt/block_ildlt.cc against the culip_b200 facade.  Its
    include root holds only a link to the checkout's apps/ folder, so every
    <libs/...> header it includes comes from include/culip_compat."""
    import tempfile

    repo = os.path.dirname(HERE)
    lib_dir = os.path.join(repo, "culip_b200", "lib")
    if not os.path.exists(os.path.join(lib_dir, "libculipx.so")):
        raise FileNotFoundError("build libculipx.so first (culip_b200/build.py)")
    exe = os.path.join(OUT, "culip-block-ildlt-b200")
    src = os.path.join(culip, DRIVER)
    deps = [src, os.path.join(culip, "apps/block_ildlt/block_ildlt_invariants.h"),
            os.path.join(repo, "include", "culip_la.hpp"), os.path.join(repo, "include", "culipx.h"),
            os.path.join(lib_dir, "libculipx.so")]
    if os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(d) for d in deps):
        return exe
    cuda = os.path.dirname(os.path.dirname(_nvcc()))
    os.makedirs(OUT, exist_ok=True)
    with tempfile.TemporaryDirectory() as root:
        os.symlink(os.path.join(culip, "apps"), os.path.join(root, "apps"))
        cmd = ["g++", "-std=c++17", "-O2", "-w", "-I", os.path.join(repo, "include", "culip_compat"),
               "-I", os.path.join(repo, "include"), "-I", root, "-I", os.path.join(cuda, "include"), src,
               "-o", exe, "-L", lib_dir, "-lculipx", "-Wl,-rpath,$ORIGIN/../../culip_b200/lib",
               "-L", os.path.join(cuda, "lib64"), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"facade driver build failed:\n{r.stdout}\n{r.stderr[-6000:]}")
    return exe


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--culip", default=None, help="path to the culip checkout (read only; default: "
                    "$CULIP_REFERENCE or the build machine's checkout)")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    src = a.culip or default_checkout()
    if not src:
        ap.error("no culip checkout found: pass --culip")
    for k, v in build(src, a.jobs).items():
        print(f"{k}: {v}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
