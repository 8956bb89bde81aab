"""include/culipx.h is a C ABI: a C99 program (not C++) that includes it
compiles warning-free under -Wall -Wextra -pedantic, links against
libculipx.so and calls the host-only entry points (orderings, KKT
generator), with no GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "culip_b200", "lib")

PROGRAM = r"""
#include <culipx.h>
#include <stdio.h>

int main(void)
{
    /* a 3 x 3 path pattern: rows {1}, {0, 2}, {1} */
    int rp[4] = {0, 1, 3, 4}, ci[4] = {1, 0, 2, 1};
    int perm[3], rmatch[3], cmatch[3], rank = -1;
    if (culipx_ordering_rcm(3, rp, ci, perm) != CULIPX_OK) return 1;
    if (culipx_sprank(3, 3, rp, ci, rmatch, cmatch, &rank) != CULIPX_OK) return 2;
    /* an invalid column is rejected with a status, not a crash */
    ci[0] = 7;
    if (culipx_sprank(3, 3, rp, ci, 0, 0, &rank) != CULIPX_INVALID_ARG) return 3;
    printf("%d %d %d %d %s\n", perm[0], perm[1], perm[2], rank, culipx_last_error() ? "msg" : "none");
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_is_c99_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libculipx.so")):
        pytest.skip("libculipx.so not built")
    src = tmp_path / "abi.c"
    exe = tmp_path / "abi"
    src.write_text(PROGRAM)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                         os.path.join(ROOT, "include"), str(src), "-o", str(exe), "-L", LIBDIR, "-lculipx",
                         f"-Wl,-rpath,{LIBDIR}"], capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, (run.returncode, run.stdout, run.stderr)
    p0, p1, p2, rank, msg = run.stdout.split()
    assert sorted(int(p) for p in (p0, p1, p2)) == [0, 1, 2]
    assert int(rank) == 2 and msg == "msg"
