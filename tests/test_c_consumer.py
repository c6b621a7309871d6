"""The C ABI from plain C, as a non-Python caller (a C program, or a cgo / JNI
shim) uses it: include/cuphu_b200.h compiles as C99, and a program linked
against libcuphu_b200.so reads the defaults and gets a clear status for an
unsupported request without touching a GPU.  CPU only."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "cuphu_b200", "lib")

PROGRAM = r"""
#include <stdio.h>
#include "cuphu_b200.h"

int main(void)
{
    CuPhuParams p;
    CuPhuTileParams t;
    CuPhuSolveOptions o;
    cuphu_default_params(&p);
    cuphu_default_tile_params(&t);
    cuphu_default_solve_options(&o);
    printf("%g %g %ld %d %d %d\n", p.costscale, p.nshortcycle, (long)p.sigsqshortmin,
           t.ntilerow, o.max_iter, o.precision);
    /* MCF initialisation is outside the library: an error status, no exception */
    CuPhuResult r;
    float x[4] = {1, 0, 1, 0}, g[4] = {0.9f, 0.9f, 0.9f, 0.9f};
    int rc = cuphu_unwrap(x, x, g, 0, 0, 2, 2, CUPHU_COST_SMOOTH, CUPHU_INIT_MCF, &p, &t, 0, 0, 0,
                          &r);
    printf("%d %s\n", rc, cuphu_last_error());
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_c_program_uses_the_abi(tmp_path):
    lib = os.path.join(LIB_DIR, "libcuphu_b200.so")
    if not os.path.exists(lib):
        pytest.skip("library not built")
    src = tmp_path / "consumer.c"
    exe = tmp_path / "consumer"
    src.write_text(PROGRAM)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", LIB_DIR, "-lcuphu_b200",
                    "-Wl,-rpath," + LIB_DIR], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True,
                         timeout=120).stdout.splitlines()
    max_iter = str(int(os.environ.get("CUPHU_LAPLACE_MAX_ITER", "1000")))
    assert out[0].split() == ["100", "200", "1", "1", max_iter, "0"]
    rc, msg = out[1].split(" ", 1)
    assert int(rc) == -4 and "laplace" in msg          # CUPHU_ERR_UNSUPPORTED
