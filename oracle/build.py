"""Build recipe for the test oracle (TEST INFRASTRUCTURE ONLY).

Produces
  oracle/_build/libcuphu_oracle.so  -- the C restatement (cuphu_oracle.c,
                                       cuphu_oracle_post.c, cuphu_oracle_bridge.c;
                                       gcc, OpenMP,
                                       -ffp-contract=off so only the explicit
                                       fma() calls fuse)
  oracle/_ref/libcuphu_ref.so       -- the reference cuPHU hot-path kernels,
                                       compiled for sm_100a from the sources
                                       where they lie under the reference
                                       checkout, plus ref_harness.cu and the
                                       three-item shim header in ref_shim/.

The reference build is skipped when the reference checkout is absent (the
GPU box uses the prebuilt .so that travels with the repository).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout read by this recipe (and by the CPU tests that
# compare against the reference's own sources); CUPHU_REFERENCE_ROOT moves it
REF_ROOT = os.environ.get("CUPHU_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "src", "cxx", "cuphu")
REF_KERNELS = ["cuphu_util.cu", "cuphu_cost.cu", "cuphu_laplace.cu", "cuphu_phase.cu",
               "cuphu_conncomp.cu", "cuphu_incrcost.cu"]
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_oracle(force: bool = False) -> str:
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "libcuphu_oracle.so")
    srcs = [os.path.join(HERE, n) for n in ("cuphu_oracle.c", "cuphu_oracle_post.c",
                                             "cuphu_oracle_bridge.c")]
    hdr = os.path.join(HERE, "cuphu_oracle.h")
    if force or _stale(out, srcs + [hdr, __file__]):
        _run(["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", "-fopenmp", "-mfma",
              "-ffp-contract=off", "-fno-fast-math", "-o", out, *srcs, "-lm"])
    return out


def build_reference(force: bool = False) -> str | None:
    if not os.path.isdir(REF_SRC):
        return None
    out_dir = os.path.join(HERE, "_ref")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "libcuphu_ref.so")
    srcs = [os.path.join(REF_SRC, k) for k in REF_KERNELS]
    harness = os.path.join(HERE, "ref_harness.cu")
    shim = os.path.join(HERE, "ref_shim")
    deps = srcs + [harness, os.path.join(shim, "snaphu.h"), __file__]
    if force or _stale(out, deps):
        objs = []
        for s in srcs + [harness]:
            o = os.path.join(out_dir, os.path.splitext(os.path.basename(s))[0] + ".o")
            _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "--extended-lambda", "-I" + shim, "-I" + REF_SRC, "-c", s, "-o", o])
            objs.append(o)
        _run([NVCC, *ARCH, "-shared", "--cudart", "static", "-o", out, *objs])
    return out


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_oracle(force))
    print(build_reference(force))
