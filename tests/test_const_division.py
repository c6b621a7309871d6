"""The cost kernels divide by 2 pi and by 7 with a correction step
(Markstein) instead of IEEE division; this checks that arithmetic against
IEEE division on the CPU over the float ranges the kernels use.  The default
run takes every 61st float; CUPHU_EXHAUSTIVE=1 checks every float (about
two minutes with hardware FMA), which is how the ranges were established."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _has_fma():
    try:
        with open("/proc/cpuinfo") as f:
            return " fma " in f.read()
    except OSError:
        return False


def test_division_by_constants_matches_ieee(tmp_path):
    exe = str(tmp_path / "const_div_check")
    flags = ["-O2", "-ffp-contract=off"] + (["-mfma"] if _has_fma() else [])
    try:
        subprocess.run(["gcc", *flags, "-o", exe, os.path.join(HERE, "const_div_check.c"), "-lm"],
                       check=True, capture_output=True)
    except (OSError, subprocess.CalledProcessError) as e:
        pytest.skip(f"gcc unavailable: {e}")
    stride = "1" if os.environ.get("CUPHU_EXHAUSTIVE") else "61"
    out = subprocess.run([exe, stride], check=True, capture_output=True, text=True).stdout
    res = {ln.split()[0]: (int(ln.split()[1]), int(ln.split()[2])) for ln in out.splitlines()}
    assert res["2pi"][0] > 10_000_000 // (1 if stride == "1" else 61) and res["2pi"][1] == 0
    assert res["7"][0] > 10_000_000 // (1 if stride == "1" else 61) and res["7"][1] == 0
