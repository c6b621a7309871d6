"""CPU-only checks: the C-ABI library loads and exports every entry point
declared in include/*.h, struct layouts match the reference header, Python
validation and helper behaviour match the reference tests (test_unwrap.py
:44-80, test_looks.py, test_auto_tiling.py, test_mask_pad_distance.py)."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from oracle.build import REF_ROOT

import cuphu_b200 as cuphu
from cuphu_b200 import _lib
from cuphu_b200._check import check_cost_mode, check_init_method
from cuphu_b200._unwrap import _auto_ntiles_by_target_size, _dilate_mask

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names.update(re.findall(r"\b(cuphu_\w+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_bindings_cover_declared_symbols():
    assert set(_declared_functions()) <= set(_lib.SIGNATURES)


def test_defaults_and_no_gpu_queries():
    p = _lib.default_params()
    assert (p.rhosconst1, p.rhosconst2, p.cstd1, p.cstd2, p.cstd3) == (1.3, 0.14, 0.4, 0.35, 0.06)
    assert (p.costscale, p.nshortcycle, p.sigsqshortmin) == (100.0, 200.0, 1)
    assert (p.kperpdpsi, p.kpardpsi, p.maxncomps, p.conncompthresh) == (7, 7, 32, 300)
    o = _lib.default_solve_options()
    assert o.n_irls == int(os.environ.get("CUPHU_N_IRLS", 16))
    t = _lib.default_tile_params()
    assert (t.ntilerow, t.ntilecol, t.tilecostthresh, t.minregionsize) == (1, 1, 500, 100)
    # a misspelt override is an error, not a silent Python-side attribute
    assert _lib.default_params(nlooks=5.0).nlooks == 5.0
    for make, bad in ((_lib.default_params, "nlook"), (_lib.default_tile_params, "ntilerows"),
                      (_lib.default_solve_options, "nirls")):
        with pytest.raises(TypeError):
            make(**{bad: 1})


REF_H = os.path.join(REF_ROOT, "src/cxx/cuphu/cuphu.h")


@pytest.mark.skipif(not os.path.exists(REF_H), reason="reference header not present")
def test_struct_layout_matches_reference_header(tmp_path):
    fields = {"CuPhuParams": ["nlooks", "sigsqshortmin", "transmitmode", "shadow", "laywidth",
                              "defomax", "kperpdpsi", "p", "cs2scalefactor", "minconncompfrac",
                              "maxncomps"],
              "CuPhuTileParams": ["ntilerow", "nproc", "fix_cycle_spikes"],
              "CuPhuBridgeParams": ["enabled", "ramp_type", "ramp_max_num_sample"]}
    prog = ["#include <stdio.h>", "#include <stddef.h>", "#include HDR", "int main(void){"]
    for s, fs in fields.items():
        prog.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for f in fs:
            prog.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    prog.append("return 0;}")
    src = tmp_path / "l.c"
    src.write_text("\n".join(prog))
    out = {}
    for tag, hdr in (("ref", REF_H), ("ours", os.path.join(ROOT, "include", "cuphu_b200.h"))):
        exe = tmp_path / f"l_{tag}"
        subprocess.run(["gcc", "-x", "c", f'-DHDR="{hdr}"', str(src), "-o", str(exe)], check=True)
        out[tag] = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert out["ref"] == out["ours"]
    assert C.sizeof(_lib.CuPhuParams) == int(out["ours"].split("\n")[0].split()[1])


def test_invalid_cost_and_init():
    with pytest.raises(ValueError, match="cost must be"):
        check_cost_mode("bilinear")
    with pytest.raises(ValueError, match="init must be"):
        check_init_method("dijkstra")


def test_unwrap_validation():
    corr = np.full((50, 60), 0.9, np.float32)
    ig = np.ones((50, 60), np.complex64)
    with pytest.raises(ValueError, match="2-D"):
        cuphu.unwrap(np.ones((2, 50, 60), np.complex64), corr, 10.0)
    with pytest.raises(ValueError, match="shape"):
        cuphu.unwrap(ig, np.ones((10, 10), np.float32), 10.0)
    with pytest.raises(ValueError, match="nlooks"):
        cuphu.unwrap(ig, corr, 0.5)
    with pytest.raises(TypeError, match="complex"):
        cuphu.unwrap(np.ones((50, 60), np.float32), corr, 10.0)
    with pytest.raises(TypeError, match="floating"):
        cuphu.unwrap(ig, np.ones((50, 60), np.int16), 10.0)
    with pytest.raises(NotImplementedError, match="laplace"):
        cuphu.unwrap(ig, corr, 10.0, init="mcf")
    with pytest.raises(NotImplementedError):
        cuphu.unwrap(ig, corr, 10.0, init="laplace", single_tile_reoptimize=True)
    with pytest.raises(ValueError, match="precision"):
        cuphu.unwrap(ig, corr, 10.0, init="laplace", precision="fp16")


def test_effective_looks():
    kw = dict(range_spacing=2.33, azimuth_spacing=2.75, range_resolution=7.5,
              azimuth_resolution=6.0)
    assert cuphu.get_effective_looks(range_looks=13, azimuth_looks=16, **kw) == \
        pytest.approx(29.616888888888894)
    assert cuphu.get_effective_looks(13, 16, 3.0, 4.0, 3.0, 4.0) == pytest.approx(13 * 16)
    n1 = cuphu.get_effective_looks(range_looks=1, azimuth_looks=1, **kw)
    assert cuphu.get_effective_looks(range_looks=2, azimuth_looks=3, **kw) == pytest.approx(6 * n1)


def test_auto_tiling():
    nr, nc = _auto_ntiles_by_target_size(18240, 13162, 1024, 64, 64)
    assert 700 < 18240 / nr < 2000 and 700 < 13162 / nc < 2000 and nr >= nc
    assert _auto_ntiles_by_target_size(200, 200, 1024, 64, 64) == (1, 1)
    assert _auto_ntiles_by_target_size(4096, 4096, 1024, 64, 64) == (4, 4)
    assert _auto_ntiles_by_target_size(8192, 8192, 1024, 64, 64) == (9, 9)


def test_dilate_mask():
    m = np.zeros((21, 21), bool)
    m[10, 10] = True
    g = _dilate_mask(m, 3)
    ys, xs = np.where(g)
    assert (np.abs(ys - 10) + np.abs(xs - 10)).max() == 3
    assert g.sum() == 1 + 4 + 8 + 12
    r = np.random.default_rng(0).random((30, 30)) > 0.5
    assert np.array_equal(_dilate_mask(r, 0), r)


def test_status_errors_on_cpu():
    """Without a GPU the host entry points fail with a CUDA status, never crash."""
    L = _lib.lib()
    if L.cuphu_gpu_count() > 0:
        pytest.skip("a GPU is present")
    res = _lib.CuPhuResult()
    p = _lib.default_params()
    t = _lib.default_tile_params()
    a = np.ones(16, np.float32)
    rc = L.cuphu_unwrap(_lib.ptr(a), _lib.ptr(a), _lib.ptr(a), None, None, 4, 4, 0, 1,
                        C.byref(p), C.byref(t), None, None, 0, C.byref(res))
    assert rc == -4   # init MCF: unsupported, checked before touching CUDA
    rc = L.cuphu_unwrap(_lib.ptr(a), _lib.ptr(a), _lib.ptr(a), None, None, 4, 4, 0, 2,
                        C.byref(p), C.byref(t), None, None, 0, C.byref(res))
    assert rc == -3
    assert L.cuphu_last_error()


def test_new_entry_points_validate_before_touching_cuda():
    """WLS solve/gradient, batch graph and autotuner reject bad arguments
    with CUPHU_ERR_INVALID before any CUDA call (runs without a GPU)."""
    L = _lib.lib()
    o = _lib.default_solve_options()
    p = _lib.default_params()
    t = _lib.default_tile_params()
    a = np.ones(16, np.float32)
    pa = _lib.ptr(a)
    u = np.zeros(16, np.float64)
    pu = _lib.ptr(u)
    # both targets and a right-hand side
    assert L.cuphu_wls_solve_device(pa, pa, pa, pa, pa, None, 4, 4, C.byref(o), pu, None,
                                    None) == -2
    assert b"either" in L.cuphu_last_error()
    # only one of the two target planes
    assert L.cuphu_wls_solve_device(pa, None, None, pa, pa, None, 4, 4, C.byref(o), pu, None,
                                    None) == -2
    # missing weights / output / empty shape
    assert L.cuphu_wls_solve_device(pa, pa, None, None, pa, None, 4, 4, C.byref(o), pu, None,
                                    None) == -2
    assert L.cuphu_wls_solve_device(pa, pa, None, pa, pa, None, 0, 4, C.byref(o), pu, None,
                                    None) == -2
    assert L.cuphu_wls_grad_device(pu, pu, pa, pa, pa, pa, 4, 4, pu, pu, pu, None, None) == -2
    graph = C.c_void_p()
    assert L.cuphu_batch_graph_create(None, 0, 0, C.byref(p), C.byref(o), C.byref(graph)) == -2
    assert L.cuphu_batch_graph_create(None, 1, 0, C.byref(p), C.byref(o), None) == -2
    assert L.cuphu_batch_graph_launch(None, None) == -2
    assert L.cuphu_batch_graph_destroy(None) == 0
    assert L.cuphu_autotune(pa, pa, 1, 4, 0, C.byref(p), C.byref(t), 0, None) == -2
    assert L.cuphu_autotune(pa, pa, 4, 4, 7, C.byref(p), C.byref(t), 0, None) == -2
