"""Parity on the benchmark configurations at their full sizes.

* The 512x512 DEFO scene (3 bumps, coherence 0.3-0.95, nlooks 5; one auto
  tile, 16 IRLS passes, FP64 PCG, conncomp at the default threshold) through
  the host-buffer entry point, against the oracle's restatement of the
  reference pipeline on the reference's host phase: bit for bit.
* The same scene through the device's phase kernel (a correctly rounded
  angle instead of the host C library's atan2f): the mismatch counts of
  phase, costs, residues, cycle map and labels against the reference's phase
  are reported and bounded, and the pipeline on the device phase equals the
  oracle on that phase bit for bit (the phase is the only difference).
* The 4096x4096 SMOOTH scene with a 15 % water blob (nlooks 9, 4x4 auto
  tiles, 3 IRLS passes): the SMOOTH costs and the connected components
  against the reference's own kernels on the GPU, and the full tiled FP64
  pipeline against the oracle, bit for bit.

Each case prints one JSON line with its counts.
"""
import ctypes as C
import json

import numpy as np
import pytest

import oracle as O
from cuphu_b200 import synthetic as S
from cuphu_b200._lib import (CuPhuSolveStats, check, default_params, default_solve_options,
                             default_tile_params, lib, ptr)
from cuphu_b200._unwrap import _auto_ntiles_by_target_size
from tests.devbuf import dptr, empty, to_dev, to_host

pytestmark = pytest.mark.gpu

MODE = {"smooth": 0, "defo": 1, "topo": 2}


def unwrap_ex(ig, g, nlooks, mode, ntiles, ovl, precision, n_irls, device_phase=0):
    """cuphu_unwrap_ex (host buffers) without the reference-pixel shift, as
    the reference's C entry point leaves it."""
    nr, nc = g.shape
    ig = np.ascontiguousarray(ig, np.complex64)
    g = np.ascontiguousarray(g, np.float32)
    p = default_params(nlooks=float(nlooks), ncorrlooks=float(nlooks))
    t = default_tile_params(ntilerow=ntiles[0], ntilecol=ntiles[1], rowovrlp=ovl, colovrlp=ovl)
    o = default_solve_options(precision=precision, n_irls=n_irls, ref_row=-1, ref_col=-1,
                              device_phase=device_phase)
    u = np.empty((nr, nc), np.float32)
    c = np.empty((nr, nc), np.uint32)
    st = CuPhuSolveStats()
    check(lib().cuphu_unwrap_ex(ptr(ig.view(np.float32)), ptr(g), None, None, nr, nc, mode,
                                C.byref(p), C.byref(t), C.byref(o), 0, ptr(u), ptr(c),
                                C.byref(st)))
    return u, c, st


def device_phase(torch, ig):
    d_ig = to_dev(np.ascontiguousarray(ig, np.complex64).view(np.float32))
    d_ph = empty(ig.shape, torch.float32)
    check(lib().cuphu_phase_gpu(dptr(d_ig), C.c_longlong(ig.size), dptr(d_ph), None))
    return to_host(d_ph)


def device_costs(torch, ph, g, nlooks, mode):
    nr, nc = ph.shape
    narcs = (nr - 1) * nc + nr * (nc - 1)
    es = 2 if mode == 0 else 4
    d_c = empty((narcs, es), torch.int16)
    d_res = empty((nr - 1, nc - 1), torch.int8)
    p = default_params(nlooks=float(nlooks), ncorrlooks=float(nlooks))
    dph, dg = to_dev(ph), to_dev(g)
    check(lib().cuphu_build_costs_device(dptr(dph), dptr(dg), None, nr, nc, mode, C.byref(p),
                                         dptr(d_c), dptr(d_res), None))
    return to_host(d_c), to_host(d_res)


@pytest.fixture(scope="module")
def c0():
    ig, g, _, ex = S.config_scene("c0_512_defo", seed=0)
    nr, nc = g.shape
    nt = _auto_ntiles_by_target_size(nr, nc, 1024, 64, 64)
    ph = O.phase_from_igram(ig)
    want_u, want_c, _ = O.unwrap_tiled(ph, g, ex["nlooks"], mode=MODE[ex["cost"]], ntiles=nt,
                                       overlap=(64, 64), opts=O.lap_opts(n_irls=16))
    return ig, g, ex, nt, ph, want_u, want_c


def test_c0_512_defo_host_phase_bit_exact(torch_cuda, c0):
    ig, g, ex, nt, ph, want_u, want_c = c0
    u, c, st = unwrap_ex(ig, g, ex["nlooks"], MODE[ex["cost"]], nt, 64, precision=1, n_irls=16)
    print(json.dumps({"case": "c0_512_defo_fp64_host_phase", "tiles": list(nt),
                      "pcg_iterations": st.total_iters,
                      "unw_mismatch": int(np.sum(u.view(np.int32) != want_u.view(np.int32))),
                      "conncomp_mismatch": int(np.sum(c != want_c)),
                      "components": int(want_c.max())}))
    assert np.array_equal(u.view(np.int32), want_u.view(np.int32))
    assert np.array_equal(c, want_c)


def test_c0_512_defo_mixed_vs_oracle(torch_cuda, c0):
    ig, g, ex, nt, ph, want_u, want_c = c0
    u, c, _ = unwrap_ex(ig, g, ex["nlooks"], MODE[ex["cost"]], nt, 64, precision=0, n_irls=16)
    cyc = int(np.sum(np.abs(u.astype(np.float64) - want_u) > np.pi))
    print(json.dumps({"case": "c0_512_defo_mixed", "cycle_mismatches": cyc,
                      "conncomp_mismatch": int(np.sum(c != want_c))}))
    assert cyc <= max(3, int(1e-4 * u.size))


def test_c0_512_defo_device_phase_counts(torch_cuda, c0):
    """The device's correctly rounded phase against the reference's host
    atan2f phase: every difference is one unit in the last place, and the
    downstream differences are counted and bounded."""
    ig, g, ex, nt, ph, want_u, want_c = c0
    mode = MODE[ex["cost"]]
    dph = device_phase(torch_cuda, ig)
    ulp = np.abs(dph.view(np.int32).astype(np.int64) - ph.view(np.int32).astype(np.int64))
    wrapped = np.abs(dph.astype(np.float64) - ph) > np.pi      # 0 <-> 2pi at the wrap point
    ulp[wrapped] = 0
    assert int(ulp.max()) <= 1
    costs_d, res_d = device_costs(torch_cuda, dph, g, ex["nlooks"], mode)
    costs_h = O.build_costs(ph, g, ex["nlooks"], mode=mode)
    res_h = O.residues(ph)
    u, c, _ = unwrap_ex(ig, g, ex["nlooks"], mode, nt, 64, precision=1, n_irls=16, device_phase=1)
    cyc = int(np.sum(np.abs(u.astype(np.float64) - want_u) > np.pi))
    out = {"case": "c0_512_defo_fp64_device_phase", "pixels": int(ph.size),
           "phase_ulp_diffs": int(np.sum(ph.view(np.int32) != dph.view(np.int32))),
           "cost_arc_mismatch": int(np.sum(np.any(costs_d != costs_h, axis=1))),
           "residue_mismatch": int(np.sum(res_d != res_h)),
           "cycle_mismatches": cyc,
           "conncomp_mismatch": int(np.sum(c != want_c))}
    print(json.dumps(out))
    # the phase kernel is the only difference: the oracle on the device phase
    # reproduces the device pipeline bit for bit
    du, dc, _ = O.unwrap_tiled(dph, g, ex["nlooks"], mode=mode, ntiles=nt, overlap=(64, 64),
                               opts=O.lap_opts(n_irls=16))
    assert np.array_equal(u.view(np.int32), du.view(np.int32))
    assert np.array_equal(c, dc)
    assert np.array_equal(costs_d, O.build_costs(dph, g, ex["nlooks"], mode=mode))
    # bounds on the effect of a last-bit phase difference
    assert out["residue_mismatch"] <= max(2, int(1e-5 * res_h.size))
    assert out["cost_arc_mismatch"] <= 0.01 * costs_h.shape[0]
    assert cyc <= max(3, int(1e-4 * ph.size))


@pytest.fixture(scope="module")
def c1():
    ig, g, _, ex = S.config_scene("c1_4096_smooth", seed=0)
    return ig, np.ascontiguousarray(g), ex, O.phase_from_igram(ig)


def test_c1_4096_smooth_costs_vs_reference_kernels(torch_cuda, c1):
    if O.ref_lib() is None:
        pytest.skip("reference kernels not built")
    ig, g, ex, ph = c1
    got, res = device_costs(torch_cuda, ph, g, ex["nlooks"], 0)
    torch_cuda.cuda.empty_cache()
    ref, _ = O.ref_build_costs(ph, g, ex["nlooks"], mode=0)
    print(json.dumps({"case": "c1_4096_smooth_costs", "arcs": int(ref.shape[0]),
                      "mismatch": int(np.sum(np.any(got != ref, axis=1)))}))
    assert np.array_equal(got, ref)
    assert np.array_equal(res, O.residues(ph))


def test_c1_4096_smooth_pipeline_and_conncomp(torch_cuda, c1):
    ig, g, ex, ph = c1
    nr, nc = g.shape
    nt = _auto_ntiles_by_target_size(nr, nc, 1024, 64, 64)
    assert nt == (4, 4)
    u, c, st = unwrap_ex(ig, g, ex["nlooks"], 0, nt, 64, precision=1, n_irls=ex["n_irls"])
    want_u, want_c, _ = O.unwrap_tiled(ph, g, ex["nlooks"], mode=0, ntiles=nt, overlap=(64, 64),
                                       opts=O.lap_opts(n_irls=ex["n_irls"]))
    out = {"case": "c1_4096_smooth_fp64", "tiles": list(nt), "pcg_iterations": st.total_iters,
           "unw_mismatch": int(np.sum(u.view(np.int32) != want_u.view(np.int32))),
           "conncomp_mismatch": int(np.sum(c != want_c)), "components": int(want_c.max())}
    # connected components of the whole unwrapped scene: this build's kernel
    # against the reference's (cuphu_conncomp_gpu) on the same input
    if O.ref_lib() is not None:
        p = default_params(nlooks=float(ex["nlooks"]), ncorrlooks=float(ex["nlooks"]))
        du, dg = to_dev(u), to_dev(g)
        dl = empty((nr, nc), torch_cuda.int32)
        check(lib().cuphu_conncomp_gpu(dptr(du), dptr(dg), None, nr, nc, None, None, C.byref(p),
                                       0, dptr(dl)))
        lab = to_host(dl).view(np.uint32)
        ref = O.ref_conncomp(u, g)
        out["scene_conncomp_mismatch_vs_reference"] = int(np.sum(lab != ref))
        out["scene_components"] = int(ref.max())
    print(json.dumps(out))
    assert np.array_equal(u.view(np.int32), want_u.view(np.int32))
    assert np.array_equal(c, want_c)
    if "scene_conncomp_mismatch_vs_reference" in out:
        assert out["scene_conncomp_mismatch_vs_reference"] == 0
