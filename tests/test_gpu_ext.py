"""The reference-signature entry points on the GPU.

* ``_cuphu_ext.unwrap_arrays`` (the module the reference's ``_unwrap.py``
  drives) reaches ``cuphu_unwrap`` with split planes and callee-allocated
  results; its outputs equal ``cuphu_b200.unwrap``'s (``cuphu_unwrap_ex``)
  bit for bit, and the reference-pixel shift that ``cuphu_b200.unwrap``
  applies on the device equals the reference's Python formula
  (_unwrap.py:605-617) applied to the unshifted output.
* ``cuphu_unwrap`` in FP64 equals the oracle's pipeline on the reference's
  host phase bit for bit.
* ``_cuphu_ext.build_costs`` / ``cuphu_build_costs_gpu`` return the
  reference kernels' cost bytes on the same interferogram.
* The launcher-level ``cuphu_build_smooth_costs_gpu`` /
  ``cuphu_build_defo_costs_gpu`` (device output allocated by the callee) and
  ``cuphu_laplace_unwrap_gpu`` against this build's own device entry points.
"""
import ctypes as C

import numpy as np
import pytest

import cuphu_b200
import oracle as O
from cuphu_b200 import _cuphu_ext
from cuphu_b200 import synthetic as S
from cuphu_b200._lib import (CuPhuResult, CuPhuSolveStats, check, default_params,
                             default_solve_options, default_tile_params, lib, ptr)
from tests.devbuf import dptr, empty, to_dev, to_host

pytestmark = pytest.mark.gpu


def scene(nr=150, nc=170, seed=12):
    ig, g, _, _ = S.bumps(nr, nc, seed=seed, nbumps=3, amp_range=(10, 30), sigma_range=(12, 35))
    return ig, g


def test_unwrap_arrays_equals_unwrap(torch_cuda):
    ig, g = scene()
    u1, c1 = _cuphu_ext.unwrap_arrays(ig, g, 5.0, cost="defo", init="laplace", ntilerow=2,
                                      ntilecol=2, tile_rowovrlp=16, tile_colovrlp=16)
    u2, c2 = cuphu_b200.unwrap(ig, g, 5.0, cost="defo", init="laplace", ntiles=(2, 2),
                               tile_overlap=16, reference_pixel=None)
    assert u1.dtype == np.float32 and c1.dtype == np.uint32
    assert np.array_equal(u1.view(np.int32), u2.view(np.int32))
    assert np.array_equal(c1, c2)


@pytest.mark.parametrize("rp", [(0, 0), (77, 131)])
def test_reference_pixel_shift_matches_the_reference_formula(torch_cuda, rp):
    ig, g = scene(seed=13)
    base, _ = cuphu_b200.unwrap(ig, g, 5.0, init="laplace", reference_pixel=None)
    got, _ = cuphu_b200.unwrap(ig, g, 5.0, init="laplace", reference_pixel=rp)
    # _unwrap.py:605-617 on the unshifted output
    ref_phase = float(np.angle(np.ascontiguousarray(ig, np.complex64)[rp]))
    if ref_phase < 0.0:
        ref_phase += 2.0 * np.pi
    n = round((float(base[rp]) - ref_phase) / (2.0 * np.pi))
    want = base - np.float32(n * 2.0 * np.pi) if n != 0 else base
    assert np.array_equal(got.view(np.int32), want.view(np.int32))


def test_cuphu_unwrap_reference_abi(torch_cuda, monkeypatch):
    """cuphu_unwrap (split planes, callee-allocated results, solver knobs
    from the reference's environment variables) gives cuphu_unwrap_ex's
    output for the same job; both take the reference's host phase, so in FP64
    the oracle on O.phase_from_igram is the exact expectation."""
    ig, g = scene(96, 128, seed=14)
    nr, nc = g.shape
    monkeypatch.setenv("CUPHU_N_IRLS", "3")
    ig = np.ascontiguousarray(ig, np.complex64)
    re, im = np.ascontiguousarray(ig.real), np.ascontiguousarray(ig.imag)
    p = default_params(nlooks=5.0, ncorrlooks=5.0)
    t = default_tile_params(ntilerow=2, ntilecol=1, rowovrlp=12, colovrlp=0)
    res = CuPhuResult()
    check(lib().cuphu_unwrap(ptr(re), ptr(im), ptr(g), None, None, nr, nc, 1, 2, C.byref(p),
                             C.byref(t), None, None, 0, C.byref(res)))
    n = nr * nc
    u = np.ctypeslib.as_array(C.cast(res.unw, C.POINTER(C.c_float)), (n,)).reshape(nr, nc).copy()
    c = np.ctypeslib.as_array(C.cast(res.conncomp, C.POINTER(C.c_uint32)), (n,)).reshape(nr,
                                                                                          nc).copy()
    _cuphu_ext._free(C.cast(res.unw, C.c_void_p))
    _cuphu_ext._free(C.cast(res.conncomp, C.c_void_p))
    # the same job through cuphu_unwrap_ex (mixed default): identical
    o = default_solve_options(ref_row=-1, ref_col=-1)
    u2 = np.empty((nr, nc), np.float32)
    c2 = np.empty((nr, nc), np.uint32)
    check(lib().cuphu_unwrap_ex(ptr(ig.view(np.float32)), ptr(g), None, None, nr, nc, 1,
                                C.byref(p), C.byref(t), C.byref(o), 0, ptr(u2), ptr(c2), None))
    assert np.array_equal(u.view(np.int32), u2.view(np.int32))
    assert np.array_equal(c, c2)
    # FP64 through the same host phase equals the oracle bit for bit
    o64 = default_solve_options(precision=1, ref_row=-1, ref_col=-1)
    check(lib().cuphu_unwrap_ex(ptr(ig.view(np.float32)), ptr(g), None, None, nr, nc, 1,
                                C.byref(p), C.byref(t), C.byref(o64), 0, ptr(u2), ptr(c2), None))
    want_u, want_c, _ = O.unwrap_tiled(O.phase_from_igram(ig), g, 5.0, mode=1, ntiles=(2, 1),
                                       overlap=(12, 0), opts=O.lap_opts(n_irls=3))
    assert np.array_equal(u2.view(np.int32), want_u.view(np.int32))
    assert np.array_equal(c2, want_c)


@pytest.mark.parametrize("cost,mode", [("smooth", 0), ("defo", 1), ("topo", 1)])
def test_build_costs_bytes_equal_reference_kernels(torch_cuda, cost, mode):
    if O.ref_lib() is None:
        pytest.skip("reference kernels not built")
    ig, g = scene(130, 90, seed=15)
    got = _cuphu_ext.build_costs(ig, g, 5.0, cost=cost)
    ref, _ = O.ref_build_costs(O.phase_from_igram(ig), g, 5.0, mode=mode)
    assert got.dtype == np.uint8
    assert np.array_equal(got, ref.view(np.uint8).ravel())


def _cudart():
    """The CUDA runtime torch has loaded, for raw-pointer copies and frees
    of buffers the library allocates."""
    rt = C.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    rt.cudaFree.argtypes = [C.c_void_p]
    return rt


@pytest.mark.parametrize("mode", [0, 1])
def test_launcher_cost_entry_points(torch_cuda, mode):
    """cuphu_build_{smooth,defo}_costs_gpu allocate the cost buffer on the
    stream (the caller frees it) and fill it with the reference kernels'
    bytes."""
    if O.ref_lib() is None:
        pytest.skip("reference kernels not built")
    ig, g = scene(70, 95, seed=16)
    ph = O.phase_from_igram(ig)
    nr, nc = ph.shape
    narcs = (nr - 1) * nc + nr * (nc - 1)
    es = 2 if mode == 0 else 4
    dph, dg = to_dev(ph), to_dev(g)
    p = default_params(nlooks=5.0, ncorrlooks=5.0)
    out = C.c_void_p()
    fn = lib().cuphu_build_smooth_costs_gpu if mode == 0 else lib().cuphu_build_defo_costs_gpu
    check(fn(dptr(dph), dptr(dg), None, None, nr, nc, C.byref(p), 7, 7, C.byref(out), None))
    torch_cuda.cuda.synchronize()
    host = np.empty((narcs, es), np.int16)
    rt = _cudart()
    assert rt.cudaMemcpy(host.ctypes.data, out, host.nbytes, 2) == 0   # device to host
    assert rt.cudaFree(out) == 0
    ref, _ = O.ref_build_costs(ph, g, 5.0, mode=mode)
    assert np.array_equal(host, ref)


def test_laplace_unwrap_gpu_equals_device_solve(torch_cuda):
    ig, g = scene(120, 100, seed=17)
    ph = O.phase_from_igram(ig)
    nr, nc = ph.shape
    costs = O.build_costs(ph, g, 5.0, mode=0)
    dcost, dph = to_dev(costs), to_dev(ph)
    du = empty((nr, nc), torch_cuda.float32)
    check(lib().cuphu_laplace_unwrap_gpu(dptr(dcost), dptr(dph), nr, nc, 200.0, 1000, 1e-3, 0,
                                         dptr(du), None))
    got = to_host(du)
    du2 = empty((nr, nc), torch_cuda.float32)
    o = default_solve_options()
    st = CuPhuSolveStats()
    check(lib().cuphu_laplace_solve_device(dptr(dcost), 2, dptr(dph), nr, nc, C.byref(o),
                                           dptr(du2), None, None, C.byref(st), None))
    assert np.array_equal(got.view(np.int32), to_host(du2).view(np.int32))


def test_gpu_info_keys(torch_cuda):
    info = _cuphu_ext.gpu_info(0)
    assert set(info) == {"name", "total_memory", "sm_count", "compute_cap"}
    assert info["sm_count"] > 0 and info["compute_cap"].count(".") == 1
    assert _cuphu_ext.gpu_count() >= 1
    assert _cuphu_ext.gpu_name(0) == info["name"]
