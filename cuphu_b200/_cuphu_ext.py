"""``_cuphu_ext``-compatible module over libcuphu_b200.

The reference's Python layer reaches its CUDA code through one extension
module, ``cuphu._cuphu_ext`` (pybind11, src/cxx/cuphu/cuphu_py.cu:460-638),
imported by ``cuphu/_ext.py``.  This module offers the same functions with
the same keyword names, defaults, return types and error types, implemented
with ctypes over this build's C ABI, so the reference's unmodified
``_unwrap.py``, ``_gpu.py`` and callers of ``build_costs`` run on
libcuphu_b200 when it is installed as ``cuphu._cuphu_ext``::

    import sys, cuphu_b200._cuphu_ext as ext
    sys.modules["cuphu._cuphu_ext"] = ext      # before importing cuphu

* ``unwrap_arrays`` -> ``cuphu_unwrap`` (the reference's C entry point:
  split real/imaginary planes, callee-allocated results, cuphu_py.cu:113-256).
* ``build_costs`` -> ``cuphu_build_costs_gpu`` (raw SNAPHU cost bytes,
  cuphu_py.cu:260-314).
* ``gpu_count`` / ``gpu_name`` / ``gpu_info`` (cuphu_py.cu:435-456).

Options whose implementation needs SNAPHU's CPU network-flow solver
(``init='mcf'``/``'mst'``, ``single_tile_reoptimize``) raise
NotImplementedError: an option is never dropped silently.  The post-passes
``laplace_neighbor_feedback``, ``fix_cycle_spikes`` and ``bridge`` run on the
device, with their test hooks.  Failures of the
library raise RuntimeError, as the reference's C++ exceptions surface
through pybind11.
"""
from __future__ import annotations

import ctypes as C
import ctypes.util

import numpy as np

from cuphu_b200._lib import (CuPhuBridgeParams, CuPhuResult, check, default_params,
                             default_tile_params, lib, ptr)
from cuphu_b200 import _gpu

__all__ = ["unwrap_arrays", "build_costs", "gpu_count", "gpu_name", "gpu_info"]

# SNAPHU's documented configuration defaults, which the reference binds as
# the DEF_* keyword defaults of unwrap_arrays / build_costs
_DEF_COSTSCALE = 100.0
_DEF_NSHORTCYCLE = 200
_DEF_KPERPDPSI = 7
_DEF_KPARDPSI = 7
_DEF_DEFOMAX = 1.2
_DEF_MINCONNCOMPFRAC = 0.01
_DEF_MAXNCOMPS = 32
_DEF_CONNCOMPTHRESH = 300
_DEF_TILECOSTTHRESH = 500
_DEF_MINREGIONSIZE = 100

_COST = {"smooth": 0, "defo": 1, "topo": 2}
_INIT = {"mst": 0, "mcf": 1, "laplace": 2}
_COST_MSG = "cost must be 'smooth', 'defo', or 'topo'"
_INIT_MSG = "init must be 'mst', 'mcf', or 'laplace'"
_RAMPS = ("linear", "quadratic", "linear_range", "linear_azimuth", "quadratic_range",
          "quadratic_azimuth")

_libc = None


def _free(p):
    global _libc
    if _libc is None:
        _libc = C.CDLL(ctypes.util.find_library("c"))
        _libc.free.argtypes = [C.c_void_p]
        _libc.free.restype = None
    _libc.free(p)


def _array2d(a, dtype, name):
    a = np.ascontiguousarray(a, dtype=dtype)
    if a.ndim != 2:
        raise RuntimeError(f"{name} must be 2-D")
    return a


def _parse(table, value, msg):
    """Enum of a mode string; pybind11 turns the reference's
    std::invalid_argument into ValueError with its message."""
    try:
        return table[value]
    except (KeyError, TypeError):
        raise ValueError(msg) from None


def _call(code):
    """Status of a library call as the reference's exceptions: the
    unsupported-feature status as NotImplementedError, any other failure as
    RuntimeError (pybind11's translation of std::runtime_error)."""
    try:
        return check(code)
    except NotImplementedError:
        raise
    except Exception as e:
        raise RuntimeError(str(e)) from None


def _params(nlooks, costscale, nshortcycle, kperpdpsi, kpardpsi, defomax, min_conncomp_frac,
            max_ncomps, conncompthresh):
    """CuPhuParams as the reference's make_params fills them (cuphu_py.cu:85-109)."""
    return default_params(nlooks=float(nlooks), ncorrlooks=float(nlooks),
                          costscale=float(costscale), nshortcycle=float(nshortcycle),
                          kperpdpsi=int(kperpdpsi), kpardpsi=int(kpardpsi),
                          defomax=float(defomax), minconncompfrac=float(min_conncomp_frac),
                          maxncomps=int(max_ncomps), conncompthresh=int(conncompthresh))


def _split(igram):
    """Real and imaginary planes of a complex64 interferogram (the
    reference's host split, cuphu_py.cu:163-171)."""
    ig = _array2d(igram, np.complex64, "igram")
    return ig, np.ascontiguousarray(ig.real), np.ascontiguousarray(ig.imag)


def unwrap_arrays(igram, corr, nlooks, cost="smooth", init="mcf", mask=None, mag=None,
                  orig_mask=None, costscale=_DEF_COSTSCALE, nshortcycle=_DEF_NSHORTCYCLE,
                  kperpdpsi=_DEF_KPERPDPSI, kpardpsi=_DEF_KPARDPSI, defomax=_DEF_DEFOMAX,
                  min_conncomp_frac=_DEF_MINCONNCOMPFRAC, max_ncomps=_DEF_MAXNCOMPS,
                  conncompthresh=_DEF_CONNCOMPTHRESH, ntilerow=1, ntilecol=1, tile_rowovrlp=0,
                  tile_colovrlp=0, tilecostthresh=_DEF_TILECOSTTHRESH,
                  minregionsize=_DEF_MINREGIONSIZE, nproc=1, single_tile_reoptimize=False,
                  laplace_neighbor_feedback=False, laplace_neighbor_feedback_feather=200,
                  fix_cycle_spikes=False, bridge=False, bridge_radius=500,
                  bridge_min_num_pixel=14, bridge_erosion_size=2,
                  bridge_max_boundary_samples=4096, bridge_ramp_type=None,
                  bridge_ramp_max_num_sample=1000000, gpu_id=0):
    """Unwrap an interferogram; returns ``(unw float32, conncomp uint32)``.

    Same keywords and defaults as the reference's ``unwrap_arrays``.  The
    wrapped phase is taken from the host C library's atan2, as the
    reference takes it, so the outputs equal the reference pipeline's on the
    same inputs (Laplace path)."""
    ig, re, im = _split(igram)
    nrow, ncol = ig.shape
    corr = _array2d(corr, np.float32, "corr")
    if corr.shape != (nrow, ncol):
        raise RuntimeError("corr must have the same shape as igram")
    if nlooks < 1.0:
        raise RuntimeError("nlooks must be >= 1")
    mag = None if mag is None else _array2d(mag, np.float32, "mag")
    mask = None if mask is None else _array2d(mask, np.uint8, "mask")
    orig_mask = None if orig_mask is None else _array2d(orig_mask, np.uint8, "orig_mask")
    cost_mode = _parse(_COST, cost, _COST_MSG)
    init_meth = _parse(_INIT, init, _INIT_MSG)
    if single_tile_reoptimize:
        raise NotImplementedError("single_tile_reoptimize is outside this build")
    params = _params(nlooks, costscale, nshortcycle, kperpdpsi, kpardpsi, defomax,
                     min_conncomp_frac, max_ncomps, conncompthresh)
    tile = default_tile_params(ntilerow=int(ntilerow), ntilecol=int(ntilecol),
                               rowovrlp=int(tile_rowovrlp), colovrlp=int(tile_colovrlp),
                               tilecostthresh=int(tilecostthresh),
                               minregionsize=int(minregionsize), nproc=int(nproc),
                               laplace_neighbor_feedback=int(bool(laplace_neighbor_feedback)),
                               laplace_neighbor_feedback_feather=int(
                                   laplace_neighbor_feedback_feather),
                               fix_cycle_spikes=int(bool(fix_cycle_spikes)))
    bp = _bridge_params(bool(bridge), bridge_radius, bridge_min_num_pixel, bridge_erosion_size,
                        bridge_max_boundary_samples, bridge_ramp_type,
                        bridge_ramp_max_num_sample)
    res = CuPhuResult()
    rc = lib().cuphu_unwrap(ptr(re), ptr(im), ptr(corr), ptr(mag), ptr(mask), nrow, ncol,
                            cost_mode, init_meth, C.byref(params), C.byref(tile), C.byref(bp),
                            ptr(orig_mask), int(gpu_id), C.byref(res))
    try:
        _call(rc)
        n = nrow * ncol
        unw = np.ctypeslib.as_array(C.cast(res.unw, C.POINTER(C.c_float)), (n,))
        cc = np.ctypeslib.as_array(C.cast(res.conncomp, C.POINTER(C.c_uint32)), (n,))
        return unw.reshape(nrow, ncol).copy(), cc.reshape(nrow, ncol).copy()
    finally:
        # the callee malloc'd both planes (cuphu.h:215); the reference hands
        # them to numpy with a free() capsule, this module copies and frees
        if res.unw:
            _free(C.cast(res.unw, C.c_void_p))
        if res.conncomp:
            _free(C.cast(res.conncomp, C.c_void_p))


def build_costs(igram, corr, nlooks, cost="smooth", costscale=_DEF_COSTSCALE,
                nshortcycle=_DEF_NSHORTCYCLE, kperpdpsi=_DEF_KPERPDPSI, kpardpsi=_DEF_KPARDPSI,
                defomax=_DEF_DEFOMAX, gpu_id=0):
    """SNAPHU cost arrays of all arcs (row arcs, then column arcs) as a flat
    uint8 byte array: 4 bytes per arc for 'smooth' ({offset, sigsq} int16),
    8 for 'defo'/'topo' ({offset, sigsq, dzmax, laycost})."""
    ig, re, im = _split(igram)
    nrow, ncol = ig.shape
    corr = _array2d(corr, np.float32, "corr")
    cost_mode = _parse(_COST, cost, _COST_MSG)
    params = _params(nlooks, costscale, nshortcycle, kperpdpsi, kpardpsi, defomax,
                     _DEF_MINCONNCOMPFRAC, _DEF_MAXNCOMPS, _DEF_CONNCOMPTHRESH)
    out = C.c_void_p()
    es = C.c_size_t()
    rc = lib().cuphu_build_costs_gpu(ptr(re), ptr(im), ptr(corr), None, None, nrow, ncol,
                                     cost_mode, C.byref(params), int(gpu_id), C.byref(out),
                                     C.byref(es))
    try:
        _call(rc)
        if not out.value:
            raise RuntimeError("cuphu_build_costs_gpu returned null")
        nbytes = ((nrow - 1) * ncol + nrow * (ncol - 1)) * es.value
        return np.ctypeslib.as_array(C.cast(out, C.POINTER(C.c_uint8)), (nbytes,)).copy()
    finally:
        if out.value:
            _free(out)


def gpu_count() -> int:
    return _gpu.gpu_count()


def gpu_name(device_id: int = 0) -> str:
    return _gpu.gpu_name(device_id)


def gpu_info(device_id: int = 0) -> dict:
    return _gpu.gpu_info(device_id)


def _bridge_params(enabled, radius, min_num_pixel, erosion_size, max_boundary_samples,
                   ramp_type, ramp_max_num_sample):
    if ramp_type is not None and ramp_type not in _RAMPS:
        raise ValueError("bridge_ramp_type must be one of: linear, quadratic, linear_range, "
                         "linear_azimuth, quadratic_range, quadratic_azimuth, or None")
    bp = CuPhuBridgeParams()
    lib().cuphu_default_bridge_params(C.byref(bp))
    bp.enabled, bp.radius = int(enabled), int(radius)
    bp.min_num_pixel, bp.erosion_size = int(min_num_pixel), int(erosion_size)
    bp.max_boundary_samples = int(max_boundary_samples)
    bp.ramp_type = 0 if ramp_type is None else 1 + _RAMPS.index(ramp_type)
    bp.ramp_max_num_sample = int(ramp_max_num_sample)
    return bp


def _bridge_apply_test(unw, mask=None, bridge_radius=500, bridge_min_num_pixel=14,
                       bridge_erosion_size=2, bridge_max_boundary_samples=4096,
                       bridge_ramp_type=None, bridge_ramp_max_num_sample=1000000, gpu_id=0):
    """Phase bridging on a caller's ``unw``; returns ``(unw, conncomp)``
    copies (cuphu_py.cu:323-367)."""
    u = np.array(_array2d(unw, np.float32, "unw"), copy=True)
    m = None if mask is None else _array2d(mask, np.uint8, "mask")
    cc = np.zeros(u.shape, np.uint32)
    bp = _bridge_params(True, bridge_radius, bridge_min_num_pixel, bridge_erosion_size,
                        bridge_max_boundary_samples, bridge_ramp_type, bridge_ramp_max_num_sample)
    _call(lib().cuphu_bridge_apply_test(ptr(u), ptr(cc), u.shape[0], u.shape[1], C.byref(bp),
                                        ptr(m), int(gpu_id)))
    return u, cc


def _laplace_neighbor_feedback_test(unw, mask=None, ntilerow=1, ntilecol=1, row_ovrlp=0,
                                    col_ovrlp=0, feather_px=200):
    """The tile-boundary refinement on a caller's stitched ``unw``; returns a
    refined copy (cuphu_py.cu:360-403)."""
    u = np.array(_array2d(unw, np.float32, "unw"), copy=True)
    m = None if mask is None else _array2d(mask, np.uint8, "mask")
    _call(lib().cuphu_laplace_neighbor_feedback_test(ptr(u), ptr(m), u.shape[0], u.shape[1],
                                                     int(ntilerow), int(ntilecol),
                                                     int(row_ovrlp), int(col_ovrlp),
                                                     int(feather_px)))
    return u


def _fix_cycle_spikes_test(unw, mask=None):
    """The isolated row/column whole-cycle spike correction on a caller's
    ``unw``; returns a corrected copy (cuphu_py.cu:408-431)."""
    u = np.array(_array2d(unw, np.float32, "unw"), copy=True)
    m = None if mask is None else _array2d(mask, np.uint8, "mask")
    _call(lib().cuphu_fix_cycle_spikes_test(ptr(u), ptr(m), u.shape[0], u.shape[1]))
    return u
