"""CPU oracle for cuPHU's data-parallel unwrapping path (TEST INFRASTRUCTURE).

ctypes bindings over oracle/_build/libcuphu_oracle.so (the C restatement in
cuphu_oracle.c) and, when present, oracle/_ref/libcuphu_ref.so (the
reference cuPHU kernels compiled for sm_100a).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use this package, as
the checker; the product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

# SNAPHU's documented configuration defaults (snaphu.conf): the reference
# takes them from the DEF_* macros of the absent snaphu.h
# (cuphu_solver.cpp:151-216, cuphu_py.cu:122-135).  The product library
# states the same values in cuphu_b200/csrc/params.h.
DEFAULTS = dict(
    rhosconst1=1.3, rhosconst2=0.14, cstd1=0.4, cstd2=0.35, cstd3=0.06,
    defothreshfactor=1.2, sigsqcorr=0.05, costscale=100.0, nshortcycle=200.0,
    sigsqshortmin=1, defomax=1.2, kperpdpsi=7, kpardpsi=7,
    minconncompfrac=0.01, conncompthresh=300, maxncomps=32,
)

# canonical reduction geometry shared with the GPU solver (threads per item
# row, pixels per thread, item rows)
ITEM_TX, ITEM_VX, ITEM_BY = 16, 4, 16


class CostParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "ncorrlooks", "defothreshfactor", "rhosconst1", "rhosconst2", "cstd1", "cstd2",
        "cstd3", "sigsqcorr", "costscale", "nshortcycle")] + [
        ("sigsqshortmin", C.c_long), ("defomax", C.c_double)]


class LapOpts(C.Structure):
    _fields_ = [("n_irls", C.c_int), ("delta_max", C.c_float), ("delta_min", C.c_float),
                ("max_iter", C.c_int), ("tol", C.c_float), ("item_tx", C.c_int),
                ("item_vx", C.c_int), ("item_by", C.c_int)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "libcuphu_oracle.so")
        if not os.path.exists(path):
            from oracle.build import build_oracle
            build_oracle()
        _LIB = C.CDLL(path)
    return _LIB


def ref_lib():
    """The reference kernels compiled for sm_100a, or None when not built."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libcuphu_ref.so")
        if not os.path.exists(path):
            return None
        _REF = C.CDLL(path)
    return _REF


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def cost_params(nlooks: float, **kw) -> CostParams:
    d = dict(DEFAULTS)
    d.update(kw)
    return CostParams(float(nlooks), d["defothreshfactor"], d["rhosconst1"], d["rhosconst2"],
                      d["cstd1"], d["cstd2"], d["cstd3"], d["sigsqcorr"], d["costscale"],
                      d["nshortcycle"], int(d["sigsqshortmin"]), d["defomax"])


def lap_opts(n_irls=16, delta_max=0.5, delta_min=0.01, max_iter=1000, tol=1e-3) -> LapOpts:
    return LapOpts(int(n_irls), float(delta_max), float(delta_min), int(max_iter), float(tol),
                   ITEM_TX, ITEM_VX, ITEM_BY)


def phase_from_igram(igram: np.ndarray) -> np.ndarray:
    """Host atan2f phase in [0,2pi), as the reference computes it."""
    ig = np.ascontiguousarray(igram, dtype=np.complex64)
    out = np.empty(ig.shape, np.float32)
    lib().orc_phase_from_c64(_p(ig.view(np.float32)), C.c_long(ig.size), _p(out))
    return out


def phase_diffs(phase):
    phase = np.ascontiguousarray(phase, np.float32)
    nr, nc = phase.shape
    rng = np.empty((nr, max(nc - 1, 0)), np.float32)
    az = np.empty((max(nr - 1, 0), nc), np.float32)
    lib().orc_phase_diffs(_p(phase), nr, nc, _p(rng), _p(az))
    return rng, az


def boxcar2d(src, kr, kc):
    src = np.ascontiguousarray(src, np.float32)
    dst = np.empty_like(src)
    lib().orc_boxcar2d(_p(src), _p(dst), src.shape[0], src.shape[1], int(kr), int(kc))
    return dst


def arc_weights_from_mask(mask):
    mask = np.ascontiguousarray(mask, np.uint8)
    nr, nc = mask.shape
    w = np.empty((nr - 1) * nc + nr * (nc - 1), np.int16)
    lib().orc_arc_weights_from_mask(_p(mask), nr, nc, _p(w))
    return w


def build_costs(phase, corr, nlooks, mode=0, weights=None, kperp=7, kpar=7, **kw):
    """Flat int16 cost array: (narcs, 2) for smooth, (narcs, 4) for defo/topo."""
    phase = np.ascontiguousarray(phase, np.float32)
    corr = np.ascontiguousarray(corr, np.float32)
    nr, nc = phase.shape
    narcs = (nr - 1) * nc + nr * (nc - 1)
    es = 4 if mode else 2
    out = np.empty((narcs, es), np.int16)
    w = None if weights is None else np.ascontiguousarray(weights, np.int16)
    p = cost_params(nlooks, **kw)
    lib().orc_build_costs(_p(phase), _p(corr), _p(w), nr, nc, int(mode), C.byref(p),
                          int(kperp), int(kpar), _p(out))
    return out


def residues(phase):
    phase = np.ascontiguousarray(phase, np.float32)
    nr, nc = phase.shape
    out = np.empty((max(nr - 1, 0), max(nc - 1, 0)), np.int8)
    lib().orc_residues(_p(phase), nr, nc, _p(out))
    return out


def laplace_f64(costs, phase, opts: LapOpts | None = None):
    """FP64 Jacobi-PCG + IRLS.  Returns (x, k, unw, iters per pass)."""
    opts = opts or lap_opts()
    costs = np.ascontiguousarray(costs, np.int16)
    phase = np.ascontiguousarray(phase, np.float32)
    nr, nc = phase.shape
    x = np.empty((nr, nc), np.float64)
    k = np.empty((nr, nc), np.int32)
    unw = np.empty((nr, nc), np.float32)
    iters = np.zeros(opts.n_irls + 1, np.int32)
    lib().orc_laplace_f64(_p(costs), costs.shape[1], _p(phase), nr, nc, C.byref(opts),
                          _p(x), _p(k), _p(unw), _p(iters))
    return x, k, unw, iters


def conncomp(unw, corr, mask=None, poscost=None, negcost=None, minfrac=0.01,
             maxncomps=32, conncompthresh=300):
    unw = np.ascontiguousarray(unw, np.float32)
    corr = np.ascontiguousarray(corr, np.float32)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    pc = None if poscost is None else np.ascontiguousarray(poscost, np.int16)
    nc_ = None if negcost is None else np.ascontiguousarray(negcost, np.int16)
    out = np.empty(unw.shape, np.uint32)
    lib().orc_conncomp(_p(unw), _p(corr), _p(m), unw.shape[0], unw.shape[1], _p(pc), _p(nc_),
                       C.c_double(minfrac), C.c_long(maxncomps), C.c_long(conncompthresh),
                       _p(out))
    return out


def integrate_phase(phase, hflows, vflows):
    phase = np.ascontiguousarray(phase, np.float32)
    out = np.empty_like(phase)
    lib().orc_integrate_phase(_p(phase), _p(np.ascontiguousarray(hflows, np.int16)),
                              _p(np.ascontiguousarray(vflows, np.int16)),
                              phase.shape[0], phase.shape[1], _p(out))
    return out


def incrcost(costs, flows, nshortcycle=200, nflow=1):
    costs = np.ascontiguousarray(costs, np.int16)
    flows = np.ascontiguousarray(flows, np.int16)
    n = flows.size
    pos = np.empty(n, np.int16)
    neg = np.empty(n, np.int16)
    ex = lib().orc_incrcost(_p(costs), _p(flows), C.c_long(n), C.c_long(nshortcycle),
                            int(nflow), _p(pos), _p(neg))
    return pos, neg, bool(ex)


def tile_bounds(n, nt, ovl, t):
    f, ln = C.c_int(), C.c_int()
    lib().orc_tile_bounds(int(n), int(nt), int(ovl), int(t), C.byref(f), C.byref(ln))
    return f.value, ln.value


def unwrap_tiled(phase, corr, nlooks, mode=0, mask=None, conf_mask=None, ntiles=(1, 1),
                 overlap=(0, 0), opts: LapOpts | None = None, kperp=7, kpar=7,
                 minfrac=0.01, maxncomps=32, conncompthresh=300, **kw):
    """The reference's tiled Laplace pipeline (cuphu_solver.cpp:1675-2031) on
    the FP64 oracle solver.  Returns (unw, conncomp, tile_k)."""
    opts = opts or lap_opts()
    phase = np.ascontiguousarray(phase, np.float32)
    corr = np.ascontiguousarray(corr, np.float32)
    nr, nc = phase.shape
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    cm = None if conf_mask is None else np.ascontiguousarray(conf_mask, np.uint8)
    unw = np.zeros((nr, nc), np.float32)
    cc = np.zeros((nr, nc), np.uint32)
    tk = np.zeros(ntiles[0] * ntiles[1], np.float64)
    p = cost_params(nlooks, **kw)
    lib().orc_unwrap_tiled(_p(phase), _p(corr), _p(m), _p(cm), nr, nc, int(mode), C.byref(p),
                           int(kperp), int(kpar), C.byref(opts), int(ntiles[0]),
                           int(ntiles[1]), int(overlap[0]), int(overlap[1]),
                           C.c_double(minfrac), C.c_long(maxncomps), C.c_long(conncompthresh),
                           _p(unw), _p(cc), _p(tk))
    return unw, cc, tk


def fix_cycle_spikes(unw, mask=None):
    """The reference's isolated row/column whole-cycle spike correction on a
    copy of ``unw`` (cuphu_solver.cpp:1385-1441)."""
    out = np.array(unw, dtype=np.float32, order="C", copy=True)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    lib().orc_fix_cycle_spikes(_p(out), _p(m), out.shape[0], out.shape[1])
    return out


def neighbor_feedback(unw, ntiles, overlap, feather=200, mask=None):
    """The reference's Laplace tile-boundary refinement on a copy of ``unw``
    (cuphu_solver.cpp:1469-1656)."""
    out = np.array(unw, dtype=np.float32, order="C", copy=True)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    lib().orc_neighbor_feedback(_p(out), _p(m), out.shape[0], out.shape[1], int(ntiles[0]),
                                int(ntiles[1]), int(overlap[0]), int(overlap[1]), int(feather))
    return out


RAMPS = (None, "linear", "quadratic", "linear_range", "linear_azimuth", "quadratic_range",
         "quadratic_azimuth")


def bridge(unw, mask=None, radius=500, min_num_pixel=14, erosion_size=2,
           max_boundary_samples=4096, ramp_type=None, ramp_max_num_sample=1000000):
    """The reference's phase bridging (cuphu_solver.cpp:996-1352) on a copy of
    ``unw``.  Returns (unw, conncomp); conncomp is zero when there was
    nothing to bridge."""
    out = np.array(unw, dtype=np.float32, order="C", copy=True)
    cc = np.zeros(out.shape, np.uint32)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    lib().orc_bridge(_p(out), _p(cc), out.shape[0], out.shape[1], _p(m), int(radius),
                     int(min_num_pixel), int(erosion_size), int(max_boundary_samples),
                     RAMPS.index(ramp_type), int(ramp_max_num_sample))
    return out, cc


def dot_canonical(a, b):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    lib().orc_dot_canonical.restype = C.c_double
    return lib().orc_dot_canonical(_p(a), _p(b), a.shape[0], a.shape[1], ITEM_TX, ITEM_VX,
                                   ITEM_BY)


# ── reference-kernel (GPU) wrappers ────────────────────────────────────────

def _ref_pd(nlooks, **kw):
    d = dict(DEFAULTS)
    d.update(kw)
    pd = np.array([nlooks, d["defothreshfactor"], d["rhosconst1"], d["rhosconst2"], d["cstd1"],
                   d["cstd2"], d["cstd3"], d["sigsqcorr"], d["costscale"], d["nshortcycle"],
                   d["defomax"]], np.float64)
    pl = np.array([int(d["sigsqshortmin"])], np.int64)
    return pd, pl


def ref_build_costs(phase, corr, nlooks, mode=0, weights=None, kperp=7, kpar=7, reps=1, **kw):
    """Reference cuPHU cost kernels on the GPU.  Returns (costs, best ms)."""
    rl = ref_lib()
    phase = np.ascontiguousarray(phase, np.float32)
    corr = np.ascontiguousarray(corr, np.float32)
    nr, nc = phase.shape
    narcs = (nr - 1) * nc + nr * (nc - 1)
    es = 4 if mode else 2
    out = np.empty((narcs, es), np.int16)
    w = None if weights is None else np.ascontiguousarray(weights, np.int16)
    pd, pl = _ref_pd(nlooks, **kw)
    ms = C.c_float()
    rc = rl.ref_build_costs(_p(phase), _p(corr), _p(w), nr, nc, int(mode), _p(pd), _p(pl),
                            int(kperp), int(kpar), _p(out), C.byref(ms), int(reps))
    if rc != 0:
        raise RuntimeError("reference cost kernels failed")
    return out, ms.value


def ref_laplace(costs, phase, max_iter=1000, tol=1e-3):
    rl = ref_lib()
    costs = np.ascontiguousarray(costs, np.int16)
    phase = np.ascontiguousarray(phase, np.float32)
    unw = np.empty_like(phase)
    ms = C.c_float()
    rc = rl.ref_laplace(_p(costs), _p(phase), phase.shape[0], phase.shape[1], int(max_iter),
                        C.c_float(tol), _p(unw), C.byref(ms))
    if rc != 0:
        raise RuntimeError("reference laplace failed")
    return unw, ms.value


def ref_conncomp(unw, corr, mask=None, poscost=None, negcost=None, minfrac=0.01,
                 maxncomps=32, conncompthresh=300):
    rl = ref_lib()
    unw = np.ascontiguousarray(unw, np.float32)
    corr = np.ascontiguousarray(corr, np.float32)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    pc = None if poscost is None else np.ascontiguousarray(poscost, np.int16)
    ng = None if negcost is None else np.ascontiguousarray(negcost, np.int16)
    out = np.empty(unw.shape, np.uint32)
    rc = rl.ref_conncomp(_p(unw), _p(corr), _p(m), unw.shape[0], unw.shape[1], _p(pc), _p(ng),
                         C.c_double(minfrac), C.c_long(maxncomps), C.c_long(conncompthresh),
                         _p(out))
    if rc != 0:
        raise RuntimeError("reference conncomp failed")
    return out


def ref_integrate(phase, hflows, vflows):
    rl = ref_lib()
    phase = np.ascontiguousarray(phase, np.float32)
    out = np.empty_like(phase)
    rc = rl.ref_integrate(_p(phase), _p(np.ascontiguousarray(hflows, np.int16)),
                          _p(np.ascontiguousarray(vflows, np.int16)), phase.shape[0],
                          phase.shape[1], _p(out))
    if rc != 0:
        raise RuntimeError("reference integrate failed")
    return out


def ref_incrcost(costs, flows, nshortcycle=200, nflow=1):
    rl = ref_lib()
    costs = np.ascontiguousarray(costs, np.int16)
    flows = np.ascontiguousarray(flows, np.int16)
    n = flows.size
    pos = np.empty(n, np.int16)
    neg = np.empty(n, np.int16)
    rc = rl.ref_incrcost(_p(costs), _p(flows), int(n), C.c_long(nshortcycle), int(nflow),
                         _p(pos), _p(neg))
    if rc < 0:
        raise RuntimeError("reference incrcost failed")
    return pos, neg, bool(rc)
