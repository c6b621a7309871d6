"""The drop-in at the Python boundary, on CPU.

The reference's own, unmodified ``cuphu`` package (``_unwrap.py``, ``_ext.py``,
``_gpu.py``, read from the reference checkout) is imported with this build's
``cuphu_b200._cuphu_ext`` installed as ``cuphu._cuphu_ext``.  Without a GPU
the two compute entry points underneath -- ``cuphu_unwrap`` (reached by the
reference's ``_unwrap.py`` through ``unwrap_arrays``) and ``cuphu_unwrap_ex``
(reached by ``cuphu_b200.unwrap``) -- are replaced by one CPU stand-in that
unwraps with the oracle, so the comparison isolates the Python layers:
keyword plumbing, auto-tiling, NaN cleaning, mask dilation, the conncomp mask
restore, output buffers and validation errors.  The GPU side of the same
chain is covered by tests/test_gpu_ext.py.  Skipped when the reference
checkout is absent.
"""
import ctypes as C
import ctypes.util
import importlib.util
import os
import sys

import numpy as np
import pytest

import oracle as O
from cuphu_b200 import _cuphu_ext, _lib
from cuphu_b200 import _unwrap as ours_mod
from cuphu_b200 import synthetic as S
from oracle.build import REF_ROOT

REF_PKG = os.path.join(REF_ROOT, "src", "cuphu")
pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(REF_PKG, "_unwrap.py")),
                                reason="reference checkout not present")

_libc = C.CDLL(ctypes.util.find_library("c"))
_libc.malloc.restype = C.c_void_p
_libc.malloc.argtypes = [C.c_size_t]


def _host(p, n, ctype):
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(ctype)), (n,))


def _struct(ref):
    return ref._obj if hasattr(ref, "_obj") else ref


def _oracle_unwrap(ig, corr, mask, orig_mask, nrow, ncol, cost, params, tile, n_irls):
    """The stand-in's unwrap: the oracle's tiled Laplace pipeline (FP64) on
    the reference's host phase, no reference-pixel shift."""
    # non-finite samples read as 0 inside the library (host phase and
    # coherence loads), as the reference's Python layer cleans them
    ig = np.where(np.isfinite(ig), ig, 0).astype(np.complex64)
    corr = np.where(np.isfinite(corr), corr, 0).astype(np.float32)
    ph = O.phase_from_igram(ig.reshape(nrow, ncol))
    conf = orig_mask if orig_mask is not None else mask
    u, c, _ = O.unwrap_tiled(ph, corr.reshape(nrow, ncol), params.ncorrlooks, mode=int(cost),
                             mask=None if mask is None else mask.reshape(nrow, ncol),
                             conf_mask=None if conf is None else conf.reshape(nrow, ncol),
                             ntiles=(tile.ntilerow, tile.ntilecol),
                             overlap=(tile.rowovrlp, tile.colovrlp), opts=O.lap_opts(n_irls=n_irls),
                             kperp=params.kperpdpsi, kpar=params.kpardpsi,
                             minfrac=params.minconncompfrac, maxncomps=params.maxncomps,
                             conncompthresh=params.conncompthresh)
    # the library's post-passes on multi-tile scenes (feedback, then spikes)
    if tile.ntilerow * tile.ntilecol > 1:
        m2 = None if mask is None else mask.reshape(nrow, ncol)
        if tile.laplace_neighbor_feedback:
            u = O.neighbor_feedback(u, (tile.ntilerow, tile.ntilecol),
                                    (tile.rowovrlp, tile.colovrlp),
                                    tile.laplace_neighbor_feedback_feather, m2)
        if tile.fix_cycle_spikes:
            u = O.fix_cycle_spikes(u, m2)
    return u, c


class StandIn:
    """The real library for everything host-side (defaults, validation),
    with its two GPU pipelines replaced by the oracle."""

    N_IRLS = 2

    def __init__(self, real):
        self._real = real
        self.calls = []

    def __getattr__(self, name):
        return getattr(self._real, name)

    def cuphu_unwrap(self, re, im, corr, mag, mask, nrow, ncol, cost, init, params, tile, bridge,
                     orig_mask, gpu_id, result):
        n = nrow * ncol
        if init != 2:
            return self._real.cuphu_unwrap(re, im, corr, mag, mask, nrow, ncol, cost, init,
                                           params, tile, bridge, orig_mask, gpu_id, result)
        ig = (_host(re, n, C.c_float) + 1j * _host(im, n, C.c_float)).astype(np.complex64)
        m = None if not mask else _host(mask, n, C.c_uint8).copy()
        om = None if not orig_mask else _host(orig_mask, n, C.c_uint8).copy()
        u, c = _oracle_unwrap(ig, _host(corr, n, C.c_float).copy(), m, om, nrow, ncol, cost,
                              _struct(params), _struct(tile), self.N_IRLS)
        b = _struct(bridge) if bridge else None
        if b is not None and b.enabled:
            u, c = O.bridge(u, m.reshape(nrow, ncol) if m is not None else None, b.radius,
                            b.min_num_pixel, b.erosion_size, b.max_boundary_samples,
                            O.RAMPS[b.ramp_type], b.ramp_max_num_sample)
        res = _struct(result)
        pu, pc = _libc.malloc(4 * n), _libc.malloc(4 * n)
        C.memmove(pu, u.ctypes.data, 4 * n)
        C.memmove(pc, c.ctypes.data, 4 * n)
        res.unw = C.cast(pu, C.POINTER(C.c_float))
        res.conncomp = C.cast(pc, C.POINTER(C.c_uint32))
        res.nrow, res.ncol = nrow, ncol
        self.calls.append(("cuphu_unwrap", _struct(tile).ntilerow, _struct(tile).ntilecol))
        return 0

    def cuphu_bridge_apply_test(self, unw, cc, nrow, ncol, bridge, mask, gpu_id):
        n = nrow * ncol
        u = _host(unw, n, C.c_float)
        c = _host(cc, n, C.c_uint32)
        m = None if not mask else _host(mask, n, C.c_uint8).reshape(nrow, ncol).copy()
        b = _struct(bridge)
        ou, oc = O.bridge(u.reshape(nrow, ncol).copy(), m, b.radius, b.min_num_pixel,
                          b.erosion_size, b.max_boundary_samples, O.RAMPS[b.ramp_type],
                          b.ramp_max_num_sample)
        if oc.any():      # bridging ran: both outputs replaced
            u[:] = ou.ravel()
            c[:] = oc.ravel()
        self.calls.append(("bridge_hook",))
        return 0

    def cuphu_laplace_neighbor_feedback_test(self, unw, mask, nrow, ncol, ntr, ntc, rovl, covl,
                                             feather):
        n = nrow * ncol
        u = _host(unw, n, C.c_float)
        m = None if not mask else _host(mask, n, C.c_uint8).reshape(nrow, ncol).copy()
        out = O.neighbor_feedback(u.reshape(nrow, ncol).copy(), (ntr, ntc), (rovl, covl), feather,
                                  m)
        u[:] = out.ravel()
        self.calls.append(("feedback_hook", ntr, ntc))
        return 0

    def cuphu_unwrap_ex(self, igram, corr, mask, orig_mask, nrow, ncol, cost, params, tile, opts,
                        gpu_id, unw_out, cc_out, stats):
        n = nrow * ncol
        o = _struct(opts)
        assert o.ref_row < 0, "the stand-in runs without the reference-pixel shift"
        ig = _host(igram, 2 * n, C.c_float).view(np.complex64).copy()
        m = None if not mask else _host(mask, n, C.c_uint8).copy()
        om = None if not orig_mask else _host(orig_mask, n, C.c_uint8).copy()
        u, c = _oracle_unwrap(ig, _host(corr, n, C.c_float).copy(), m, om, nrow, ncol, cost,
                              _struct(params), _struct(tile), o.n_irls)
        C.memmove(unw_out, u.ctypes.data, 4 * n)
        C.memmove(cc_out, c.ctypes.data, 4 * n)
        self.calls.append(("cuphu_unwrap_ex", _struct(tile).ntilerow, _struct(tile).ntilecol))
        return 0


@pytest.fixture()
def ref(monkeypatch):
    """The reference's cuphu package on top of this build's _cuphu_ext, with
    the stand-in under both."""
    stand = StandIn(_lib.lib())
    monkeypatch.setattr(_cuphu_ext, "lib", lambda: stand)
    monkeypatch.setattr(ours_mod, "lib", lambda: stand)
    saved = {k: v for k, v in sys.modules.items() if k == "cuphu" or k.startswith("cuphu.")}
    for k in saved:
        del sys.modules[k]
    sys.modules["cuphu._cuphu_ext"] = _cuphu_ext
    spec = importlib.util.spec_from_file_location("cuphu", os.path.join(REF_PKG, "__init__.py"),
                                                  submodule_search_locations=[REF_PKG])
    pkg = importlib.util.module_from_spec(spec)
    sys.modules["cuphu"] = pkg
    try:
        spec.loader.exec_module(pkg)
        yield pkg, stand
    finally:
        for k in [k for k in sys.modules if k == "cuphu" or k.startswith("cuphu.")]:
            del sys.modules[k]
        sys.modules.update(saved)


def _scene(nr=96, nc=112, seed=3):
    ig, g, _, _ = S.bumps(nr, nc, seed=seed, nbumps=3, amp_range=(8, 25), sigma_range=(10, 30))
    return ig, g


CASES = {
    "auto_tiles": dict(cost="defo"),
    "tiles_2x2": dict(cost="smooth", ntiles=(2, 2), tile_overlap=16, target_tile_size=64),
    "mask_pad": dict(cost="smooth", mask_pad_distance=3),
    "nan_samples": dict(cost="topo"),
    "feedback": dict(cost="defo", ntiles=(2, 2), tile_overlap=16,
                     laplace_neighbor_feedback=True, laplace_neighbor_feedback_feather=30),
    "feedback_mask_pad": dict(cost="smooth", ntiles=(1, 2), tile_overlap=20, mask_pad_distance=2,
                              laplace_neighbor_feedback=True,
                              laplace_neighbor_feedback_feather=25),
    "spikes": dict(cost="smooth", ntiles=(2, 1), tile_overlap=12, fix_cycle_spikes=True),
    "bridge": dict(cost="defo", bridge=True, bridge_radius=30, bridge_min_num_pixel=20,
                   bridge_erosion_size=1),
    "bridge_ramp_shift": dict(cost="smooth", ntiles=(1, 2), tile_overlap=16, bridge=True,
                              bridge_radius=25, bridge_erosion_size=0,
                              bridge_ramp_type="linear", reference_pixel=(3, 100)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_unwrap_py_runs_on_this_extension(ref, case):
    pkg, stand = ref
    import cuphu_b200
    ig, g = _scene()
    kw = dict(CASES[case])
    kw["n_irls"] = StandIn.N_IRLS
    if case in ("mask_pad", "feedback_mask_pad", "bridge", "bridge_ramp_shift"):
        mask = np.ones(g.shape, np.uint8)
        mask[30:40, 20:90] = 0
        kw["mask"] = mask
    if case == "nan_samples":
        ig = ig.copy()
        g = g.copy()
        ig[5, 7] = np.nan
        g[11, 13] = np.inf
    if case.startswith("bridge"):
        kw["mask"][:, 50:53] = 0          # splits the scene into two regions
    kw.setdefault("reference_pixel", None)
    ref_kw = {k: v for k, v in kw.items() if k != "n_irls"}
    u_ref, c_ref = pkg.unwrap(ig, g, 5.0, init="laplace", **ref_kw)
    n_ref = len(stand.calls)
    u_out = np.zeros(g.shape, np.float32)
    c_out = np.zeros(g.shape, np.uint32)
    u, c = cuphu_b200.unwrap(ig, g, 5.0, init="laplace", unw=u_out, conncomp=c_out, **kw)
    assert u is u_out and c is c_out
    # the same library calls in the same order: one unwrap (split-plane or
    # interleaved entry point), then the boundary hook when it is needed
    def norm(calls):
        return [("unwrap" if c[0].startswith("cuphu_unwrap") else c[0],) + tuple(c[1:])
                for c in calls if c[0] != "bridge_hook"]
    assert norm(stand.calls[:n_ref]) == norm(stand.calls[n_ref:])
    if case.startswith("bridge"):
        assert c_ref.max() == 2           # the two bridged regions label the scene
    assert u_ref.dtype == np.float32 and c_ref.dtype == np.uint32
    assert np.array_equal(u.view(np.int32), u_ref.view(np.int32))
    assert np.array_equal(c, c_ref)


@pytest.mark.parametrize("bad", ["cost", "init", "ndim", "shape", "nlooks", "igram_dtype",
                                 "corr_dtype", "mask_dtype"])
def test_validation_errors_match_the_reference(ref, bad):
    pkg, _ = ref
    import cuphu_b200
    ig, g = _scene(20, 24)
    args = [ig, g, 5.0]
    kw = dict(init="laplace")
    if bad == "cost":
        kw["cost"] = "bilinear"
    elif bad == "init":
        kw["init"] = "dijkstra"
    elif bad == "ndim":
        args[0] = np.ones((2, 20, 24), np.complex64)
    elif bad == "shape":
        args[1] = np.ones((10, 10), np.float32)
    elif bad == "nlooks":
        args[2] = 0.5
    elif bad == "igram_dtype":
        args[0] = np.ones((20, 24), np.float32)
    elif bad == "corr_dtype":
        args[1] = np.ones((20, 24), np.int16)
    elif bad == "mask_dtype":
        kw["mask"] = np.ones((20, 24), np.float32)
    with pytest.raises(Exception) as e_ref:
        pkg.unwrap(*args, **kw)
    with pytest.raises(Exception) as e_ours:
        cuphu_b200.unwrap(*args, **kw)
    assert type(e_ours.value) is type(e_ref.value)
    msg_ref, msg_ours = str(e_ref.value), str(e_ours.value)
    if bad in ("cost", "init"):
        # the message lists a set, whose order follows the string hashes
        msg_ref, msg_ours = msg_ref.split(" one of")[0], msg_ours.split(" one of")[0]
    assert msg_ours == msg_ref


def test_unsupported_options_raise_instead_of_being_dropped(ref):
    pkg, _ = ref
    ig, g = _scene(20, 24)
    with pytest.raises(NotImplementedError):
        pkg.unwrap(ig, g, 5.0, init="laplace", single_tile_reoptimize=True)
    with pytest.raises(NotImplementedError):
        _cuphu_ext.unwrap_arrays(ig, g, 5.0, init="laplace", single_tile_reoptimize=True)
    with pytest.raises(ValueError, match="bridge_ramp_type"):
        _cuphu_ext.unwrap_arrays(ig, g, 5.0, init="laplace", bridge=True, bridge_ramp_type="x")
    with pytest.raises(ValueError, match="cost must be"):
        _cuphu_ext.unwrap_arrays(ig, g, 5.0, cost="nope")
    with pytest.raises(RuntimeError, match="2-D"):
        _cuphu_ext.unwrap_arrays(ig[None], g, 5.0)


def test_extension_signature_matches_the_reference_binding():
    """The keywords the reference binds for unwrap_arrays / build_costs
    (cuphu_py.cu:463-496, 590-599), in the same order."""
    import inspect
    import re
    src = open(os.path.join(REF_ROOT, "src", "cxx", "cuphu", "cuphu_py.cu")).read()
    for fn in ("unwrap_arrays", "build_costs"):
        block = src[src.index(f'm.def("{fn}"'):]
        ends = [i for i in (block.find('R"('), block.find(");")) if i >= 0]
        names = re.findall(r'"(\w+)"_a', block[:min(ends)])
        assert len(names) >= 10
        sig = inspect.signature(getattr(_cuphu_ext, fn))
        assert list(sig.parameters) == names, fn
