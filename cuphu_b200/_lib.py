"""ctypes binding of libcuphu_b200.so (the C ABI in include/cuphu_b200.h).

The shared library is built in-tree by ``cuphu_b200/build.py`` (or
``__graft_entry__.build()``).  There is no CPU fallback: importing an API that
needs the library raises ImportError when it is missing.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcuphu_b200.so")

_D, _L, _I = C.c_double, C.c_long, C.c_int


def _fields(spec):
    out = []
    for typ, names in spec:
        out += [(n.strip(), typ) for n in names.split(",")]
    return out


class CuPhuParams(C.Structure):
    """Mirror of CuPhuParams (reference cuphu.h:33-92)."""
    _fields_ = _fields([
        (_D, "nlooks, ncorrlooks, defothreshfactor, rhosconst1, rhosconst2"),
        (_D, "cstd1, cstd2, cstd3"),
        (_D, "sigsqcorr, costscale, nshortcycle"),
        (_L, "sigsqshortmin"),
        (_D, "orbitradius, altitude, earthradius, baseline, baselineangle, bperp"),
        (_I, "transmitmode"),
        (_L, "nlooksrange, nlooksaz, nlooksother, ncorrlooksrange, ncorrlooksaz"),
        (_D, "nearrange, dr, da, rangeres, azres, lambda_"),
        (_D, "kds, specularexp, dzrcritfactor"),
        (_I, "shadow"),
        (_D, "dzeimin"),
        (_L, "laywidth"),
        (_D, "layminei, sloperatiofactor, sigsqei"),
        (_D, "dzlaypeak, azdzfactor, dzeifactor, dzeiweight"),
        (_D, "dzlayfactor, layconst, layfalloffconst, sigsqlayfactor"),
        (_D, "defoazdzfactor, defomax, defolayconst"),
        (_I, "kperpdpsi, kpardpsi"),
        (_D, "p, maxcost, costscaleambight, dnomincangle"),
        (_D, "initdzr, initdzstep, threshold"),
        (_L, "initmaxflow, arcmaxflowconst, maxflow, nshortcycleL"),
        (_L, "cs2scalefactor"),
        (_D, "minconncompfrac"),
        (_L, "conncompthresh"),
        (_L, "maxncomps"),
    ])


class CuPhuTileParams(C.Structure):
    """Mirror of CuPhuTileParams (reference cuphu.h:95-138)."""
    _fields_ = [(n, _I) for n in (
        "ntilerow", "ntilecol", "rowovrlp", "colovrlp", "tilecostthresh", "minregionsize",
        "nproc", "ngpustreams", "single_tile_reoptimize", "laplace_neighbor_feedback",
        "laplace_neighbor_feedback_feather", "fix_cycle_spikes")]


class CuPhuBridgeParams(C.Structure):
    _fields_ = [(n, _I) for n in ("enabled", "radius", "min_num_pixel", "erosion_size",
                                  "max_boundary_samples", "ramp_type", "ramp_max_num_sample")]


class CuPhuResult(C.Structure):
    _fields_ = [("unw", C.POINTER(C.c_float)), ("conncomp", C.POINTER(C.c_uint32)),
                ("nrow", _I), ("ncol", _I)]


class CuPhuSolveOptions(C.Structure):
    _fields_ = [("precision", _I), ("n_irls", _I), ("irls_delta_max", C.c_float),
                ("irls_delta_min", C.c_float), ("max_iter", _I), ("tol", C.c_float),
                ("replace_every", _I), ("ref_row", _I), ("ref_col", _I), ("timeout_ms", _I),
                ("device_phase", _I), ("merge_conncomp", _I)]


class CuPhuSolveStats(C.Structure):
    _fields_ = [("ntiles", _I), ("total_iters", _I), ("max_iters_pass", _I),
                ("solve_ms", _D), ("total_ms", _D), ("px_iters", _D)]


class CuPhuScene(C.Structure):
    _fields_ = [("igram_c64", C.c_void_p), ("phase", C.c_void_p), ("corr", C.c_void_p),
                ("mask", C.c_void_p), ("orig_mask", C.c_void_p), ("nrow", _I), ("ncol", _I),
                ("ntilerow", _I), ("ntilecol", _I), ("rowovrlp", _I), ("colovrlp", _I),
                ("nlooks", _D), ("unw_out", C.c_void_p), ("conncomp_out", C.c_void_p)]


VP, P = C.c_void_p, C.POINTER

# name -> (restype, argtypes)
SIGNATURES = {
    "cuphu_default_params": (None, [P(CuPhuParams)]),
    "cuphu_default_tile_params": (None, [P(CuPhuTileParams)]),
    "cuphu_default_bridge_params": (None, [P(CuPhuBridgeParams)]),
    "cuphu_default_solve_options": (None, [P(CuPhuSolveOptions)]),
    "cuphu_last_error": (C.c_char_p, []),
    "cuphu_unwrap": (_I, [VP, VP, VP, VP, VP, _I, _I, _I, _I, P(CuPhuParams),
                          P(CuPhuTileParams), P(CuPhuBridgeParams), VP, _I, P(CuPhuResult)]),
    "cuphu_unwrap_ex": (_I, [VP, VP, VP, VP, _I, _I, _I, P(CuPhuParams), P(CuPhuTileParams),
                             P(CuPhuSolveOptions), _I, VP, VP, P(CuPhuSolveStats)]),
    "cuphu_unwrap_device": (_I, [VP, VP, VP, VP, VP, _I, _I, _I, P(CuPhuParams),
                                 P(CuPhuTileParams), P(CuPhuSolveOptions), VP, VP, VP,
                                 P(CuPhuSolveStats), VP]),
    "cuphu_unwrap_batch_device": (_I, [P(CuPhuScene), _I, _I, P(CuPhuParams),
                                       P(CuPhuSolveOptions), P(CuPhuSolveStats), VP]),
    "cuphu_build_costs_gpu": (_I, [VP, VP, VP, VP, VP, _I, _I, _I, P(CuPhuParams), _I,
                                   P(VP), P(C.c_size_t)]),
    "cuphu_build_smooth_costs_gpu": (_I, [VP, VP, VP, VP, _I, _I, P(CuPhuParams), _I, _I,
                                          P(VP), VP]),
    "cuphu_build_defo_costs_gpu": (_I, [VP, VP, VP, VP, _I, _I, P(CuPhuParams), _I, _I,
                                        P(VP), VP]),
    "cuphu_build_costs_device": (_I, [VP, VP, VP, _I, _I, _I, P(CuPhuParams), VP, VP, VP]),
    "cuphu_residues_gpu": (_I, [VP, _I, _I, VP, VP]),
    "cuphu_phase_gpu": (_I, [VP, C.c_longlong, VP, VP]),
    "cuphu_laplace_unwrap_gpu": (_I, [VP, VP, _I, _I, _D, _I, C.c_float, _I, VP, VP]),
    "cuphu_laplace_solve_device": (_I, [VP, _I, VP, _I, _I, P(CuPhuSolveOptions), VP, VP, VP,
                                        P(CuPhuSolveStats), VP]),
    "cuphu_integrate_phase_gpu": (_I, [VP, VP, VP, _I, _I, _I, VP]),
    "cuphu_integrate_phase_noalloc": (_I, [VP, VP, VP, _I, _I, VP, VP]),
    "cuphu_stream_create": (_I, [_I, _I, _I, _I, P(VP)]),
    "cuphu_stream_put_rows": (_I, [VP, _I, _I, VP, VP, VP, VP]),
    "cuphu_stream_unwrap": (_I, [VP, _I, P(CuPhuParams), P(CuPhuTileParams),
                                 P(CuPhuSolveOptions), P(CuPhuSolveStats)]),
    "cuphu_stream_get_rows": (_I, [VP, _I, _I, VP, VP]),
    "cuphu_stream_destroy": (_I, [VP]),
    "cuphu_mst_costs_device": (_I, [VP, C.c_longlong, _L, _L, VP, VP]),
    "cuphu_mcf_inputs": (_I, [VP, VP, VP, VP, _I, _I, _I, P(CuPhuParams), _I, VP, VP, VP]),
    "cuphu_laplace_neighbor_feedback_test": (_I, [VP, VP, _I, _I, _I, _I, _I, _I, _I]),
    "cuphu_fix_cycle_spikes_test": (_I, [VP, VP, _I, _I]),
    "cuphu_laplace_neighbor_feedback_device": (_I, [VP, VP, _I, _I, _I, _I, _I, _I, _I, VP]),
    "cuphu_fix_cycle_spikes_device": (_I, [VP, VP, _I, _I, VP]),
    "cuphu_conncomp_gpu": (_I, [VP, VP, VP, _I, _I, VP, VP, P(CuPhuParams), _I, VP]),
    "cuphu_conncomp_ex": (_I, [VP, VP, VP, _I, _I, C.c_float, _D, _L, _I, VP]),
    "cuphu_incrcost_early_exit": (_I, [VP, VP, _I, _L, _I, VP, VP, VP]),
    "cuphu_wls_solve_device": (_I, [VP, VP, VP, VP, VP, VP, _I, _I, P(CuPhuSolveOptions), VP,
                                    P(CuPhuSolveStats), VP]),
    "cuphu_autotune": (_I, [VP, VP, _I, _I, _I, P(CuPhuParams), P(CuPhuTileParams), _I, P(_I)]),
    "cuphu_batch_graph_create": (_I, [P(CuPhuScene), _I, _I, P(CuPhuParams), P(CuPhuSolveOptions),
                                      P(VP)]),
    "cuphu_batch_graph_launch": (_I, [VP, VP]),
    "cuphu_batch_graph_destroy": (_I, [VP]),
    "cuphu_wls_grad_device": (_I, [VP, VP, VP, VP, VP, VP, _I, _I, VP, VP, VP, VP, VP]),
    "cuphu_gpu_count": (_I, []),
    "cuphu_gpu_name": (_I, [_I, C.c_char_p, _I]),
    "cuphu_gpu_info": (_I, [_I, P(C.c_longlong), P(_I), P(_I), P(_I)]),
    "cuphu_bridge_apply_test": (_I, [VP, VP, _I, _I, P(CuPhuBridgeParams), VP, _I]),
    "cuphu_bridge_device": (_I, [VP, VP, VP, _I, _I, P(CuPhuBridgeParams), VP]),
    "cuphu_test_skip_barrier_once": (_I, [_I, _I]),
    "cuphu_test_force_solve_shape": (_I, [_I]),
    "cuphu_last_status": (_I, [_I]),
    "cuphu_release_workspace": (_I, [_I]),
}

_lib = None


def lib():
    """The loaded library; raises ImportError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libcuphu_b200.so not found at {LIB_PATH}; build it with "
                "`python cuphu_b200/build.py` (nvcc, sm_100a). There is no CPU fallback.")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class CuPhuError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


def check(code: int) -> int:
    if code < 0:
        msg = lib().cuphu_last_error()
        msg = msg.decode() if msg else "cuphu call failed"
        if code == -4:
            raise NotImplementedError(msg)
        raise CuPhuError(code, msg)
    return code


def _override(s, kw):
    """Set struct fields by name; an unknown name is an error, not a new
    Python attribute the library never sees."""
    names = {f[0] for f in type(s)._fields_}
    for k, v in kw.items():
        if k not in names:
            raise TypeError(f"{type(s).__name__} has no field {k!r}")
        setattr(s, k, v)
    return s


def default_params(**kw) -> CuPhuParams:
    p = CuPhuParams()
    lib().cuphu_default_params(C.byref(p))
    return _override(p, kw)


def default_tile_params(**kw) -> CuPhuTileParams:
    t = CuPhuTileParams()
    lib().cuphu_default_tile_params(C.byref(t))
    return _override(t, kw)


def default_solve_options(**kw) -> CuPhuSolveOptions:
    o = CuPhuSolveOptions()
    lib().cuphu_default_solve_options(C.byref(o))
    return _override(o, kw)


def ptr(a):
    """Host pointer of a numpy array (or None)."""
    return None if a is None else a.ctypes.data_as(C.c_void_p)
