"""``unwrap()`` -- drop-in for ``cuphu.unwrap`` on the Laplace path.

Same signature, defaults, validation and output conventions as the reference
(cuphu/_unwrap.py:167-629); the work runs in libcuphu_b200 through the C ABI
(``cuphu_unwrap_ex``), the optional post-passes ``laplace_neighbor_feedback``
and ``fix_cycle_spikes`` included.  ``init='mcf'`` / ``'mst'`` and
``single_tile_reoptimize`` need SNAPHU's CPU network-flow solver and raise
NotImplementedError; ``bridge`` runs the device bridging pass.  New keyword-only options
(``precision``, ``n_irls``, ``max_iter``, ``tol``, ``stats``) default to the
reference behaviour.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from cuphu_b200._check import (
    check_bool_or_byte_dtype,
    check_complex_dtype,
    check_cost_mode,
    check_float_dtype,
    check_init_method,
    check_shape_match,
)
from cuphu_b200._lib import (
    CuPhuBridgeParams,
    CuPhuSolveStats,
    check,
    default_params,
    default_solve_options,
    default_tile_params,
    lib,
    ptr,
)

__all__ = ["unwrap"]

_DEFAULT_LAPLACE_TILE_OVERLAP = 64
_COST = {"smooth": 0, "defo": 1, "topo": 2}
_PRECISION = {"mixed": 0, "fp64": 1}
_RAMPS = (None, "linear", "quadratic", "linear_range", "linear_azimuth", "quadratic_range",
          "quadratic_azimuth")


def _auto_ntiles_by_target_size(nrow, ncol, target_tile_size, row_ovrlp, col_ovrlp):
    """Tile counts giving every tile about the same edge length near
    ``target_tile_size`` (reference _unwrap.py:31-61): one reference edge from
    the larger dimension, rounded (not ceiled) tile counts."""
    ovrlp = max(row_ovrlp, col_ovrlp)
    step = max(1, target_tile_size - ovrlp)
    max_dim = max(nrow, ncol)
    n_max = max(1, round(max_dim / step))
    edge = max_dim / n_max
    ntilerow = max(1, round(nrow / edge))
    ntilecol = max(1, round(ncol / edge))
    return ntilerow, ntilecol


_BAND_BYTES = 64 << 20     # interferogram bytes per streamed band


def _streamable(a) -> bool:
    """A 2-D dataset that is not an in-memory array and can be read by row
    slices (h5py and zarr datasets, and the like)."""
    return (not isinstance(a, np.ndarray) and hasattr(a, "__getitem__") and
            hasattr(a, "dtype") and getattr(a, "ndim", None) == 2)


def _unwrap_streamed(igram, corr, solve_mask, orig_mask, nrow, ncol, cost, params, tile, opts,
                     gpu_id):
    """Feed the scene to the GPU in row bands (cuphu_stream_*): each band is
    read from its dataset while the previous one is uploaded."""
    flags = (1 if solve_mask is not None else 0) | (2 if orig_mask is not None else 0)
    h = C.c_void_p()
    check(lib().cuphu_stream_create(nrow, ncol, flags, gpu_id, C.byref(h)))
    try:
        band = max(1, _BAND_BYTES // (8 * ncol))
        for r0 in range(0, nrow, band):
            r1 = min(nrow, r0 + band)
            ig = np.ascontiguousarray(igram[r0:r1], dtype=np.complex64)
            co = np.ascontiguousarray(corr[r0:r1], dtype=np.float32)
            m = None if solve_mask is None else np.ascontiguousarray(solve_mask[r0:r1])
            om = None if orig_mask is None else np.ascontiguousarray(orig_mask[r0:r1])
            check(lib().cuphu_stream_put_rows(h, r0, r1 - r0, ptr(ig.view(np.float32)), ptr(co),
                                              ptr(m), ptr(om)))
        st = CuPhuSolveStats()
        check(lib().cuphu_stream_unwrap(h, cost, C.byref(params), C.byref(tile), C.byref(opts),
                                        C.byref(st)))
        unw_out = np.empty((nrow, ncol), dtype=np.float32)
        cc_out = np.empty((nrow, ncol), dtype=np.uint32)
        check(lib().cuphu_stream_get_rows(h, 0, nrow, ptr(unw_out), ptr(cc_out)))
    finally:
        lib().cuphu_stream_destroy(h)
    return unw_out, cc_out, st


def _dilate_mask(valid: np.ndarray, pixels: int) -> np.ndarray:
    """``pixels`` rounds of 4-connectivity dilation of a boolean mask (a
    Manhattan-distance diamond), reference _unwrap.py:64-84."""
    m = valid
    for _ in range(pixels):
        grown = m.copy()
        grown[1:, :] |= m[:-1, :]
        grown[:-1, :] |= m[1:, :]
        grown[:, 1:] |= m[:, :-1]
        grown[:, :-1] |= m[:, 1:]
        m = grown
    return m


def unwrap(igram, corr, nlooks, cost="smooth", init="mcf", *, mask=None, mask_pad_distance=0,
           mag=None, min_conncomp_frac=0.01, phase_grad_window=(7, 7), ntiles=None,
           tile_overlap=None, target_tile_size=1024, nproc=1, tile_cost_thresh=500,
           min_region_size=100, single_tile_reoptimize=False, laplace_neighbor_feedback=False,
           laplace_neighbor_feedback_feather=200, fix_cycle_spikes=False, bridge=False,
           bridge_radius=500, bridge_min_num_pixel=14, bridge_erosion_size=2,
           bridge_max_boundary_samples=4096, bridge_ramp_type=None,
           bridge_ramp_max_num_sample=1000000, reference_pixel=(0, 0), gpu_id=0, unw=None,
           conncomp=None, precision="mixed", n_irls=None, max_iter=None, tol=None, stats=None,
           merge_conncomp=False):
    """Unwrap an interferogram with the weighted-least-squares Laplace solver.

    Parameters mirror ``cuphu.unwrap``: ``igram`` complex 2-D, ``corr`` float
    coherence of the same shape, ``nlooks`` >= 1, ``cost`` in
    {'smooth','defo','topo'} (all three give the same Laplace weights: the
    solve uses only the cost variance, which depends on coherence), ``init``
    must be 'laplace'.  Scenes are auto-tiled toward ``target_tile_size``
    with a 64-pixel overlap unless ``ntiles`` / ``tile_overlap`` are given;
    tiles are registered by the coherence-weighted median of their overlap
    and merged.  ``reference_pixel`` shifts the output by whole cycles so
    that pixel equals its wrapped phase (None disables).  ``mask`` pixels
    with 0 are excluded; ``mask_pad_distance`` grows the solve mask and
    restores the original one for the reported conncomp.

    New options: ``precision`` 'mixed' (FP32 vectors, FP64 dots, residual
    replacement; default) or 'fp64'; ``n_irls``, ``max_iter``, ``tol``
    override the IRLS pass count (16), PCG iteration cap (1000) and
    tolerance (1e-3) and otherwise honour CUPHU_N_IRLS,
    CUPHU_LAPLACE_MAX_ITER and CUPHU_LAPLACE_TOL like the reference; a dict
    passed as ``stats`` receives solver statistics; ``merge_conncomp=True``
    labels the whole stitched scene at once, so components that cross tile
    seams get one label (the reference offsets per-tile labels instead).

    Returns ``(unw float32, conncomp uint32)``, written into ``unw`` /
    ``conncomp`` with ``[...]`` when those are given.
    """
    # datasets that can be read by row bands (h5py, zarr, ...) stream to the
    # GPU band by band; everything else is read whole, as the reference does
    streamed = _streamable(igram) and _streamable(corr)
    if not streamed:
        igram = np.asarray(igram)
        corr = np.asarray(corr)
    if np.ndim(igram) != 2:
        raise ValueError(f"igram must be 2-D, got ndim={np.ndim(igram)}")
    nrow, ncol = np.shape(igram)
    check_shape_match((nrow, ncol), corr=corr)
    if mask is not None:
        mask = np.asarray(mask)
        check_shape_match((nrow, ncol), mask=mask)
    if mag is not None:
        mag = np.asarray(mag)
        check_shape_match((nrow, ncol), mag=mag)
    check_complex_dtype(igram=igram)
    check_float_dtype(corr=corr)
    if mask is not None:
        check_bool_or_byte_dtype(mask=mask)
    if mag is not None:
        check_float_dtype(mag=mag)
    check_cost_mode(cost)
    check_init_method(init)
    if nlooks < 1.0:
        raise ValueError(f"nlooks must be >= 1, got {nlooks}")
    if precision not in _PRECISION:
        raise ValueError(f"precision must be one of {set(_PRECISION)}, got {precision!r}")
    if init != "laplace":
        raise NotImplementedError(
            f"init={init!r} runs SNAPHU's CPU network-flow solver, which is outside this "
            "build; use init='laplace'")
    if single_tile_reoptimize:
        raise NotImplementedError("single_tile_reoptimize is outside this build")
    if bridge_ramp_type is not None and bridge_ramp_type not in _RAMPS:
        raise ValueError("bridge_ramp_type must be one of: linear, quadratic, linear_range, "
                         "linear_azimuth, quadratic_range, quadratic_azimuth, or None")

    if nproc < 1:
        nproc = os.cpu_count() or 1
    if tile_overlap is None:
        tile_overlap = _DEFAULT_LAPLACE_TILE_OVERLAP
    if np.ndim(tile_overlap) == 0:
        tile_overlap = (int(tile_overlap), int(tile_overlap))
    row_ovrlp, col_ovrlp = int(tile_overlap[0]), int(tile_overlap[1])
    if ntiles is None:
        ntilerow, ntilecol = _auto_ntiles_by_target_size(nrow, ncol, target_tile_size,
                                                         row_ovrlp, col_ovrlp)
    else:
        ntilerow, ntilecol = int(ntiles[0]), int(ntiles[1])

    # Non-finite igram samples read as 0 and non-finite coherence as 0 inside
    # the library, which is what the reference's host-side cleaning produces.
    igram_c64 = None if streamed else np.ascontiguousarray(igram, dtype=np.complex64)
    corr_f32 = None if streamed else np.ascontiguousarray(corr, dtype=np.float32)
    mask_u8 = np.ascontiguousarray(mask, dtype=np.uint8) if mask is not None else None
    solve_mask_u8 = mask_u8
    if mask_u8 is not None and mask_pad_distance > 0:
        solve_mask_u8 = _dilate_mask(mask_u8 != 0, int(mask_pad_distance)).astype(np.uint8)

    # With a grown solve mask the boundary refinement must trust only the
    # original mask's pixels: solve without it, then refine on the stitched
    # result with the original mask (reference _unwrap.py:539-598).
    feedback_needs_orig_mask = (mask_u8 is not None and mask_pad_distance > 0
                                and bool(laplace_neighbor_feedback))
    internal_feedback = bool(laplace_neighbor_feedback) and not feedback_needs_orig_mask
    # bridging and that refinement follow the library's pipeline here, so the
    # reference-pixel shift follows them too (as in the reference's Python)
    shift_here = feedback_needs_orig_mask or bool(bridge)

    kperp, kpar = int(phase_grad_window[0]), int(phase_grad_window[1])
    params = default_params(nlooks=float(nlooks), ncorrlooks=float(nlooks), kperpdpsi=kperp,
                            kpardpsi=kpar, minconncompfrac=float(min_conncomp_frac))
    tile = default_tile_params(ntilerow=ntilerow, ntilecol=ntilecol, rowovrlp=row_ovrlp,
                               colovrlp=col_ovrlp, tilecostthresh=int(tile_cost_thresh),
                               minregionsize=int(min_region_size), nproc=int(nproc),
                               laplace_neighbor_feedback=int(internal_feedback),
                               laplace_neighbor_feedback_feather=int(
                                   laplace_neighbor_feedback_feather),
                               fix_cycle_spikes=int(bool(fix_cycle_spikes)))
    opts = default_solve_options(precision=_PRECISION[precision],
                                 merge_conncomp=int(bool(merge_conncomp)))
    if n_irls is not None:
        opts.n_irls = int(n_irls)
    if max_iter is not None:
        opts.max_iter = int(max_iter)
    if tol is not None:
        opts.tol = float(tol)
    if reference_pixel is not None:
        rp, rc = int(reference_pixel[0]), int(reference_pixel[1])
        if not (0 <= rp < nrow and 0 <= rc < ncol):
            raise IndexError(f"reference_pixel {reference_pixel} outside {nrow}x{ncol}")
        if not shift_here:
            opts.ref_row, opts.ref_col = rp, rc

    if streamed:
        unw_out, cc_out, st = _unwrap_streamed(igram, corr, solve_mask_u8, mask_u8, nrow, ncol,
                                               _COST[cost], params, tile, opts, int(gpu_id))
    else:
        unw_out = np.empty((nrow, ncol), dtype=np.float32)
        cc_out = np.empty((nrow, ncol), dtype=np.uint32)
        st = CuPhuSolveStats()
        check(lib().cuphu_unwrap_ex(ptr(igram_c64.view(np.float32)), ptr(corr_f32),
                                    ptr(solve_mask_u8), ptr(mask_u8), nrow, ncol, _COST[cost],
                                    C.byref(params), C.byref(tile), C.byref(opts), int(gpu_id),
                                    ptr(unw_out), ptr(cc_out), C.byref(st)))
    if stats is not None:
        stats.update(ntiles=st.ntiles, total_iters=st.total_iters,
                     max_iters_pass=st.max_iters_pass, solve_ms=st.solve_ms,
                     total_ms=st.total_ms, tiles=(ntilerow, ntilecol))

    if bridge:
        bp = CuPhuBridgeParams()
        lib().cuphu_default_bridge_params(C.byref(bp))
        bp.enabled, bp.radius = 1, int(bridge_radius)
        bp.min_num_pixel, bp.erosion_size = int(bridge_min_num_pixel), int(bridge_erosion_size)
        bp.max_boundary_samples = int(bridge_max_boundary_samples)
        bp.ramp_type = _RAMPS.index(bridge_ramp_type)
        bp.ramp_max_num_sample = int(bridge_ramp_max_num_sample)
        check(lib().cuphu_bridge_apply_test(ptr(unw_out), ptr(cc_out), nrow, ncol, C.byref(bp),
                                            ptr(solve_mask_u8), int(gpu_id)))
    if feedback_needs_orig_mask:
        check(lib().cuphu_laplace_neighbor_feedback_test(
            ptr(unw_out), ptr(mask_u8), nrow, ncol, ntilerow, ntilecol, row_ovrlp, col_ovrlp,
            int(laplace_neighbor_feedback_feather)))
    if shift_here and reference_pixel is not None:
        # _unwrap.py:605-617: whole cycles so the reference pixel equals its
        # wrapped phase
        ref_val = (np.complex64(np.asarray(igram[rp:rp + 1, rc:rc + 1])[0, 0]) if streamed
                   else igram_c64[rp, rc])
        ref_phase = float(np.angle(ref_val))
        if ref_phase < 0.0:
            ref_phase += 2.0 * np.pi
        k = round((float(unw_out[rp, rc]) - ref_phase) / (2.0 * np.pi))
        if k != 0:
            unw_out = unw_out - np.float32(k * 2.0 * np.pi)

    if mask_u8 is not None and mask_pad_distance > 0:
        cc_out = np.where(mask_u8 != 0, cc_out, 0).astype(cc_out.dtype)

    if unw is not None:
        unw[...] = unw_out
        unw_out = unw
    if conncomp is not None:
        conncomp[...] = cc_out.astype(conncomp.dtype)
        cc_out = conncomp
    return unw_out, cc_out
