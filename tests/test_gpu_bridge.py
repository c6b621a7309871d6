"""Phase bridging on the device against the oracle's restatement of the
reference (cuphu_solver.cpp:996-1352), bit for bit: the reference's own
test cases through the ``_bridge_apply_test`` hook, seeded multi-region
scenes (size pruning, both erosion tests, every ramp type, masked gaps), and
bridging as the last stage of ``cuphu_unwrap`` (the reference's C entry)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from cuphu_b200 import _cuphu_ext
from cuphu_b200 import synthetic as S
from cuphu_b200._lib import (CuPhuBridgeParams, CuPhuResult, check, default_params,
                             default_tile_params, lib, ptr)

pytestmark = pytest.mark.gpu

TWO_PI = 2.0 * np.pi


def _both(unw, mask=None, **kw):
    ref_kw = {k.replace("bridge_", ""): v for k, v in kw.items()}
    want = O.bridge(unw, mask, **ref_kw)
    got = _cuphu_ext._bridge_apply_test(unw, mask=mask, **kw)
    return got, want


def _islands(nr, nc, seed, nisl=6):
    rng = np.random.default_rng(seed)
    r, c = np.mgrid[0:nr, 0:nc]
    unw = (1.0 + 0.01 * r + 0.02 * c + rng.normal(0, 0.1, (nr, nc))).astype(np.float32)
    valid = np.zeros((nr, nc), bool)
    for _ in range(nisl):
        cy, cx = rng.integers(0, nr), rng.integers(0, nc)
        ry, rx = rng.integers(5, nr // 4), rng.integers(5, nc // 4)
        valid |= ((r - cy) / ry) ** 2 + ((c - cx) / rx) ** 2 < 1.0
        unw[((r - cy) / ry) ** 2 + ((c - cx) / rx) ** 2 < 1.0] += np.float32(
            TWO_PI * rng.integers(-3, 4))
    valid[rng.random((nr, nc)) < 0.01] = True           # isolated specks: pruned
    unw[~valid] = 0.0
    return unw


@pytest.mark.parametrize("seed,erosion,minpx,ramp", [(1, 2, 14, None), (2, 0, 1, "linear"),
                                                     (3, 1, 30, "quadratic"),
                                                     (4, 2, 14, "quadratic_azimuth")])
def test_bridge_bit_exact_vs_oracle(torch_cuda, seed, erosion, minpx, ramp):
    unw = _islands(240, 300, seed)
    (gu, gc), (wu, wc) = _both(unw, bridge_radius=40, bridge_min_num_pixel=minpx,
                               bridge_erosion_size=erosion, bridge_ramp_type=ramp)
    assert wc.max() >= 2
    assert np.array_equal(gc, wc)
    assert np.array_equal(gu.view(np.int32), wu.view(np.int32))


def test_bridge_masked_gaps_and_sampling_cap(torch_cuda):
    rng = np.random.default_rng(7)
    r, c = np.mgrid[0:300, 0:280]
    unw = (2.0 + 0.02 * r + 0.01 * c).astype(np.float32)
    unw[:, 150:] += np.float32(2 * TWO_PI)
    unw[200:, :] -= np.float32(TWO_PI)
    mask = np.ones(unw.shape, np.uint8)
    mask[:, 140:146] = 0
    mask[190:196, :] = 0
    mask[rng.random(unw.shape) < 0.002] = 0
    (gu, gc), (wu, wc) = _both(unw, mask, bridge_radius=60, bridge_min_num_pixel=10,
                               bridge_erosion_size=1, bridge_max_boundary_samples=37)
    assert wc.max() >= 3
    assert np.array_equal(gc, wc)
    assert np.array_equal(gu.view(np.int32), wu.view(np.int32))


def test_reference_bridge_cases(torch_cuda):
    """test/test_bridge.py:25-136 through the hook."""
    rng = np.random.default_rng(0)
    r, c = np.mgrid[0:60, 0:90]
    ramp = 0.02 * r + 0.015 * c
    off = np.zeros((60, 90))
    off[(r >= 20) & (r < 39)] = 3.0 * TWO_PI
    off[r >= 40] = -2.0 * TWO_PI
    unw = (ramp + off).astype(np.float32) + rng.normal(0, 0.05, (60, 90)).astype(np.float32)
    mask = np.ones((60, 90), np.uint8)
    mask[19, :] = 0
    mask[39, :] = 0
    out, cc = _cuphu_ext._bridge_apply_test(unw, mask=mask, bridge_min_num_pixel=1,
                                            bridge_erosion_size=0)
    valid = mask == 1
    assert (out[valid] - ramp[valid]).std() < 0.3
    flat = np.full((30, 30), 1.2345, np.float32)
    np.testing.assert_array_equal(_cuphu_ext._bridge_apply_test(flat)[0], flat)
    r, _ = np.mgrid[0:200, 0:10]
    steep = (5.0 + 0.2 * r).astype(np.float32)
    gap = np.ones((200, 10), np.uint8)
    gap[90:110, :] = 0
    fixed, _ = _cuphu_ext._bridge_apply_test(steep, mask=gap, bridge_min_num_pixel=1,
                                             bridge_erosion_size=0, bridge_radius=15,
                                             bridge_ramp_type="linear_azimuth")
    np.testing.assert_allclose(fixed[gap == 1], (5.0 + 0.2 * r)[gap == 1], atol=1e-3)


def test_cuphu_unwrap_bridge_stage(torch_cuda):
    """cuphu_unwrap with bridging enabled: the pipeline's output bridged over
    the solve mask (FP64 through the environment is not available there, so
    the expectation is the same call without bridging, then the oracle's
    bridging)."""
    ig, g, _, _ = S.bumps(120, 160, seed=61, nbumps=2, amp_range=(5, 20), sigma_range=(15, 40))
    ig = np.ascontiguousarray(ig, np.complex64)
    nr, nc = g.shape
    mask = np.ones((nr, nc), np.uint8)
    mask[:, 78:84] = 0
    re, im = np.ascontiguousarray(ig.real), np.ascontiguousarray(ig.imag)
    p = default_params(nlooks=5.0, ncorrlooks=5.0)
    t = default_tile_params()
    outs = []
    for enabled in (0, 1):
        bp = CuPhuBridgeParams()
        lib().cuphu_default_bridge_params(C.byref(bp))
        bp.enabled, bp.radius, bp.min_num_pixel, bp.erosion_size = enabled, 50, 14, 1
        res = CuPhuResult()
        check(lib().cuphu_unwrap(ptr(re), ptr(im), ptr(g), None, ptr(mask), nr, nc, 1, 2,
                                 C.byref(p), C.byref(t), C.byref(bp), None, 0, C.byref(res)))
        n = nr * nc
        u = np.ctypeslib.as_array(C.cast(res.unw, C.POINTER(C.c_float)), (n,)).reshape(nr, nc)
        cc = np.ctypeslib.as_array(C.cast(res.conncomp, C.POINTER(C.c_uint32)), (n,))
        outs.append((u.copy(), cc.reshape(nr, nc).copy()))
        _cuphu_ext._free(C.cast(res.unw, C.c_void_p))
        _cuphu_ext._free(C.cast(res.conncomp, C.c_void_p))
    wu, wc = O.bridge(outs[0][0], mask, radius=50, min_num_pixel=14, erosion_size=1)
    assert wc.max() >= 2
    assert np.array_equal(outs[1][1], wc)
    assert np.array_equal(outs[1][0].view(np.int32), wu.view(np.int32))
