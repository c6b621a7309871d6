"""The optional post-passes on the device against the oracle, bit for bit:
fix_cycle_spikes (cuphu_solver.cpp:1385-1441) and the Laplace neighbor
feedback (:1469-1656), through the reference's test hooks
(``_cuphu_ext._fix_cycle_spikes_test`` / ``_laplace_neighbor_feedback_test``,
the reference's own test cases) and inside the tiled pipeline, where they run
after the merge and before the reference-pixel shift."""
import ctypes as C

import numpy as np
import pytest

import cuphu_b200
import oracle as O
from cuphu_b200 import _cuphu_ext
from cuphu_b200 import synthetic as S
from cuphu_b200._lib import (check, default_params, default_solve_options, default_tile_params,
                             lib, ptr)

pytestmark = pytest.mark.gpu

TWO_PI = 2.0 * np.pi


def _spiky(nr, nc, seed, mask_frac=0.0):
    rng = np.random.default_rng(seed)
    r, c = np.mgrid[0:nr, 0:nc]
    unw = (0.01 * r + 0.02 * c + rng.normal(0, 0.05, (nr, nc))).astype(np.float32)
    for i in rng.choice(np.arange(2, nr - 2), 4, replace=False):
        unw[i, :] += np.float32(TWO_PI * rng.choice([-2, -1, 1, 2]))
    for j in rng.choice(np.arange(2, nc - 2), 3, replace=False):
        unw[:, j] -= np.float32(TWO_PI)
    mask = None
    if mask_frac:
        mask = (rng.random((nr, nc)) > mask_frac).astype(np.uint8)
    return unw, mask


@pytest.mark.parametrize("shape,seed,mfrac", [((60, 40), 1, 0.0), ((301, 417), 2, 0.1),
                                              ((1000, 77), 3, 0.3), ((24, 2000), 4, 0.0)])
def test_fix_cycle_spikes_bit_exact_vs_oracle(torch_cuda, shape, seed, mfrac):
    unw, mask = _spiky(*shape, seed, mfrac)
    got = _cuphu_ext._fix_cycle_spikes_test(unw, mask)
    want = O.fix_cycle_spikes(unw, mask)
    assert not np.array_equal(want, unw)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))


def _seamed(nr, nc, ntiles, ovl, seed, mask_frac=0.0):
    rng = np.random.default_rng(seed)
    unw = rng.normal(0, 0.2, (nr, nc)).astype(np.float32)
    for tr in range(ntiles[0]):
        for tc in range(ntiles[1]):
            r0, ln = O.tile_bounds(nr, ntiles[0], ovl[0], tr)
            c0, lc = O.tile_bounds(nc, ntiles[1], ovl[1], tc)
            unw[r0:r0 + ln, c0:c0 + lc] += np.float32(rng.uniform(-4, 4))
    mask = None
    if mask_frac:
        mask = (rng.random((nr, nc)) > mask_frac).astype(np.uint8)
        mask[:, nc // 3] = 1
    return unw, mask


@pytest.mark.parametrize("shape,ntiles,ovl,feather,seed,mfrac", [
    ((50, 200), (1, 2), (0, 64), 50, 1, 0.0),
    ((400, 520), (2, 3), (32, 40), 60, 2, 0.2),
    ((777, 300), (4, 1), (20, 0), 200, 3, 0.9),
    ((260, 260), (3, 3), (17, 17), 300, 4, 0.0)])
def test_neighbor_feedback_bit_exact_vs_oracle(torch_cuda, shape, ntiles, ovl, feather, seed,
                                               mfrac):
    unw, mask = _seamed(*shape, ntiles, ovl, seed, mfrac)
    got = _cuphu_ext._laplace_neighbor_feedback_test(unw, mask, ntiles[0], ntiles[1], ovl[0],
                                                     ovl[1], feather)
    want = O.neighbor_feedback(unw, ntiles, ovl, feather, mask)
    assert not np.array_equal(want, unw)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))


def test_reference_hook_cases(torch_cuda):
    """The reference's own test cases (test_fix_cycle_spikes.py:25-102,
    test_laplace_neighbor_feedback.py:22-165) through the hooks."""
    r, c = np.mgrid[0:60, 0:40]
    ramp = 0.02 * r + 0.01 * c
    unw = ramp.astype(np.float32)
    unw[27, :] -= np.float32(TWO_PI)
    np.testing.assert_allclose(_cuphu_ext._fix_cycle_spikes_test(unw), ramp, atol=1e-3)
    band = ramp.astype(np.float32)
    band[20:40, :] -= np.float32(TWO_PI)
    np.testing.assert_array_equal(_cuphu_ext._fix_cycle_spikes_test(band), band)
    two = np.zeros((50, 200), np.float32)
    two[:, 100:] = 5.0
    fixed = _cuphu_ext._laplace_neighbor_feedback_test(two, np.ones(two.shape, np.uint8), 1, 2, 0,
                                                       64, 50)
    assert abs(fixed[0, 100] - fixed[0, 99]) < 0.5
    np.testing.assert_allclose(fixed[:, :90], two[:, :90])
    flat = np.full((40, 40), 3.5, np.float32)
    np.testing.assert_array_equal(
        _cuphu_ext._laplace_neighbor_feedback_test(flat, None, 1, 1, 0, 0, 200), flat)


@pytest.mark.parametrize("feedback,spikes", [(True, False), (False, True), (True, True)])
def test_pipeline_post_passes_vs_oracle(torch_cuda, feedback, spikes):
    """cuphu_unwrap_ex with the post-passes (FP64, host phase) equals the
    oracle pipeline followed by the oracle post-passes, and the reference
    shift follows them."""
    ig, g, _, _ = S.bumps(150, 180, seed=31, nbumps=3, amp_range=(10, 30), sigma_range=(10, 30))
    nr, nc = g.shape
    mask = np.ones((nr, nc), np.uint8)
    mask[100:115, 20:90] = 0
    ig = np.ascontiguousarray(ig, np.complex64)
    p = default_params(nlooks=5.0, ncorrlooks=5.0)
    t = default_tile_params(ntilerow=2, ntilecol=2, rowovrlp=20, colovrlp=24,
                            laplace_neighbor_feedback=int(feedback),
                            laplace_neighbor_feedback_feather=40, fix_cycle_spikes=int(spikes))
    o = default_solve_options(precision=1, n_irls=2, ref_row=-1, ref_col=-1)
    u = np.empty((nr, nc), np.float32)
    cc = np.empty((nr, nc), np.uint32)
    check(lib().cuphu_unwrap_ex(ptr(ig.view(np.float32)), ptr(g), ptr(mask), None, nr, nc, 0,
                                C.byref(p), C.byref(t), C.byref(o), 0, ptr(u), ptr(cc), None))
    want_u, want_c, _ = O.unwrap_tiled(O.phase_from_igram(ig), g, 5.0, mode=0, mask=mask,
                                       ntiles=(2, 2), overlap=(20, 24), opts=O.lap_opts(n_irls=2))
    if feedback:
        want_u = O.neighbor_feedback(want_u, (2, 2), (20, 24), 40, mask)
    if spikes:
        want_u = O.fix_cycle_spikes(want_u, mask)
    assert np.array_equal(u.view(np.int32), want_u.view(np.int32))
    assert np.array_equal(cc, want_c)
    # with a reference pixel: the shift applies to the post-processed scene
    o2 = default_solve_options(precision=1, n_irls=2, ref_row=70, ref_col=33)
    u2 = np.empty((nr, nc), np.float32)
    check(lib().cuphu_unwrap_ex(ptr(ig.view(np.float32)), ptr(g), ptr(mask), None, nr, nc, 0,
                                C.byref(p), C.byref(t), C.byref(o2), 0, ptr(u2), ptr(cc), None))
    ph = O.phase_from_igram(ig)
    k = np.rint((np.float64(u[70, 33]) - np.float64(ph[70, 33])) / TWO_PI)
    want2 = u - np.float32(k * TWO_PI) if k != 0 else u
    assert np.array_equal(u2.view(np.int32), want2.view(np.int32))


def test_unwrap_feedback_with_padded_mask_runs(torch_cuda):
    """The reference's special case: a grown solve mask with the boundary
    refinement solves without it and refines with the original mask."""
    ig, g, _, _ = S.bumps(90, 140, seed=32, nbumps=2, amp_range=(5, 20), sigma_range=(10, 30))
    mask = np.ones(g.shape, np.uint8)
    mask[40:50, 10:120] = 0
    unw, cc = cuphu_b200.unwrap(ig, g, 5.0, init="laplace", ntiles=(1, 2), tile_overlap=20,
                                mask=mask, mask_pad_distance=2, laplace_neighbor_feedback=True,
                                laplace_neighbor_feedback_feather=30, precision="fp64",
                                n_irls=2, reference_pixel=None)
    base, _ = cuphu_b200.unwrap(ig, g, 5.0, init="laplace", ntiles=(1, 2), tile_overlap=20,
                                mask=mask, mask_pad_distance=2, precision="fp64", n_irls=2,
                                reference_pixel=None)
    want = O.neighbor_feedback(base, (1, 2), (20, 20), 30, mask)
    assert np.array_equal(unw.view(np.int32), want.view(np.int32))
    assert np.all(cc[mask == 0] == 0)


def test_merge_conncomp_labels_the_stitched_scene(torch_cuda):
    """merge_conncomp=True: one labelling of the whole stitched scene (the
    oracle's connected components of the merged output, bit for bit), with
    fewer labels than the per-tile label spaces the reference concatenates."""
    ig, g, _, _ = S.bumps(160, 200, seed=33, nbumps=2, amp_range=(5, 15), sigma_range=(20, 40))
    g = g.copy()
    g[70:80, :] = 0.02                      # a low-coherence band splits the scene
    kw = dict(init="laplace", ntiles=(2, 3), tile_overlap=16, precision="fp64", n_irls=2,
              reference_pixel=None)
    u0, c0 = cuphu_b200.unwrap(ig, g, 5.0, **kw)
    u1, c1 = cuphu_b200.unwrap(ig, g, 5.0, merge_conncomp=True, **kw)
    assert np.array_equal(u0.view(np.int32), u1.view(np.int32))
    want = O.conncomp(u1, g)
    assert np.array_equal(c1, want)
    assert np.unique(c1).size < np.unique(c0).size
