"""CPU pins of the oracle's post-passes: the behaviours the reference's own
tests require of fix_cycle_spikes (test/test_fix_cycle_spikes.py:25-102) and
of the Laplace neighbor feedback (test/test_laplace_neighbor_feedback.py
:22-165), on the same synthetic cases.  The reference's host code for these
passes cannot be built here (cuphu_solver.cpp needs the absent SNAPHU
headers), so these behaviours are what pins the restatement."""
import numpy as np

import oracle as O

TWO_PI = 2.0 * np.pi


def test_spike_row_corrected():
    r, c = np.mgrid[0:60, 0:40]
    ramp = 0.02 * r + 0.01 * c
    unw = ramp.astype(np.float32)
    unw[27, :] -= np.float32(TWO_PI)
    np.testing.assert_allclose(O.fix_cycle_spikes(unw), ramp, atol=1e-3)


def test_spike_column_corrected():
    r, c = np.mgrid[0:40, 0:60]
    ramp = 0.015 * r + 0.02 * c
    unw = ramp.astype(np.float32)
    unw[:, 33] += np.float32(2.0 * TWO_PI)
    np.testing.assert_allclose(O.fix_cycle_spikes(unw), ramp, atol=1e-3)


def test_spikes_leave_ramp_and_band_alone():
    r, c = np.mgrid[0:50, 0:50]
    unw = (0.05 * r + 0.03 * c).astype(np.float32)
    np.testing.assert_array_equal(O.fix_cycle_spikes(unw), unw)
    r, c = np.mgrid[0:60, 0:40]
    unw = (0.02 * r + 0.01 * c).astype(np.float32)
    unw[20:40, :] -= np.float32(TWO_PI)
    np.testing.assert_array_equal(O.fix_cycle_spikes(unw), unw)


def test_spikes_respect_mask():
    r, c = np.mgrid[0:60, 0:40]
    ramp = 0.02 * r + 0.01 * c
    unw = ramp.astype(np.float32)
    unw[27, :] -= np.float32(TWO_PI)
    mask = np.ones(unw.shape, np.uint8)
    mask[27, :10] = 0
    out = O.fix_cycle_spikes(unw, mask)
    np.testing.assert_array_equal(out[27, :10], unw[27, :10])
    np.testing.assert_allclose(out[27, 10:], ramp[27, 10:], atol=1e-3)


def _two_tiles(nrow, ncol=200):
    unw = np.zeros((nrow, ncol), np.float32)
    unw[:, :100] = 10.0
    unw[:, 100:] = 15.0
    return unw


def test_feedback_reduces_constant_offset():
    unw = _two_tiles(50)
    fixed = O.neighbor_feedback(unw, (1, 2), (0, 64), 50, np.ones(unw.shape, np.uint8))
    assert abs(fixed[0, 100] - fixed[0, 99]) < 0.5
    np.testing.assert_allclose(fixed[:, :90], unw[:, :90])
    np.testing.assert_allclose(fixed[:, 160:], unw[:, 160:])


def test_feedback_keeps_a_continuous_gradient():
    r, c = np.mgrid[0:500, 0:200]
    unw = (0.15 * c).astype(np.float32)
    fixed = O.neighbor_feedback(unw, (1, 2), (0, 64), 200, np.ones(unw.shape, np.uint8))
    before = np.abs(unw[:, 100] - unw[:, 99]).mean()
    assert np.abs(fixed[:, 100] - fixed[:, 99]).mean() <= before * 1.1


def test_feedback_interpolates_sparse_boundary_data():
    unw = _two_tiles(60)
    mask = np.ones(unw.shape, np.uint8)
    mask[:, 99:101] = 0
    mask[::10, 99:101] = 1
    fixed = O.neighbor_feedback(unw, (1, 2), (0, 64), 50, mask)
    corr = fixed[:, 110] - unw[:, 110]
    sparse = np.delete(corr, np.arange(0, 60, 10))
    assert np.abs(sparse).min() > 1.0
    np.testing.assert_allclose(sparse, np.median(corr[::10]), atol=1.0)
    assert np.abs(np.diff(corr)).max() < 2.0


def test_feedback_fades_far_from_measurements():
    unw = _two_tiles(400)
    mask = np.zeros(unw.shape, np.uint8)
    mask[:, 150] = 1
    mask[190:200, 99:101] = 1
    fixed = O.neighbor_feedback(unw, (1, 2), (0, 64), 50, mask)
    corr = fixed[:, 150] - unw[:, 150]
    for i in (0, -1, 50, 350):
        assert abs(corr[i]) < 0.5


def test_feedback_single_tile_is_noop():
    unw = np.full((40, 40), 3.5, np.float32)
    np.testing.assert_array_equal(O.neighbor_feedback(unw, (1, 1), (0, 0), 200), unw)
