"""CPU pins of the oracle's phase bridging: the reference's own bridging
test cases (test/test_bridge.py:25-136) on the restatement, plus the
structure of its stages.  The reference's orchestration (cuphu_solver.cpp)
cannot be built here, so these behaviours pin the restatement."""
import numpy as np

import oracle as O

TWO_PI = 2.0 * np.pi


def test_reconciles_constant_region_offsets():
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
    out, cc = O.bridge(unw, mask, min_num_pixel=1, erosion_size=0)
    valid = mask == 1
    assert (out[valid] - ramp[valid]).std() < 0.3
    assert set(np.unique(cc[valid])) == {1, 2, 3}
    assert not np.allclose(out[valid], unw[valid])


def test_single_region_is_noop():
    unw = np.full((30, 30), 1.2345, np.float32)
    out, cc = O.bridge(unw)
    np.testing.assert_array_equal(out, unw)
    assert not cc.any()


def test_uses_mask_not_raw_zero():
    r, c = np.mgrid[0:40, 0:60]
    ramp = 1.0 + 0.02 * r + 0.01 * c
    unw = (ramp + np.where(c >= 30, 4.0 * TWO_PI, 0.0)).astype(np.float32)
    mask = np.ones((40, 60), np.uint8)
    mask[:, 28:32] = 0
    unw[:, 28:32] = 99.0
    out, _ = O.bridge(unw, mask, min_num_pixel=1, erosion_size=0)
    valid = mask == 1
    assert (out[valid] - ramp[valid]).std() < 0.3
    np.testing.assert_array_equal(out[:, 28:32], unw[:, 28:32])


def test_ramp_fixes_wrong_jump_from_steep_gradient():
    r, _ = np.mgrid[0:200, 0:10]
    ramp = 5.0 + 0.2 * r.astype(np.float64)
    unw = ramp.astype(np.float32)
    mask = np.ones((200, 10), np.uint8)
    mask[90:110, :] = 0
    no_ramp, _ = O.bridge(unw, mask, radius=15, min_num_pixel=1, erosion_size=0)
    with_ramp, _ = O.bridge(unw, mask, radius=15, min_num_pixel=1, erosion_size=0,
                            ramp_type="linear_azimuth")
    valid = mask == 1
    assert (no_ramp[valid] - ramp[valid]).std() > 1.0
    np.testing.assert_allclose(with_ramp[valid], ramp[valid], atol=1e-3)


def test_small_and_thin_regions_are_dropped():
    """A region under min_num_pixel, and a one-pixel-wide strip that does not
    survive erosion, get no label and keep their values."""
    unw = np.zeros((50, 50), np.float32)
    unw[2:20, 2:20] = 1.0
    unw[30:48, 2:20] = 1.0 + np.float32(TWO_PI)
    unw[2:40, 30] = 7.0                      # thin: dropped by erosion
    unw[45:47, 40:42] = 3.0                  # small: 4 pixels
    out, cc = O.bridge(unw, min_num_pixel=5, erosion_size=2)
    assert cc[10, 10] and cc[40, 10] and cc[10, 10] != cc[40, 10]
    assert cc[20, 30] == 0 and cc[46, 41] == 0
    assert out[20, 30] == unw[20, 30] and out[46, 41] == unw[46, 41]
    assert abs(out[40, 10] - out[10, 10]) < 1e-5
