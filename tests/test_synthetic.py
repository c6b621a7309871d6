"""The seeded synthetic scenes stand in for the benchmark configurations: the
recipes (bump and fractal-topography truth, coherence ranges, the water blob,
look numbers, the Cramer-Rao noise level, the uneven batch) checked on CPU at
reduced edge lengths of the same generators."""
import numpy as np
import pytest

from cuphu_b200 import synthetic as S


def test_scenes_are_seeded():
    a = S.config_scene("c0_512_defo", seed=3, scale=96)
    b = S.config_scene("c0_512_defo", seed=3, scale=96)
    c = S.config_scene("c0_512_defo", seed=4, scale=96)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])


@pytest.mark.parametrize("name,lo,hi,nlooks,cost", [
    ("c0_512_defo", 0.3, 0.95, 5.0, "defo"),
    ("c4_2048_defo", 0.3, 0.95, 5.0, "defo"),
    ("c2_8192_topo", 0.2, 0.9, 20.0, "topo"),
])
def test_coherence_ranges_and_looks(name, lo, hi, nlooks, cost):
    ig, g, t, ex = S.config_scene(name, seed=0, scale=256)
    assert ig.dtype == np.complex64 and g.dtype == np.float32 and ig.shape == g.shape
    assert g.min() >= lo - 1e-6 and g.max() <= hi + 1e-6
    assert g.max() - g.min() > 0.5 * (hi - lo)          # the range is used
    assert ex["nlooks"] == nlooks and ex["cost"] == cost


def test_water_blob_of_the_4096_scene():
    ig, g, t, ex = S.config_scene("c1_4096_smooth", seed=0, scale=512)
    water = ex["water"]
    assert 0.10 < water.mean() < 0.20
    assert g[water].min() >= 0.02 - 1e-6 and g[water].max() <= 0.1 + 1e-6
    assert ex["n_irls"] == 3 and ex["cost"] == "smooth" and ex["nlooks"] == 9.0


def test_topography_phase_and_amplitude():
    ig, g, t, ex = S.config_scene("c2_8192_topo", seed=0, scale=512)
    # 2500 m of relief through 4 pi Bperp / (lambda R sin 35 deg): ~40.3 rad
    want = 4 * np.pi * 150.0 / (0.24 * 850e3 * np.sin(np.deg2rad(35.0))) * 2500.0
    assert abs(float(t.max() - t.min()) - want) < 0.01 * want
    assert 0.9 < float(ex["mag"].mean()) < 1.1


def test_noise_follows_the_cramer_rao_bound():
    rng = np.random.default_rng(0)
    truth = np.zeros((400, 400), np.float32)
    for gamma, nlooks in ((0.8, 5.0), (0.6, 20.0)):
        z = S._noisy_igram(rng, truth, np.full(truth.shape, gamma, np.float32), nlooks)
        err = np.angle(z)
        crb = np.sqrt((1 - gamma ** 2) / (2 * nlooks * gamma ** 2))
        assert abs(float(err.std()) / crb - 1.0) < 0.05


def test_uneven_batch_sides():
    scenes = S.batch_scenes(count=3, seed=0, sides=(64, 96, 128))
    assert len(scenes) == 3
    for ig, g, t in scenes:
        assert ig.shape[0] in (64, 96, 128) and ig.shape[1] in (64, 96, 128)
        assert ig.shape == g.shape == t.shape
