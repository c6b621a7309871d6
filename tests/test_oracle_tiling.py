"""The oracle's tiled Laplace pipeline on CPU: tile geometry against the
reference's formula (cuphu_solver.cpp:1759-1765) and the reference's own
tiled-versus-single behaviour (test/test_unwrap.py:175-188 there: the 95th
percentile of |tiled - single| below 0.5 rad on a 50 x 60 ramp)."""
import numpy as np
import pytest

import oracle as O
from cuphu_b200 import synthetic as S


def _ref_bounds(n, nt, ovl, t):
    first = t * (n - ovl) // nt
    last = n if t == nt - 1 else (t + 1) * (n - ovl) // nt + ovl
    return first, last - first


@pytest.mark.parametrize("n,nt,ovl", [(50, 2, 4), (60, 3, 4), (8192, 9, 64), (4096, 4, 64),
                                      (1001, 7, 33), (17, 5, 0), (3072, 3, 64)])
def test_tile_bounds_follow_the_reference_formula(n, nt, ovl):
    got = [O.tile_bounds(n, nt, ovl, t) for t in range(nt)]
    assert got == [_ref_bounds(n, nt, ovl, t) for t in range(nt)]
    assert got[0][0] == 0 and got[-1][0] + got[-1][1] == n
    for (f0, l0), (f1, _) in zip(got, got[1:]):
        assert f1 + ovl == f0 + l0                 # neighbours overlap by ovl


def _ramp():
    r = np.arange(50, dtype=np.float32)
    c = np.arange(60, dtype=np.float32)
    truth = 0.1 * r[:, None] + 0.2 * c[None, :]
    ig = np.exp(1j * truth).astype(np.complex64)
    return O.phase_from_igram(ig), np.full((50, 60), 0.9, np.float32)


@pytest.mark.parametrize("ntiles", [(1, 1), (2, 2), (2, 3)])
def test_tiled_matches_single_on_the_reference_ramp(ntiles):
    ph, g = _ramp()
    single, _, _ = O.unwrap_tiled(ph, g, 10.0, ntiles=(1, 1))
    tiled, _, _ = O.unwrap_tiled(ph, g, 10.0, ntiles=ntiles, overlap=(4, 4))
    assert np.isfinite(tiled).all()
    assert float(np.percentile(np.abs(tiled - single), 95)) < 0.5


def test_tiled_registration_on_a_deformation_scene():
    """Bumps of up to 30 rad across 3 x 3 tiles: the tiles' own solutions
    sit whole cycles apart (their anchors differ), and the coherence-weighted
    median registration puts every tile back on the single solve's cycles."""
    ig, g, _, _ = S.bumps(150, 180, seed=5, nbumps=3, amp_range=(10.0, 30.0),
                          sigma_range=(15.0, 40.0), nlooks=10.0)
    ph = O.phase_from_igram(ig)
    single, _, _ = O.unwrap_tiled(ph, g, 10.0, ntiles=(1, 1))
    tiled, _, tk = O.unwrap_tiled(ph, g, 10.0, ntiles=(3, 3), overlap=(16, 16))
    assert tk.shape == (9,) and np.isfinite(tk).all()
    assert np.count_nonzero(np.rint(tk)) >= 4         # registration did shift tiles
    assert float(np.abs(tiled - single).max()) < 1e-3
