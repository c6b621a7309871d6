"""Residue orientation against the unwrapped output, on CPU.

cuPHU has no residue code; the residues here are defined from its wrapped
phase differences (range = right - left, azimuth = top - bottom,
cuphu_util.cu:54-92) as the rounded circulation around
(r,c) -> (r,c+1) -> (r+1,c+1) -> (r+1,c).  A network-flow solver consumes
them as node supplies, so their sign must agree with the flows that an
unwrapped phase implies: n = rint(d(unw)/2pi - wrapped cycles) per arc.
Because unw is a potential, the circulation of n around every loop is minus
the residue there, for any congruent unwrapping.  The unwrapped phase is
the oracle's Laplace solution of a scene with phase jumps."""
import numpy as np

import oracle as O
from cuphu_b200 import synthetic as S

TWOPI_F = np.float32(6.28318548202514648)


def _wrapped_cycles(a, b):
    """wrap_cycles((a - b) / 2pi) in float32: d - floorf(d + 0.5f)."""
    d = ((a - b).astype(np.float32) / TWOPI_F).astype(np.float32)
    return (d - np.floor((d + np.float32(0.5)).astype(np.float32))).astype(np.float32)


def test_residues_equal_minus_the_circulation_of_the_implied_flows():
    ig, g, _, _ = S.bumps(96, 120, seed=3, nbumps=4, amp_range=(20.0, 60.0),
                          sigma_range=(6.0, 20.0), nlooks=2.0)
    ph = O.phase_from_igram(ig)
    res = O.residues(ph).astype(np.int64)
    assert (res != 0).sum() > 20                 # a scene with residues
    costs = O.build_costs(ph, g, 2.0, mode=0)
    _, _, unw, _ = O.laplace_f64(costs, ph, O.lap_opts(n_irls=2))
    u = unw.astype(np.float64) / (2 * np.pi)
    w_rng = _wrapped_cycles(ph[:, 1:], ph[:, :-1]).astype(np.float64)
    w_az = _wrapped_cycles(ph[:-1, :], ph[1:, :]).astype(np.float64)
    n_rng = np.rint((u[:, 1:] - u[:, :-1]) - w_rng)
    n_az = np.rint((u[:-1, :] - u[1:, :]) - w_az)
    circ = n_rng[:-1, :] - n_az[:, 1:] - n_rng[1:, :] + n_az[:, :-1]
    np.testing.assert_array_equal(circ, -res)


def test_residues_of_a_single_vortex():
    """A phase vortex around a point between pixels gives one residue at the
    enclosing node: +1 when the phase grows along the loop (right, down,
    left, up: clockwise with rows drawn downwards), -1 the other way."""
    y, x = np.mgrid[0:8, 0:8].astype(np.float64)
    for sign, want in ((1.0, 1), (-1.0, -1)):
        phi = np.arctan2(sign * (y - 3.5), x - 3.5)
        ph = np.mod(phi, 2 * np.pi).astype(np.float32)
        res = O.residues(ph)
        assert np.argwhere(res != 0).tolist() == [[3, 3]]
        assert int(res[3, 3]) == want
