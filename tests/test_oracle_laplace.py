"""The oracle's Laplace solve (A9-A14, cuphu_laplace.cu:65-549) against an
independent statement of the same problem, on CPU.

The Laplace path solves, per IRLS pass, (D^T W D + eps I) x = D^T W g with
(D x)_a = x(head) - x(tail), g the float wrapped phase differences of the
arcs, w0 = 1/sigsq from the cost array (0 for sigsq <= 0 or >= 32000) and
the reweighting w = w0 / sqrt(e^2 + delta_k^2), e = D x - g, delta_k =
max(delta_min, delta_max 0.5^k).  Here that system is assembled with scipy
and solved directly; the oracle's Jacobi-PCG (run to a tight tolerance) must
reach the same solution, and its anchoring and congruence (A14) must follow
from its own solution.  The cost arrays are the golden fixtures made by the
reference's cost kernels, so the inputs are the reference's."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.csgraph as csg
import scipy.sparse.linalg as spla

import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

TWOPI_F = np.float32(6.28318548202514648)       # cuphu_util.cu:23
INV_TWOPI_F = np.float32(0.15915494309189534561)  # cuphu_laplace.cu:60
EPS = float(np.float32(1e-12))                  # cuphu_laplace.cu:61
LARGESIGSQ = 32000                              # cuphu_laplace.cu:62


def _wrap(x):
    """fmaf(-2pi_f, rintf(x * (1/2pi)_f), x) in float32 (one rounding: the
    product 2pi_f k and the sum are exact in float64)."""
    x = np.asarray(x, np.float32)
    k = np.rint(x * INV_TWOPI_F).astype(np.float64)
    return (x.astype(np.float64) - np.float64(TWOPI_F) * k).astype(np.float32)


def _arcs(nr, nc):
    idx = np.arange(nr * nc).reshape(nr, nc)
    tail = np.concatenate([idx[:-1, :].ravel(), idx[:, :-1].ravel()])
    head = np.concatenate([idx[1:, :].ravel(), idx[:, 1:].ravel()])
    return tail, head


def _incidence(tail, head, n):
    na = tail.size
    rows = np.concatenate([np.arange(na), np.arange(na)])
    cols = np.concatenate([head, tail])
    vals = np.concatenate([np.ones(na), -np.ones(na)])
    return sp.csr_matrix((vals, (rows, cols)), shape=(na, n))


def _direct_irls(costs, phase, n_irls, delta_max=0.5, delta_min=0.01):
    nr, nc = phase.shape
    tail, head = _arcs(nr, nc)
    s = costs[:, 1].astype(np.int32)
    w0 = np.where((s > 0) & (s < LARGESIGSQ), np.float32(1.0) / s.astype(np.float32),
                  np.float32(0.0)).astype(np.float32)
    ph = phase.ravel()
    g = _wrap(ph[head] - ph[tail]).astype(np.float64)
    D = _incidence(tail, head, nr * nc)
    eye = sp.eye(nr * nc)

    def solve(w):
        w = w.astype(np.float64)
        A = (D.T @ sp.diags(w) @ D + EPS * eye).tocsc()
        return spla.spsolve(A, D.T @ (w * g))

    x = solve(w0)
    for k in range(n_irls):
        delta = max(np.float32(delta_min), np.float32(delta_max) * np.float32(0.5 ** k))
        e = (x[head] - x[tail]) - g
        w = np.where(w0 > 0, (w0.astype(np.float64) / np.sqrt(e * e + float(delta) ** 2)),
                     0.0).astype(np.float32)
        x = solve(w)
    adj = abs(D).T @ sp.diags((w0 > 0).astype(np.float64)) @ abs(D)
    comps = csg.connected_components(adj, directed=False)[1]
    return x.reshape(nr, nc), comps.reshape(nr, nc)


def _center(x, comps):
    """Remove each connected component's mean (eps alone fixes it)."""
    out = x.copy()
    for c in np.unique(comps):
        m = comps == c
        out[m] -= out[m].mean()
    return out


CASES = ["costs_m0_now_48x64", "costs_m1_w_33x70", "costs_m0_w_70x41"]


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("n_irls", [0, 3])
def test_oracle_laplace_solves_the_wls_problem(name, n_irls):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    phase, costs = z["phase"], z["costs"]
    x, k, unw, iters = O.laplace_f64(costs, phase, O.lap_opts(n_irls=n_irls, max_iter=20000,
                                                                tol=1e-9))
    assert (iters > 0).all() and (iters < 20000).all(), iters
    x_ref, comps = _direct_irls(costs, phase, n_irls)
    d = _center(x, comps) - _center(x_ref, comps)
    scale = max(1.0, np.abs(x_ref).max())
    assert np.abs(d).max() < 1e-6 * scale, (np.abs(d).max(), scale)


@pytest.mark.parametrize("name", CASES)
def test_oracle_anchor_and_congruence(name):
    """A14: k = rint(((x + phase(0,0) - x(0,0)) - phase) / 2pi) in FP64 and
    unw = fmaf(2pi_f, k, phase): unw is congruent to the wrapped phase."""
    z = np.load(os.path.join(GOLD, name + ".npz"))
    phase, costs = z["phase"], z["costs"]
    x, k, unw, _ = O.laplace_f64(costs, phase, O.lap_opts())
    off = float(phase[0, 0]) - x[0, 0]
    kk = np.rint(((x + off) - phase.astype(np.float64)) / (2.0 * np.pi))
    np.testing.assert_array_equal(k, kk.astype(np.int32))
    want = (np.float64(TWOPI_F) * kk + phase.astype(np.float64)).astype(np.float32)
    np.testing.assert_array_equal(unw, want)
    assert k[0, 0] == 0 and unw[0, 0] == phase[0, 0]
