"""Inputs of the CPU network-flow front end computed on the GPU: the cost
arrays, the residues and the initial-flow arc weights
(cuphu_solver.cpp:607-633: clip(min(pos, neg) at flow 0, 1, maxcost)) in one
call, against the oracle and against the reference's own incremental-cost
kernel evaluated at flow 0."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from cuphu_b200 import synthetic as S
from cuphu_b200._lib import CuPhuError, check, default_params, lib, ptr
from tests.devbuf import dptr, empty, to_dev, to_host

pytestmark = pytest.mark.gpu


def _mst_from(pos, neg, maxcost):
    return np.clip(np.minimum(pos.astype(np.int64), neg.astype(np.int64)), 1, maxcost
                   ).astype(np.int16)


@pytest.mark.parametrize("shape,nlooks", [((97, 130), 5.0), ((400, 333), 9.0)])
def test_mcf_inputs_smooth(torch_cuda, shape, nlooks):
    ig, g, _, _ = S.bumps(*shape, seed=shape[0], nbumps=3, amp_range=(10, 30),
                          sigma_range=(10, 30), nlooks=nlooks)
    g = g.copy()
    g[10:30, 5:60] = 0.02                       # low coherence
    ig = np.ascontiguousarray(ig, np.complex64)
    nr, nc = g.shape
    narcs = (nr - 1) * nc + nr * (nc - 1)
    w = np.ones(narcs, np.int16)
    w[1000:1400] = 0                            # masked-out arcs: sigsq = LARGESHORT
    p = default_params(nlooks=nlooks, ncorrlooks=nlooks)
    costs = np.empty((narcs, 2), np.int16)
    mst = np.empty(narcs, np.int16)
    res = np.empty((nr - 1, nc - 1), np.int8)
    re, im = np.ascontiguousarray(ig.real), np.ascontiguousarray(ig.imag)
    check(lib().cuphu_mcf_inputs(ptr(re), ptr(im), ptr(g), ptr(w), nr, nc, 0, C.byref(p), 0,
                                 ptr(costs), ptr(mst), ptr(res)))
    ph = O.phase_from_igram(ig)
    want = O.build_costs(ph, g, nlooks, mode=0, weights=w)
    assert np.array_equal(costs, want)
    assert np.array_equal(res, O.residues(ph))
    pos, neg, _ = O.incrcost(want, np.zeros(narcs, np.int16), nshortcycle=200, nflow=1)
    assert np.array_equal(mst, _mst_from(pos, neg, int(p.maxcost)))
    assert (want[:, 1] == 32000).any() and (mst[want[:, 1] == 32000] == 1).all()
    if O.ref_lib() is not None:
        rpos, rneg, _ = O.ref_incrcost(want, np.zeros(narcs, np.int16), nshortcycle=200, nflow=1)
        assert np.array_equal(mst, _mst_from(rpos, rneg, int(p.maxcost)))


def test_mst_costs_device_maxcost_clip(torch_cuda):
    rng = np.random.default_rng(5)
    n = 50000
    costs = np.stack([rng.integers(-400, 400, n), rng.integers(1, 200, n)], 1).astype(np.int16)
    costs[::17, 1] = 32000
    d_c = to_dev(costs)
    for maxcost in (1000, 50):
        d_o = empty((n,), torch_cuda.int16)
        check(lib().cuphu_mst_costs_device(dptr(d_c), n, 200, maxcost, dptr(d_o), None))
        pos, neg, _ = O.incrcost(costs, np.zeros(n, np.int16), nshortcycle=200, nflow=1)
        assert np.array_equal(to_host(d_o), _mst_from(pos, neg, maxcost))


def test_mcf_inputs_defo_costs_and_residues(torch_cuda):
    ig, g, _, _ = S.bumps(80, 90, seed=3, nbumps=2)
    ig = np.ascontiguousarray(ig, np.complex64)
    nr, nc = g.shape
    narcs = (nr - 1) * nc + nr * (nc - 1)
    p = default_params(nlooks=5.0, ncorrlooks=5.0)
    costs = np.empty((narcs, 4), np.int16)
    res = np.empty((nr - 1, nc - 1), np.int8)
    re, im = np.ascontiguousarray(ig.real), np.ascontiguousarray(ig.imag)
    check(lib().cuphu_mcf_inputs(ptr(re), ptr(im), ptr(g), None, nr, nc, 1, C.byref(p), 0,
                                 ptr(costs), None, ptr(res)))
    ph = O.phase_from_igram(ig)
    assert np.array_equal(costs, O.build_costs(ph, g, 5.0, mode=1))
    assert np.array_equal(res, O.residues(ph))
    mst = np.empty(narcs, np.int16)
    with pytest.raises(NotImplementedError):
        check(lib().cuphu_mcf_inputs(ptr(re), ptr(im), ptr(g), None, nr, nc, 1, C.byref(p), 0,
                                     ptr(costs), ptr(mst), None))
    with pytest.raises(CuPhuError):
        check(lib().cuphu_mcf_inputs(ptr(re), ptr(im), ptr(g), None, 1, nc, 0, C.byref(p), 0,
                                     ptr(costs), None, None))
