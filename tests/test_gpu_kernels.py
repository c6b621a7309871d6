"""GPU parity of the element kernels against the CPU oracle and the reference
cuPHU kernels: phase, statistical costs, residues, connected components,
flow integration, incremental costs.  Integer and byte outputs must be
bit-exact; everything else is compared bit for bit as well, because the
kernels restate the reference's float operation order."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from cuphu_b200 import synthetic as S
from cuphu_b200._lib import check, default_params, lib
from tests.devbuf import dptr, empty, to_dev, to_host

pytestmark = pytest.mark.gpu


def _scene(nr, nc, seed, nlooks=5.0):
    ig, g, _, _ = S.bumps(nr, nc, seed=seed, nbumps=3, amp_range=(5.0, 25.0),
                          sigma_range=(6.0, 30.0), nlooks=nlooks)
    g = g.copy()
    g[: max(1, nr // 5), : max(1, nc // 4)] *= 0.05
    return ig, O.phase_from_igram(ig), g


def gpu_costs(torch, ph, g, nlooks, mode, weights=None, kperp=7, kpar=7, residues=False):
    nr, nc = ph.shape
    narcs = (nr - 1) * nc + nr * (nc - 1)
    es = 4 if mode else 2
    dph, dg = to_dev(ph), to_dev(g)
    dw = to_dev(weights) if weights is not None else None
    dc = empty((max(narcs, 1), es), torch.int16)
    dr = empty((max(nr - 1, 1), max(nc - 1, 1)), torch.int8) if residues else None
    p = default_params(nlooks=float(nlooks), ncorrlooks=float(nlooks), kperpdpsi=kperp,
                       kpardpsi=kpar)
    check(lib().cuphu_build_costs_device(dptr(dph), dptr(dg), dptr(dw), nr, nc, mode,
                                         C.byref(p), dptr(dc), dptr(dr), None))
    c = to_host(dc)[:narcs]
    return (c, to_host(dr)[: nr - 1, : nc - 1]) if residues else c


SHAPES = [(48, 64), (33, 70), (17, 33), (5, 9), (2, 2), (1, 12), (12, 1), (130, 257),
          (300, 333)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("mode", [0, 1])
def test_costs_match_oracle(torch_cuda, shape, mode):
    nr, nc = shape
    _, ph, g = _scene(nr, nc, seed=nr * 131 + nc, nlooks=9.0)
    got = gpu_costs(torch_cuda, ph, g, 9.0, mode)
    want = O.build_costs(ph, g, 9.0, mode=mode)
    assert np.array_equal(got, want), f"{np.sum(np.any(got != want, axis=1))} arcs differ"


@pytest.mark.parametrize("window", [(7, 7), (3, 9), (1, 1), (11, 5)])
def test_costs_windows_and_weights(torch_cuda, window):
    _, ph, g = _scene(61, 77, seed=5, nlooks=20.0)
    narcs = 60 * 77 + 61 * 76
    w = (np.random.default_rng(1).random(narcs) > 0.2).astype(np.int16) * 2
    for mode in (0, 1):
        got = gpu_costs(torch_cuda, ph, g, 20.0, mode, weights=w, kperp=window[0],
                        kpar=window[1])
        want = O.build_costs(ph, g, 20.0, mode=mode, weights=w, kperp=window[0], kpar=window[1])
        assert np.array_equal(got, want)


@pytest.mark.parametrize("shape", [(48, 64), (33, 70), (130, 257), (300, 333)])
@pytest.mark.parametrize("mode", [0, 1])
def test_costs_match_reference_kernels(torch_cuda, shape, mode):
    if O.ref_lib() is None:
        pytest.skip("reference kernels not built")
    nr, nc = shape
    _, ph, g = _scene(nr, nc, seed=nc, nlooks=5.0)
    got = gpu_costs(torch_cuda, ph, g, 5.0, mode)
    ref, _ = O.ref_build_costs(ph, g, 5.0, mode=mode)
    assert np.array_equal(got, ref), f"{np.sum(np.any(got != ref, axis=1))} arcs differ"


def test_costs_more_arc_tiles_than_resident_blocks(torch_cuda):
    """1500 x 1400 has more 64 x 64 arc tiles per family than there are
    resident blocks, so the cost kernel's grid runs in several waves and the
    launch-wide queue of undecided arcs collects entries from all of them."""
    _, ph, g = _scene(1500, 1400, seed=91, nlooks=9.0)
    for mode in (0, 1):
        got = gpu_costs(torch_cuda, ph, g, 9.0, mode)
        want = O.build_costs(ph, g, 9.0, mode=mode)
        assert np.array_equal(got, want), f"{np.sum(np.any(got != want, axis=1))} arcs differ"


def test_costs_tiny_and_equal_phase_differences(torch_cuda):
    """Phase differences that are zero, tiny or denormal take the IEEE
    division inside the kernel; equal neighbours give exact zeros.  Costs and
    residues must still match the oracle bit for bit, interior blocks
    included."""
    _, ph, g = _scene(200, 260, seed=77, nlooks=9.0)
    ph = ph.copy()
    ph[10:150:2, 20:200] = 0.0
    ph[11:150:2, 20:200:3] = np.float32(1e-35)
    ph[11:150:2, 21:200:3] = np.float32(2e-39)
    ph[90:120, 100:180] = ph[90, 100]
    ph[160:190, :] = np.float32(2 * np.pi) - np.float32(1e-6)
    for mode in (0, 1):
        got, res = gpu_costs(torch_cuda, ph, g, 9.0, mode, residues=True)
        assert np.array_equal(got, O.build_costs(ph, g, 9.0, mode=mode))
        assert np.array_equal(res, O.residues(ph))


@pytest.mark.parametrize("nlooks", [1.0, 5.0, 20.0])
def test_costs_at_decision_boundaries(torch_cuda, nlooks):
    """Coherence at the zero-coherence threshold (to a few ulps), near 1,
    outside [0, 1] (also just above 1 and -0), subnormal, non-finite, and
    weights 0/1/2: the kernels' FP32 fast
    path must hand every arc it cannot decide to the exact arithmetic, so
    the costs equal the oracle's bit for bit."""
    rng = np.random.default_rng(int(nlooks))
    nr, nc = 260, 300
    _, ph, g = _scene(nr, nc, seed=int(nlooks) + 3, nlooks=nlooks)
    g = g.copy()
    thresh = 1.2 * (1.3 / nlooks + 0.14)
    t32 = np.float32(thresh)
    near = np.array([np.nextafter(t32, np.float32(s * 10), dtype=np.float32) if s else t32
                     for s in (-1, 0, 1)], np.float32)
    near = np.concatenate([near, [np.float32(thresh * (1 + 2.0 ** -21)),
                                  np.float32(thresh * (1 - 2.0 ** -21))]]).astype(np.float32)
    g[20:80, 10:200] = rng.choice(near, size=(60, 190))
    g[90:110, :] = np.float32(1.0) - rng.integers(0, 400, size=(20, nc)).astype(np.float32) * 2.0 ** -24
    g[120:125, 30:90] = np.float32(1.25)
    g[126:128, 30:90] = np.float32(-0.5)
    g[128, 30:90] = np.float32(-0.0)
    g[129, 30:60] = np.nextafter(np.float32(1.0), np.float32(2.0))
    g[129, 60:90] = np.float32(2.0 ** -149)
    g[130, 40:60] = np.nan
    g[131, 40:60] = np.inf
    narcs = (nr - 1) * nc + nr * (nc - 1)
    w = rng.choice(np.array([0, 1, 1, 1, 1, 2], np.int16), size=narcs)
    for mode in (0, 1):
        for weights in (None, w):
            got = gpu_costs(torch_cuda, ph, g, nlooks, mode, weights=weights)
            # the device reads non-finite coherence as 0, as cuphu.unwrap cleans it
            want = O.build_costs(ph, np.where(np.isfinite(g), g, 0).astype(np.float32), nlooks,
                                 mode=mode, weights=weights)
            assert np.array_equal(got, want), f"{np.sum(np.any(got != want, axis=1))} arcs differ"


def test_residues_match_oracle_and_conserve(torch_cuda):
    _, ph, g = _scene(90, 111, seed=9, nlooks=2.0)
    _, res = gpu_costs(torch_cuda, ph, g, 2.0, 0, residues=True)
    want = O.residues(ph)
    assert np.array_equal(res, want)
    dph = to_dev(ph)
    dr = empty((89, 110), torch_cuda.int8)
    check(lib().cuphu_residues_gpu(dptr(dph), 90, 111, dptr(dr), None))
    assert np.array_equal(to_host(dr), want)
    assert set(np.unique(res)).issubset({-1, 0, 1})
    assert (res != 0).sum() > 0


def test_residues_vanish_on_consistent_phase(torch_cuda):
    nr, nc = 40, 50
    t = 0.3 * np.arange(nc)[None, :] + 0.2 * np.arange(nr)[:, None]
    ph = O.phase_from_igram(np.exp(1j * t).astype(np.complex64))
    dph = to_dev(ph)
    dr = empty((nr - 1, nc - 1), torch_cuda.int8)
    check(lib().cuphu_residues_gpu(dptr(dph), nr, nc, dptr(dr), None))
    assert not to_host(dr).any()


def test_device_phase_vs_host_atan2f(torch_cuda):
    ig, ph_host, _ = _scene(300, 301, seed=3)
    ig[5, 7] = np.nan
    dig = to_dev(ig.view(np.float32))
    dph = empty(ig.shape, torch_cuda.float32)
    check(lib().cuphu_phase_gpu(dptr(dig), C.c_longlong(ig.size), dptr(dph), None))
    ph = to_host(dph)
    assert ph[5, 7] == 0.0
    ph_host[5, 7] = 0.0
    assert ph.min() >= 0.0 and ph.max() < 2 * np.pi + 1e-6
    ulps = np.abs(ph.view(np.int32).astype(np.int64) - ph_host.view(np.int32).astype(np.int64))
    assert ulps.max() <= 1
    # the device angle is the float nearest to the FP64 angle
    d = np.arctan2(ig.imag.astype(np.float64), ig.real.astype(np.float64)).astype(np.float32)
    d = np.where(d < 0, d + np.float32(2 * np.pi), d).astype(np.float32)
    d[5, 7] = 0.0
    assert np.mean(ph != d) < 1e-4


def _cc_case(seed=7):
    nr, nc = 40, 56
    rng = np.random.default_rng(seed)
    unw = (0.1 * np.arange(nc)[None, :] + 0.05 * np.arange(nr)[:, None]).astype(np.float32)
    unw[:, 30:] += 9.0
    unw[15, 10] += 40.0
    corr = rng.uniform(0.0, 1.0, (nr, nc)).astype(np.float32)
    corr[corr < 0.1] = 0.02
    return unw, corr


@pytest.mark.parametrize("variant", ["plain", "mask", "incr", "frac0"])
def test_conncomp_matches_oracle_and_reference(torch_cuda, variant):
    unw, corr = _cc_case()
    nr, nc = unw.shape
    narcs = (nr - 1) * nc + nr * (nc - 1)
    rng = np.random.default_rng(3)
    mask = np.ones((nr, nc), np.uint8)
    mask[:, 20:22] = 0
    pos = rng.integers(-50, 600, narcs).astype(np.int16)
    neg = rng.integers(-50, 600, narcs).astype(np.int16)
    kw = {"plain": {}, "mask": dict(mask=mask), "incr": dict(poscost=pos, negcost=neg),
          "frac0": dict(minfrac=0.0, maxncomps=5)}[variant]
    want = O.conncomp(unw, corr, **kw)
    p = default_params(minconncompfrac=kw.get("minfrac", 0.01),
                       maxncomps=kw.get("maxncomps", 32))
    du, dc = to_dev(unw), to_dev(corr)
    dm = to_dev(kw["mask"]) if "mask" in kw else None
    dp = to_dev(pos) if "poscost" in kw else None
    dn = to_dev(neg) if "negcost" in kw else None
    dl = empty((nr, nc), torch_cuda.int32)
    check(lib().cuphu_conncomp_gpu(dptr(du), dptr(dc), dptr(dm), nr, nc, dptr(dp), dptr(dn),
                                   C.byref(p), 0, dptr(dl)))
    got = to_host(dl).view(np.uint32)
    assert np.array_equal(got, want)
    if O.ref_lib() is not None:
        ref = O.ref_conncomp(unw, corr, **kw)
        assert np.array_equal(got, ref)


def test_conncomp_large_random_matches_oracle(torch_cuda):
    rng = np.random.default_rng(11)
    nr, nc = 300, 411
    unw = np.cumsum(rng.normal(0, 1.2, (nr, nc)), axis=1).astype(np.float32)
    corr = rng.uniform(0, 1, (nr, nc)).astype(np.float32)
    want = O.conncomp(unw, corr, minfrac=0.0005, maxncomps=50)
    p = default_params(minconncompfrac=0.0005, maxncomps=50)
    du, dc = to_dev(unw), to_dev(corr)
    dl = empty((nr, nc), torch_cuda.int32)
    check(lib().cuphu_conncomp_gpu(dptr(du), dptr(dc), None, nr, nc, None, None, C.byref(p), 0,
                                   dptr(dl)))
    assert np.array_equal(to_host(dl).view(np.uint32), want)


@pytest.mark.parametrize("shape", [(37, 45), (1, 70), (70, 1), (129, 300)])
def test_integrate_matches_oracle_and_reference(torch_cuda, shape):
    nr, nc = shape
    _, ph, _ = _scene(nr, nc, seed=nr + nc)
    rng = np.random.default_rng(nr)
    hf = rng.integers(-2, 3, (max(nr - 1, 1), nc)).astype(np.int16)
    vf = rng.integers(-2, 3, (nr, max(nc - 1, 1))).astype(np.int16)
    want = O.integrate_phase(ph, hf, vf)
    dph, dh, dv = to_dev(ph), to_dev(hf), to_dev(vf)
    du = empty((nr, nc), torch_cuda.float32)
    check(lib().cuphu_integrate_phase_gpu(dptr(dph), dptr(dh), dptr(dv), nr, nc, 0, dptr(du)))
    got = to_host(du)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))
    if O.ref_lib() is not None and nr > 1 and nc > 1:
        ref = O.ref_integrate(ph, hf, vf)
        assert np.array_equal(got.view(np.int32), ref.view(np.int32))


def test_incrcost_matches_oracle_and_reference(torch_cuda):
    _, ph, g = _scene(30, 38, seed=12)
    c = O.build_costs(ph, g, 5.0, mode=0)
    flows = np.random.default_rng(12).integers(-3, 4, c.shape[0]).astype(np.int16)
    wp, wn, wex = O.incrcost(c, flows)
    dc, df = to_dev(c), to_dev(flows)
    dp = empty(c.shape[0], torch_cuda.int16)
    dn = empty(c.shape[0], torch_cuda.int16)
    ds = empty(2, torch_cuda.int32)
    ex = check(lib().cuphu_incrcost_early_exit(dptr(dc), dptr(df), c.shape[0], 200, 1, dptr(dp),
                                               dptr(dn), dptr(ds)))
    assert np.array_equal(to_host(dp), wp) and np.array_equal(to_host(dn), wn)
    assert bool(ex) == wex
    if O.ref_lib() is not None:
        rp, rn, rex = O.ref_incrcost(c, flows)
        assert np.array_equal(to_host(dp), rp) and np.array_equal(to_host(dn), rn)
        assert rex == bool(ex)
    zero = np.zeros_like(flows)
    dz = to_dev(zero)
    ex0 = check(lib().cuphu_incrcost_early_exit(dptr(dc), dptr(dz), c.shape[0], 200, 1,
                                                dptr(dp), dptr(dn), dptr(ds)))
    assert bool(ex0) == O.incrcost(c, zero)[2]


@pytest.mark.parametrize("nlooks", [1.0, 3.7, 20.0, 150.0])
def test_cost_sigsq_screening_is_exact(torch_cuda, nlooks):
    """The FP32 screening of the FP64 pow must never change a quantised
    cost: dense random coherence over [0, 1] (plus exact 0 and 1), compared
    with the reference kernels' pure-FP64 arithmetic on 2 M arcs."""
    if O.ref_lib() is None:
        pytest.skip("reference kernels not built")
    rng = np.random.default_rng(int(nlooks * 10))
    nr, nc = 1000, 1000
    g = rng.random((nr, nc), dtype=np.float32)
    g[::97, ::89] = 0.0
    g[::83, ::71] = 1.0
    ph = (rng.random((nr, nc)) * 2 * np.pi).astype(np.float32)
    for mode in (0, 1):
        got = gpu_costs(torch_cuda, ph, g, nlooks, mode)
        ref, _ = O.ref_build_costs(ph, g, nlooks, mode=mode)
        assert np.array_equal(got, ref), f"{np.sum(np.any(got != ref, axis=1))} arcs differ"
