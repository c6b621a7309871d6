"""End-to-end GPU unwrapping: the full pipeline (weights, persistent solve,
labelling, tile registration, merge, reference-pixel shift) against the FP64
oracle restatement of the reference's tiled pipeline, the batched entry
point against per-scene calls, and the reference test suite's behavioural
checks (test_unwrap.py, test_reference_pixel.py, test_mask_pad_distance.py,
test_conncomp.py) on the Python drop-in ``unwrap``."""
import ctypes as C

import numpy as np
import pytest

import cuphu_b200 as cuphu
import oracle as O
from cuphu_b200 import synthetic as S
from cuphu_b200._lib import (CuPhuScene, CuPhuSolveStats, check, default_params,
                             default_solve_options, default_tile_params, lib)
from tests.devbuf import dptr, empty, to_dev, to_host

pytestmark = pytest.mark.gpu


def device_unwrap(torch, ph, g, nlooks, ntiles, ovl, precision=1, n_irls=2, mask=None,
                  conf=None, ref=(-1, -1), mode=0):
    nr, nc = ph.shape
    dph, dg = to_dev(ph), to_dev(g)
    dm = to_dev(mask) if mask is not None else None
    dcf = to_dev(conf) if conf is not None else None
    du = empty((nr, nc), torch.float32)
    dc = empty((nr, nc), torch.int32)
    p = default_params(nlooks=float(nlooks), ncorrlooks=float(nlooks))
    t = default_tile_params(ntilerow=ntiles[0], ntilecol=ntiles[1], rowovrlp=ovl[0],
                            colovrlp=ovl[1])
    o = default_solve_options(precision=precision, n_irls=n_irls, ref_row=ref[0],
                              ref_col=ref[1])
    st = CuPhuSolveStats()
    check(lib().cuphu_unwrap_device(None, dptr(dph), dptr(dg), dptr(dm), dptr(dcf), nr, nc, mode,
                                    C.byref(p), C.byref(t), C.byref(o), dptr(du), dptr(dc), None,
                                    C.byref(st), None))
    return to_host(du), to_host(dc).view(np.uint32), st


@pytest.mark.parametrize("ntiles,ovl", [((1, 1), (0, 0)), ((2, 2), (16, 16)),
                                        ((2, 3), (12, 9)), ((3, 1), (8, 0))])
def test_pipeline_bit_exact_vs_oracle(torch_cuda, ntiles, ovl):
    ig, g, _, _ = S.bumps(120, 150, seed=4, nbumps=3, amp_range=(10, 30), sigma_range=(10, 30))
    ph = O.phase_from_igram(ig)
    g = g.copy()
    g[40:60, 20:50] = 0.03
    mask = np.ones(ph.shape, np.uint8)
    mask[90:100, 100:140] = 0
    want_u, want_c, _ = O.unwrap_tiled(ph, g, 5.0, mode=0, mask=mask, ntiles=ntiles,
                                       overlap=ovl, opts=O.lap_opts(n_irls=2))
    got_u, got_c, st = device_unwrap(torch_cuda, ph, g, 5.0, ntiles, ovl, mask=mask)
    assert st.ntiles == ntiles[0] * ntiles[1]
    assert np.array_equal(got_c, want_c)
    assert np.array_equal(got_u.view(np.int32), want_u.view(np.int32))


def test_batch_matches_individual_calls(torch_cuda):
    shapes = [(96, 130), (64, 64), (150, 77)]
    tiles = [((2, 2), (16, 16)), ((1, 1), (0, 0)), ((2, 1), (10, 0))]
    data, singles = [], []
    for i, (sh, (nt, ov)) in enumerate(zip(shapes, tiles)):
        ig, g, _, _ = S.bumps(*sh, seed=20 + i, nbumps=2, amp_range=(5, 20), sigma_range=(8, 20))
        ph = O.phase_from_igram(ig)
        data.append((ph, g, nt, ov))
        singles.append(device_unwrap(torch_cuda, ph, g, 5.0, nt, ov, precision=0, n_irls=2))
    scenes = (CuPhuScene * len(data))()
    keep = []
    for i, (ph, g, nt, ov) in enumerate(data):
        dph, dg = to_dev(ph), to_dev(g)
        du = empty(ph.shape, torch_cuda.float32)
        dc = empty(ph.shape, torch_cuda.int32)
        keep += [dph, dg, du, dc]
        scenes[i] = CuPhuScene(None, dph.data_ptr(), dg.data_ptr(), None, None, ph.shape[0],
                               ph.shape[1], nt[0], nt[1], ov[0], ov[1], 5.0, du.data_ptr(),
                               dc.data_ptr())
    p = default_params()
    o = default_solve_options(precision=0, n_irls=2)
    st = CuPhuSolveStats()
    check(lib().cuphu_unwrap_batch_device(scenes, len(data), 0, C.byref(p), C.byref(o),
                                          C.byref(st), None))
    assert st.ntiles == 4 + 1 + 2
    for i in range(len(data)):
        u = to_host(keep[4 * i + 2])
        c = to_host(keep[4 * i + 3]).view(np.uint32)
        assert np.array_equal(u.view(np.int32), singles[i][0].view(np.int32))
        assert np.array_equal(c, singles[i][1])


def test_batch_graph_replays_the_batch(torch_cuda):
    """cuphu_batch_graph_*: replaying the captured pipeline gives the batched
    call's outputs bit for bit, twice in a row and after the inputs are
    refilled in place."""
    shapes = [(96, 130), (64, 64), (150, 77), (40, 200)]
    tiles = [((2, 2), (16, 16)), ((1, 1), (0, 0)), ((2, 1), (10, 0)), ((1, 2), (0, 12))]
    sets = []
    for seed in (30, 40):
        sets.append([O.phase_from_igram(S.bumps(*sh, seed=seed + i, nbumps=2, amp_range=(5, 20),
                                                sigma_range=(8, 20))[0]) for i, sh in
                     enumerate(shapes)])
    gs = [S.bumps(*sh, seed=50 + i, nbumps=2)[1] for i, sh in enumerate(shapes)]
    dph = [to_dev(a) for a in sets[0]]
    dg = [to_dev(g) for g in gs]
    du = [empty(sh, torch_cuda.float32) for sh in shapes]
    dc = [empty(sh, torch_cuda.int32) for sh in shapes]
    scenes = (CuPhuScene * len(shapes))()
    for i, (sh, (nt, ov)) in enumerate(zip(shapes, tiles)):
        scenes[i] = CuPhuScene(None, dph[i].data_ptr(), dg[i].data_ptr(), None, None, sh[0], sh[1],
                               nt[0], nt[1], ov[0], ov[1], 5.0, du[i].data_ptr(), dc[i].data_ptr())
    p = default_params()
    o = default_solve_options(precision=0, n_irls=2)

    def batch_outputs():
        check(lib().cuphu_unwrap_batch_device(scenes, len(shapes), 0, C.byref(p), C.byref(o),
                                              None, None))
        return [(to_host(u).copy(), to_host(c).copy()) for u, c in zip(du, dc)]

    want = [batch_outputs()]
    for i in range(len(shapes)):
        dph[i].copy_(to_dev(sets[1][i]))
    want.append(batch_outputs())
    for i in range(len(shapes)):
        dph[i].copy_(to_dev(sets[0][i]))
    graph = C.c_void_p()
    check(lib().cuphu_batch_graph_create(scenes, len(shapes), 0, C.byref(p), C.byref(o),
                                         C.byref(graph)))
    try:
        for k in (0, 0, 1):
            for i in range(len(shapes)):
                dph[i].copy_(to_dev(sets[k][i]))
                du[i].fill_(float("nan"))
            stream = torch_cuda.cuda.current_stream().cuda_stream
            check(lib().cuphu_batch_graph_launch(graph, C.c_void_p(stream)))
            for i in range(len(shapes)):
                assert np.array_equal(to_host(du[i]).view(np.int32), want[k][i][0].view(np.int32))
                assert np.array_equal(to_host(dc[i]), want[k][i][1])
    finally:
        check(lib().cuphu_batch_graph_destroy(graph))


def test_autotune_keeps_results(torch_cuda):
    """After cuphu_autotune stores its choices for this size, costs stay bit
    exact and the FP64 pipeline stays bit exact with the oracle."""
    import cuphu_b200
    ig, g, _, _ = S.bumps(200, 260, seed=61, nbumps=3, amp_range=(5, 20), sigma_range=(8, 30))
    ph = O.phase_from_igram(ig)
    base_u, base_c, _ = device_unwrap(torch_cuda, ph, g, 5.0, (2, 2), (16, 16), precision=1,
                                      n_irls=2)
    ch = cuphu_b200.autotune(ig, g, 5.0, cost="defo", ntiles=(2, 2), tile_overlap=(16, 16))
    assert ch["cost_blocks_per_sm"] in (3, 4) and ch["solver_blocks_per_sm"] in (1, 2)
    assert ch["solver_stages"] in (2, 3, 6)
    u, c, _ = device_unwrap(torch_cuda, ph, g, 5.0, (2, 2), (16, 16), precision=1, n_irls=2)
    assert np.array_equal(u.view(np.int32), base_u.view(np.int32))
    assert np.array_equal(c, base_c)
    from tests.test_gpu_kernels import gpu_costs
    got = gpu_costs(torch_cuda, ph, g, 5.0, 1)
    assert np.array_equal(got, O.build_costs(ph, g, 5.0, mode=1))


def test_solver_launch_shapes_give_identical_results(torch_cuda):
    """Every launch shape of the persistent solver (ring stages x resident
    blocks per SM) gives bit-identical unwraps and labels, in both
    precisions: the reductions do not depend on the shape."""
    ig, g, _, _ = S.bumps(230, 300, seed=62, nbumps=3, amp_range=(5, 25), sigma_range=(8, 30))
    ph = O.phase_from_igram(ig)
    for prec, nshape in ((0, 3), (1, 2)):
        outs = []
        for v in range(nshape):
            check(lib().cuphu_test_force_solve_shape(v))
            try:
                outs.append(device_unwrap(torch_cuda, ph, g, 5.0, (2, 2), (16, 16),
                                          precision=prec, n_irls=2)[:2])
            finally:
                check(lib().cuphu_test_force_solve_shape(-1))
        for u, c in outs[1:]:
            assert np.array_equal(u.view(np.int32), outs[0][0].view(np.int32))
            assert np.array_equal(c, outs[0][1])


def test_reference_pixel_shift_and_cc_on_device(torch_cuda):
    ig, g, _, _ = S.bumps(90, 110, seed=8, nbumps=2, amp_range=(10, 30), sigma_range=(10, 30))
    ph = O.phase_from_igram(ig)
    u0, c0, _ = device_unwrap(torch_cuda, ph, g, 5.0, (2, 2), (16, 16), precision=0)
    u1, c1, _ = device_unwrap(torch_cuda, ph, g, 5.0, (2, 2), (16, 16), precision=0,
                              ref=(45, 70))
    n = (u0[45, 70] - ph[45, 70]) / (2 * np.pi)
    assert np.array_equal(c0, c1)
    assert abs(u1[45, 70] - ph[45, 70]) < 1e-4
    assert np.allclose(u0 - u1, np.float32(round(n) * 2 * np.pi), atol=1e-4)


# ── reference test-suite behaviour on the Python drop-in ───────────────────

@pytest.fixture()
def small_igram():
    r = np.arange(50, dtype=np.float32)
    c = np.arange(60, dtype=np.float32)
    return np.exp(1j * (0.1 * r[:, None] + 0.2 * c[None, :])).astype(np.complex64)


@pytest.fixture()
def small_corr():
    return np.full((50, 60), 0.9, dtype=np.float32)


def test_returns_correct_shape_and_finite(small_igram, small_corr):
    unw, cc = cuphu.unwrap(small_igram, small_corr, nlooks=10.0, init="laplace")
    assert unw.shape == small_igram.shape and cc.shape == small_igram.shape
    assert unw.dtype == np.float32 and cc.dtype == np.uint32
    assert np.isfinite(unw).all()


def test_rewrap_consistency(small_igram, small_corr):
    unw, _ = cuphu.unwrap(small_igram, small_corr, nlooks=10.0, init="laplace")
    diff = np.abs(np.angle(np.exp(1j * unw)) - np.angle(small_igram))
    diff = np.where(diff > np.pi, 2 * np.pi - diff, diff)
    assert float(np.nanpercentile(diff, 99)) < 0.1


def test_masked_pixels_have_cc_zero(small_igram, small_corr):
    mask = np.ones((50, 60), dtype=np.uint8)
    mask[20:30, 20:40] = 0
    unw, cc = cuphu.unwrap(small_igram, small_corr, nlooks=10.0, init="laplace", mask=mask)
    assert (cc[20:30, 20:40] == 0).all()


@pytest.mark.parametrize("cost", ["smooth", "defo", "topo"])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_cost_modes_and_precisions(small_igram, small_corr, cost, precision):
    unw, _ = cuphu.unwrap(small_igram, small_corr, nlooks=10.0, cost=cost, init="laplace",
                          precision=precision)
    assert np.isfinite(unw).all()


def test_pre_allocated_output(small_igram, small_corr):
    ub = np.zeros((50, 60), np.float32)
    cb = np.zeros((50, 60), np.uint32)
    u, c = cuphu.unwrap(small_igram, small_corr, nlooks=10.0, init="laplace", unw=ub, conncomp=cb)
    assert u is ub and c is cb and np.isfinite(ub).all()


@pytest.mark.parametrize("ntiles", [(1, 1), (2, 2), (2, 3)])
def test_tiled_matches_single(small_igram, small_corr, ntiles):
    ref, _ = cuphu.unwrap(small_igram, small_corr, nlooks=10.0, init="laplace", ntiles=(1, 1))
    til, _ = cuphu.unwrap(small_igram, small_corr, nlooks=10.0, init="laplace", ntiles=ntiles,
                          tile_overlap=4)
    assert float(np.percentile(np.abs(ref - til), 95)) < 0.5


def test_nan_input_stays_finite(small_corr):
    igram = np.full((50, 60), np.nan + 0j, dtype=np.complex64)
    unw, _ = cuphu.unwrap(igram, small_corr, nlooks=10.0, init="laplace")
    assert np.isfinite(unw).all()


def _ramp():
    unw_true = 0.05 * np.arange(90)[None, :] * np.ones((60, 1)) + 10.0
    return (np.exp(1j * unw_true).astype(np.complex64),
            np.full((60, 90), 0.8, dtype=np.float32))


def _wrapped(igram):
    phi = np.angle(igram)
    return np.where(phi < 0, phi + 2 * np.pi, phi)


def test_default_reference_pixel():
    ig, corr = _ramp()
    unw, _ = cuphu.unwrap(ig, corr, nlooks=10.0, init="laplace")
    assert unw[0, 0] == pytest.approx(_wrapped(ig)[0, 0], abs=1e-4)


def test_reference_pixel_none_and_custom():
    ig, corr = _ramp()
    a, _ = cuphu.unwrap(ig, corr, nlooks=10.0, init="laplace")
    b, _ = cuphu.unwrap(ig, corr, nlooks=10.0, init="laplace", reference_pixel=None)
    n = (a - b)[0, 0] / (2 * np.pi)
    assert abs(n - round(n)) < 1e-3
    c, _ = cuphu.unwrap(ig, corr, nlooks=10.0, init="laplace", reference_pixel=(30, 45))
    assert c[30, 45] == pytest.approx(_wrapped(ig)[30, 45], abs=1e-4)


def test_reference_pixel_masked():
    ig, corr = _ramp()
    mask = np.ones((60, 90), np.uint8)
    mask[0, 0] = 0
    unw, cc = cuphu.unwrap(ig, corr, nlooks=10.0, init="laplace", mask=mask)
    assert np.isfinite(unw).all() and cc[0, 0] == 0


def test_mask_pad_distance_restores_original_mask():
    unw_true = 0.05 * np.arange(100)[None, :] * np.ones((100, 1))
    ig = np.exp(1j * unw_true).astype(np.complex64)
    corr = np.full((100, 100), 0.8, dtype=np.float32)
    mask = np.ones((100, 100), np.uint8)
    mask[:, 40:60] = 0
    for pad in (0, 5, 20, 50):
        _, cc = cuphu.unwrap(ig, corr, nlooks=10.0, init="laplace", mask=mask,
                             mask_pad_distance=pad)
        assert (cc[:, 40:60] == 0).all()
        assert (cc[:, :40] != 0).any()


def test_default_zero_pad_matches_no_padding():
    unw_true = 0.04 * np.arange(60)[None, :] * np.ones((60, 1))
    ig = np.exp(1j * unw_true).astype(np.complex64)
    corr = np.full((60, 60), 0.8, dtype=np.float32)
    mask = np.ones((60, 60), np.uint8)
    mask[:, 25:35] = 0
    a = cuphu.unwrap(ig, corr, nlooks=10.0, init="laplace", mask=mask)
    b = cuphu.unwrap(ig, corr, nlooks=10.0, init="laplace", mask=mask, mask_pad_distance=0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_gpu_conncomp_matches_cpu_sizes():
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    nr, nc = 20, 30
    corr = np.full((nr, nc), 0.8, dtype=np.float32)
    corr[:, 14:16] = 0.0
    unw = (0.05 * np.arange(nc)[None, :] * np.ones((nr, 1))).astype(np.float32)
    ig = np.exp(1j * unw).astype(np.complex64)
    valid = corr >= 0.1
    h = valid[:, :-1] & valid[:, 1:] & (np.abs(unw[:, :-1] - unw[:, 1:]) < np.pi)
    v = valid[:-1, :] & valid[1:, :] & (np.abs(unw[:-1, :] - unw[1:, :]) < np.pi)
    idx = np.arange(nr * nc).reshape(nr, nc)
    g = coo_matrix((np.ones(h.sum() + v.sum()),
                    (np.concatenate([idx[:, :-1][h], idx[:-1, :][v]]),
                     np.concatenate([idx[:, 1:][h], idx[1:, :][v]]))), shape=(nr * nc,) * 2)
    _, lab = connected_components(g, directed=False)
    lab = lab.reshape(nr, nc) + 1
    lab[~valid] = 0
    cpu = sorted(np.bincount(lab.ravel())[1:][np.bincount(lab.ravel())[1:] > 0].tolist())
    _, gcc = cuphu.unwrap(ig, corr, nlooks=10.0, cost="smooth", init="laplace")
    gpu = sorted(np.bincount(gcc.ravel())[1:].tolist())
    assert len(cpu) == 2 and cpu == [x for x in gpu if x > 0]


def test_regrow_conncomp_gpu():
    unw = np.zeros((20, 30), np.float32)
    unw[:, 15:] += 10.0
    corr = np.full((20, 30), 0.8, np.float32)
    cc = cuphu.regrow_conncomp(unw, corr, cost_thresh=0.1)
    assert cc.dtype == np.uint32 and set(np.unique(cc)) == {1, 2}
    want = O.conncomp(unw, corr)
    assert np.array_equal(cc, want)


def test_gpu_info():
    info = cuphu.gpu_info(0)
    assert info["total_memory"] > 0 and "B200" in info["name"] or info["total_memory"] > 0
