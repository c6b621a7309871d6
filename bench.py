"""Benchmark of the unwrapping path: Mpix/s unwrapped at 8192^2.

Workload (default): the 8192x8192 TOPO scene -- fractal power-law topography
(beta -3, 0..2500 m) through lambda 0.24 m, B_perp 150 m, R 850 km, look 35
deg; exponential amplitudes, coherence in [0.2, 0.9], nlooks 20 -- seeded
synthetic data, unwrapped with init='laplace' and the reference's defaults
(auto-tiling toward 1024 px with 64 px overlap -> 9x9 tiles, 16 IRLS passes,
1000 PCG iterations, tol 1e-3), cost build + Laplace PCG + congruence +
conncomp + stitching.

One JSON line on rank 0.  `value` = scene pixels of all ranks / device time
(inputs resident in HBM); `e2e` = the same through cuphu_unwrap_ex with
pinned host buffers (H2D of igram+corr and D2H of unw+conncomp inside the
timed region).  Extra keys: FP64-PCG throughput and the mixed-vs-FP64
cycle-map comparison, the cost-kernel bandwidth, the solver roofline, the
CPU baseline.  Multi-GPU: one process per GPU, independent replicas of the
scene (no data-path collective; "scaling": "weak").

--impl reference times the CPU restatement of the reference path (the
oracle: cost build + FP64 Jacobi-PCG/IRLS + conncomp) on one 967x967 tile
of the same scene with all host threads.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0
METRIC = "Mpix/s unwrapped at 8192^2 (mixed-precision Laplace PCG)"


# measured k_solve DRAM bytes (mixed precision), see the roofline block:
# ncu dram__bytes_read.sum + dram__bytes_write.sum of the 4096^2 case (4 x 4
# tiles, 18.39 M tile pixels) at 20, 40 and 60 PCG iterations of one pass:
# 17.84, 33.80 and 50.52 GB.  40 - 20: the marginal bytes per pixel-iteration;
# 20 iterations' intercept: the fixed bytes per tile pixel of a pass
# (assembly, fold, final); 60 - 40 beyond 20 iterations: the one true-residual
# replacement (at iteration 50)
TRAFFIC_PER_PX_ITER = 43.4
TRAFFIC_PER_PASS_PX = 102.3
TRAFFIC_PER_REPL_PX = 40.8


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_scene(workload, seed, scale=None):
    from cuphu_b200 import synthetic as S
    name = {"c2_8192_topo": "c2_8192_topo", "c1_4096_smooth": "c1_4096_smooth",
            "c0_512_defo": "c0_512_defo", "c4_2048_defo": "c4_2048_defo"}[workload]
    ig, g, truth, ex = S.config_scene(name, seed=seed, scale=scale)
    return ig, g, ex


def tiles_for(nrow, ncol):
    from cuphu_b200._unwrap import _auto_ntiles_by_target_size
    return _auto_ntiles_by_target_size(nrow, ncol, 1024, 64, 64)


def cpu_baseline(ig, g, nlooks, mode, n_irls):
    """The oracle (CPU restatement of the reference path) on one tile-sized
    crop of the scene: cost build + FP64 PCG/IRLS + conncomp."""
    import oracle as O
    n = 967
    ph = O.phase_from_igram(np.ascontiguousarray(ig[:n, :n]))
    gg = np.ascontiguousarray(g[:n, :n])
    t0 = time.perf_counter()
    c = O.build_costs(ph, gg, nlooks, mode=mode)
    _, _, unw, it = O.laplace_f64(c, ph, O.lap_opts(n_irls=n_irls))
    O.conncomp(unw, gg)
    dt = time.perf_counter() - t0
    return n * n / dt / 1e6, dt, int(it.sum()), n


def _tile_owner(n, nt, ovl, i):
    """Tile whose merged output holds row (or column) i: tiles are written in
    order and each keeps its interior minus half the overlap on inner sides
    (cuphu_solver.cpp:2002-2031), so the last tile covering i owns it."""
    import oracle as O
    own = 0
    for t in range(nt):
        f, ln = O.tile_bounds(n, nt, ovl, t)
        lo = f + (ovl // 2 if t > 0 else 0)
        hi = f + ln - (ovl // 2 if t < nt - 1 else 0)
        if lo <= i < hi:
            own = t
    return own


def flip_details(ph, g, nlooks, mode, flips, ntiles, ovl, n_irls, limit=8):
    """For pixels whose cycle differs between the mixed and FP64 solves of the
    tiled scene: the owning tile solved alone in both precisions (each
    tile's solve does not depend on the rest of the job), and the distance
    of each continuous solution from the half cycle at which the congruence
    projection rounds the other way, in cycles."""
    import torch
    import oracle as O
    from cuphu_b200._lib import CuPhuSolveStats, check, default_params, default_solve_options, lib
    L = lib()
    nrow, ncol = ph.shape
    out = []
    for (r, c) in flips[:limit]:
        tr, tc = _tile_owner(nrow, ntiles[0], ovl, r), _tile_owner(ncol, ntiles[1], ovl, c)
        r0, nr = O.tile_bounds(nrow, ntiles[0], ovl, tr)
        c0, nc = O.tile_bounds(ncol, ntiles[1], ovl, tc)
        tph = torch.from_numpy(np.ascontiguousarray(ph[r0:r0 + nr, c0:c0 + nc])).cuda()
        tg = torch.from_numpy(np.ascontiguousarray(g[r0:r0 + nr, c0:c0 + nc])).cuda()
        narcs = (nr - 1) * nc + nr * (nc - 1)
        cost = torch.empty((narcs, 4), dtype=torch.int16, device="cuda")
        pc = default_params(nlooks=nlooks, ncorrlooks=nlooks)
        check(L.cuphu_build_costs_device(C.c_void_p(tph.data_ptr()), C.c_void_p(tg.data_ptr()),
                                         None, nr, nc, 1, C.byref(pc), C.c_void_p(cost.data_ptr()),
                                         None, None))
        rec = {"pixel": [int(r), int(c)], "tile": [tr, tc]}
        for name, prec in (("mixed", 0), ("fp64", 1)):
            du = torch.empty((nr, nc), dtype=torch.float32, device="cuda")
            dcont = torch.empty((nr, nc), dtype=torch.float32, device="cuda")
            o = default_solve_options(precision=prec, n_irls=n_irls)
            st = CuPhuSolveStats()
            check(L.cuphu_laplace_solve_device(C.c_void_p(cost.data_ptr()), 4,
                                               C.c_void_p(tph.data_ptr()), nr, nc, C.byref(o),
                                               C.c_void_p(du.data_ptr()), None,
                                               C.c_void_p(dcont.data_ptr()), C.byref(st), None))
            torch.cuda.synchronize()
            u = float(dcont[r - r0, c - c0].item())
            d = (u - float(ph[r, c])) / (2 * np.pi)
            rec[f"cycles_{name}"] = d
            rec[f"half_cycle_distance_{name}"] = abs(d - np.floor(d) - 0.5)
        out.append(rec)
    return out


def parity_crop(ig, g, nlooks, mode, n=2880, n_irls=16):
    """FP64 GPU pipeline (host-buffer entry point, the reference's host
    phase) against the oracle's restatement of the reference pipeline on an
    n x n crop of the scene (3 x 3 auto tiles at n = 2880), plus the mixed
    solve's cycle mismatches against the same oracle."""
    import oracle as O
    from cuphu_b200._lib import (check, default_params, default_solve_options,
                                 default_tile_params, lib, ptr)
    from cuphu_b200._unwrap import _auto_ntiles_by_target_size
    L = lib()
    cig = np.ascontiguousarray(ig[:n, :n])
    cg = np.ascontiguousarray(g[:n, :n])
    nt = _auto_ntiles_by_target_size(n, n, 1024, 64, 64)
    p = default_params(nlooks=nlooks, ncorrlooks=nlooks)
    t = default_tile_params(ntilerow=nt[0], ntilecol=nt[1], rowovrlp=64, colovrlp=64)
    got = {}
    for name, prec in (("fp64", 1), ("mixed", 0)):
        o = default_solve_options(precision=prec, n_irls=n_irls, ref_row=-1, ref_col=-1)
        u = np.empty((n, n), np.float32)
        c = np.empty((n, n), np.uint32)
        check(L.cuphu_unwrap_ex(ptr(cig.view(np.float32)), ptr(cg), None, None, n, n, mode,
                                C.byref(p), C.byref(t), C.byref(o), 0, ptr(u), ptr(c), None))
        got[name] = (u, c)
    t0 = time.perf_counter()
    want_u, want_c, _ = O.unwrap_tiled(O.phase_from_igram(cig), cg, nlooks, mode=mode, ntiles=nt,
                                       overlap=(64, 64), opts=O.lap_opts(n_irls=n_irls))
    oracle_s = time.perf_counter() - t0
    u64, c64 = got["fp64"]
    um = got["mixed"][0]
    return {"crop": [n, n], "tiles": list(nt), "n_irls": n_irls, "phase": "host atan2f",
            "fp64_unw_bit_mismatches": int(np.sum(u64.view(np.int32) != want_u.view(np.int32))),
            "fp64_cycle_mismatches": int(np.sum(np.abs(u64.astype(np.float64) - want_u) > np.pi)),
            "fp64_conncomp_mismatches": int(np.sum(c64 != want_c)),
            "mixed_cycle_mismatches": int(np.sum(np.abs(um.astype(np.float64) - want_u) > np.pi)),
            "oracle_s": oracle_s, "oracle_threads": os.cpu_count()}


def _arc_div(ad, ar):
    """D^T of two arc planes: at each pixel, the arcs that end there minus
    the arcs that start there ((D u)_a = u(head) - u(tail))."""
    import torch
    out = torch.zeros_like(ad)
    out[1:, :] += ad[:-1, :]
    out[:-1, :] -= ad[:-1, :]
    out[:, 1:] += ar[:, :-1]
    out[:, :-1] -= ar[:, :-1]
    return out


def _irls_weights(u, g, w0, k):
    """Pass-k IRLS weights w0 / sqrt(e^2 + delta_k^2), e = D u - g, in FP64
    (the reweighting of cuphu_b200.autograd.irls_solve)."""
    import torch
    from cuphu_b200.autograd import _arc_diffs
    delta = max(0.01, 0.5 * 0.5 ** k)
    du = _arc_diffs(u)
    return tuple(torch.where(w > 0, w * torch.rsqrt((d - gg) ** 2 + delta * delta),
                             torch.zeros_like(w)) for w, d, gg in zip(w0, du, g))


def fd_difference_form(gd, gr, w0d, w0r, loss_of, n_irls, arcs, rng, grads, h=1e-3,
                       precision="fp64", max_iter=20000, tol=1e-6):
    """Central finite differences (L(theta + h) - L(theta - h)) / 2h of the
    IRLS map on single arcs of the full scene, each side computed as the
    exact change of every pass's solution rather than as two full solves
    whose loss values are subtracted: for the perturbed pass p,
        u'_p - u_p = L'_p^-1 (D^T (W'_p (g' - D u_p) - W_p (g - D u_p))),
    with W'_p the pass's weights recomputed from u'_{p-1} = u_{p-1} +
    (u'_{p-1} - u_{p-1}) and the perturbed inputs.  The identity holds for
    exact base solutions, so the change is solved to a relative tolerance
    without the cancellation of subtracting two large losses (which at
    2048^2 would need every full solve converged to ~1e-10, beyond reach of
    Jacobi-PCG).  The base solves and the adjoint use the same tolerance."""
    import torch
    from cuphu_b200.autograd import _arc_diffs, wls_solve
    kw = dict(precision=precision, max_iter=max_iter, tol=tol)
    g = (gd.double(), gr.double())
    w0 = (w0d.double(), w0r.double())
    us, Ws = [], [w0]
    u = wls_solve(gd, gr, w0d, w0r, **kw)
    us.append(u)
    for k in range(n_irls):
        W = _irls_weights(u, g, w0, k)
        u = wls_solve(gd, gr, W[0].float(), W[1].float(), u0=u, **kw)
        us.append(u)
        Ws.append(W)
    nrow, ncol = gd.shape
    errs, scaled = [], []
    for _ in range(arcs):
        leaf = int(rng.integers(0, 4))
        r = int(rng.integers(0, nrow - 1 if leaf in (0, 2) else nrow))
        q = int(rng.integers(0, ncol if leaf in (0, 2) else ncol - 1))
        base = float((gd, gr, w0d, w0r)[leaf][r, q])
        vals = []
        for sgn in (1.0, -1.0):
            gp = [t.clone() for t in g]
            w0p = [t.clone() for t in w0]
            (gp + w0p)[leaf][r, q] = float(np.float32(base + sgn * h))
            du = None
            for p in range(n_irls + 1):
                Wp = tuple(w0p) if p == 0 else _irls_weights(us[p - 1] + du, gp, w0p, p - 1)
                dd, dr = _arc_diffs(us[p])
                sd = Wp[0] * (gp[0] - dd) - Ws[p][0] * (g[0] - dd)
                sr = Wp[1] * (gp[1] - dr) - Ws[p][1] * (g[1] - dr)
                sd[-1, :] = 0.0
                sr[:, -1] = 0.0
                rhs = _arc_div(sd, sr)
                du = wls_solve(rhs=rhs.float(), wd=Wp[0].float(), wr=Wp[1].float(), **kw)
            vals.append(float(loss_of(us[-1] + du) - loss_of(us[-1])))
        hp = float(np.float32(base + h)) - float(np.float32(base - h))
        fd = (vals[0] - vals[1]) / hp
        gval = float(grads[leaf][r, q])
        errs.append(abs(fd - gval) / max(1e-30, abs(gval), abs(fd)))
        scaled.append(abs(fd - gval) / float(grads[leaf].abs().max()))
    return errs, scaled


def adjoint_c4(seed=0, fd_arcs=0, fd_tol=1e-6, fd_max_iter=20000):
    """The differentiable WLS/IRLS solve on the 2048^2 DEFO configuration
    (5 IRLS passes, loss = mean squared difference to the scene's true
    phase, both taken about their means): forward and backward device time
    of the mixed solver, and the mixed gradient against the FP64 adjoint's.
    Optionally central finite differences (step 1e-3) on seeded random arcs
    of the full 2048^2 scene (fd_difference_form), against the FP64 adjoint
    at the same solve tolerance."""
    import torch
    from cuphu_b200 import synthetic as S
    from cuphu_b200._lib import check, default_params, lib
    from cuphu_b200.autograd import irls_solve
    L = lib()
    ig, g, truth, ex = S.config_scene("c4_2048_defo", seed=seed)
    nrow, ncol = g.shape
    sptr = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    d_ig = torch.from_numpy(ig.view(np.float32)).cuda()
    d_g = torch.from_numpy(g).cuda()
    ph = torch.empty((nrow, ncol), dtype=torch.float32, device="cuda")
    check(L.cuphu_phase_gpu(C.c_void_p(d_ig.data_ptr()), C.c_longlong(nrow * ncol),
                            C.c_void_p(ph.data_ptr()), sptr))
    narcs = (nrow - 1) * ncol + nrow * (ncol - 1)
    cost = torch.empty((narcs, 4), dtype=torch.int16, device="cuda")
    pc = default_params(nlooks=float(ex["nlooks"]), ncorrlooks=float(ex["nlooks"]))
    check(L.cuphu_build_costs_device(C.c_void_p(ph.data_ptr()), C.c_void_p(d_g.data_ptr()), None,
                                     nrow, ncol, 1, C.byref(pc), C.c_void_p(cost.data_ptr()),
                                     None, sptr))
    sig = cost[:, 1].to(torch.float32)
    w = torch.where((sig > 0) & (sig < 32000), 1.0 / sig, torch.zeros_like(sig))
    nd = (nrow - 1) * ncol
    w0d = torch.zeros((nrow, ncol), device="cuda")
    w0r = torch.zeros((nrow, ncol), device="cuda")
    w0d[:-1, :] = w[:nd].view(nrow - 1, ncol)
    w0r[:, :-1] = w[nd:].view(nrow, ncol - 1)
    two_pi = 2 * np.pi
    gd = torch.zeros_like(w0d)
    gr = torch.zeros_like(w0r)
    dd = ph[1:, :] - ph[:-1, :]
    dr = ph[:, 1:] - ph[:, :-1]
    gd[:-1, :] = dd - two_pi * torch.round(dd / two_pi)
    gr[:, :-1] = dr - two_pi * torch.round(dr / two_pi)
    t = torch.from_numpy(np.asarray(truth, np.float64)).cuda()
    t = t - t.mean()

    def loss_of(u):
        return ((u - u.mean() - t) ** 2).mean()

    n_irls = int(ex["n_irls"])

    def run(prec, **kw):
        leaves = [x.clone().requires_grad_() for x in (gd, gr, w0d, w0r)]
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        e[0].record()
        u = irls_solve(*leaves, n_irls=n_irls, precision=prec, **kw)
        loss = loss_of(u)
        e[1].record()
        loss.backward()
        e[2].record()
        torch.cuda.synchronize()
        return ([x.grad.double() for x in leaves], e[0].elapsed_time(e[1]),
                e[1].elapsed_time(e[2]))

    run("mixed")                      # warm-up
    gm, fwd_ms, bwd_ms = run("mixed")
    g64, fwd64_ms, bwd64_ms = run("fp64")
    rel = max(float((a - b).abs().max() / b.abs().max()) for a, b in zip(gm, g64))
    out = {"config": "c4_2048_defo", "shape": [nrow, ncol], "n_irls": n_irls,
           "loss": "mean squared difference to the true phase",
           "forward_ms": fwd_ms, "backward_ms": bwd_ms, "fp64_forward_ms": fwd64_ms,
           "fp64_backward_ms": bwd64_ms, "grad_rel_diff_mixed_vs_fp64": rel}
    if fd_arcs:
        t0 = time.time()
        gt, _, _ = run("fp64", max_iter=fd_max_iter, tol=fd_tol)
        errs, scaled = fd_difference_form(gd, gr, w0d, w0r, loss_of, n_irls, fd_arcs,
                                          np.random.default_rng(seed + 2), gt,
                                          max_iter=fd_max_iter, tol=fd_tol)
        out["fd"] = {"arcs": fd_arcs, "shape": [nrow, ncol], "step": 1e-3, "tol": fd_tol,
                     "max_iter": fd_max_iter, "max_rel_err": float(max(errs)),
                     "median_rel_err": float(np.median(errs)),
                     "max_err_over_max_grad": float(max(scaled)), "s": time.time() - t0}
    return out


def _batch_core(data, reps, warm_each, sync_ranks=None):
    """The three ways of solving a list of scenes on this GPU: one
    cuphu_unwrap_device call per scene, one persistent batched launch
    (cuphu_unwrap_batch_device) and replays of its CUDA graph
    (cuphu_batch_graph_*).  Returns the device time (CUDA events) and wall
    time of each per repetition, and whether the outputs are identical."""
    import torch
    from cuphu_b200._lib import (CuPhuScene, check, default_params, default_solve_options,
                                 default_tile_params, lib)
    L = lib()
    p = default_params(nlooks=5.0, ncorrlooks=5.0)
    o = default_solve_options(precision=0, ref_row=0, ref_col=0)
    stream = torch.cuda.current_stream()
    sptr = C.c_void_p(stream.cuda_stream)
    bufs = []
    for ig, g, _ in data:
        nr, nc = g.shape
        bufs.append(dict(nr=nr, nc=nc, t=tiles_for(nr, nc),
                         ig=torch.from_numpy(ig.view(np.float32)).cuda(),
                         g=torch.from_numpy(g).cuda(),
                         u=torch.empty((nr, nc), dtype=torch.float32, device="cuda"),
                         c=torch.empty((nr, nc), dtype=torch.int32, device="cuda")))
    scenes = (CuPhuScene * len(bufs))()
    for i, b in enumerate(bufs):
        scenes[i] = CuPhuScene(b["ig"].data_ptr(), None, b["g"].data_ptr(), None, None, b["nr"],
                               b["nc"], b["t"][0], b["t"][1], 64, 64, 5.0, b["u"].data_ptr(),
                               b["c"].data_ptr())

    def individual():
        for b in bufs:
            tile = default_tile_params(ntilerow=b["t"][0], ntilecol=b["t"][1], rowovrlp=64,
                                       colovrlp=64)
            check(L.cuphu_unwrap_device(C.c_void_p(b["ig"].data_ptr()), None,
                                        C.c_void_p(b["g"].data_ptr()), None, None, b["nr"], b["nc"],
                                        1, C.byref(p), C.byref(tile), C.byref(o),
                                        C.c_void_p(b["u"].data_ptr()), C.c_void_p(b["c"].data_ptr()),
                                        None, None, sptr))

    def batched():
        check(L.cuphu_unwrap_batch_device(scenes, len(bufs), 1, C.byref(p), C.byref(o), None,
                                          sptr))

    def timed(fn):
        if warm_each:
            fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, (time.perf_counter() - t0) * 1e3 / reps

    def outputs():
        return [(b["u"].cpu().numpy().copy(), b["c"].cpu().numpy().copy()) for b in bufs]

    if not warm_each:
        batched()                       # sizes the workspace once for all three
    if sync_ranks:
        sync_ranks()
    ms_ind, wall_ind = timed(individual)
    out_ind = outputs()
    ms_bat, wall_bat = timed(batched)
    out_bat = outputs()
    graph = C.c_void_p()
    check(L.cuphu_batch_graph_create(scenes, len(bufs), 1, C.byref(p), C.byref(o),
                                     C.byref(graph)))
    try:
        ms_gr, wall_gr = timed(lambda: check(L.cuphu_batch_graph_launch(graph, sptr)))
        out_gr = outputs()
    finally:
        check(L.cuphu_batch_graph_destroy(graph))

    def same(a, b):
        return all(np.array_equal(x[0].view(np.int32), y[0].view(np.int32)) and
                   np.array_equal(x[1], y[1]) for x, y in zip(a, b))

    return {"individual": (ms_ind, wall_ind), "batched": (ms_bat, wall_bat),
            "graph": (ms_gr, wall_gr),
            "identical": {"batched_vs_individual": same(out_bat, out_ind),
                          "graph_vs_batched": same(out_gr, out_bat)},
            "n_irls": o.n_irls}


def batch_c3(seed=0):
    """The 48-interferogram configuration on this GPU, one repetition of each
    way of solving it (the key the default bench line carries)."""
    from cuphu_b200 import synthetic as S
    data = S.batch_scenes(48, seed=seed)
    total_px = sum(int(g.size) for _, g, _ in data)
    r = _batch_core(data, reps=1, warm_each=False)
    del data
    mp = total_px / 1e6
    return {"config": "c3_batch48", "scenes": 48, "pixels": total_px, "cost": "defo",
            "nlooks": 5.0, "n_irls": r["n_irls"], "precision": "mixed",
            "individual_calls": {"ms": r["individual"][0], "mpix_s": mp / (r["individual"][0] * 1e-3)},
            "batched_launch": {"ms": r["batched"][0], "mpix_s": mp / (r["batched"][0] * 1e-3)},
            "graph_replay": {"ms": r["graph"][0], "mpix_s": mp / (r["graph"][0] * 1e-3)},
            "speedup_batched_vs_individual": r["individual"][0] / r["batched"][0],
            "outputs_identical": r["identical"]}


def run_batch(args, rank, world, local_rank):
    """The 48-interferogram configuration (sides from {512, 1024, 2048,
    3072}, DEFO, nlooks 5, each scene auto-tiled): 48 individual
    cuphu_unwrap_device calls, one persistent batched launch
    (cuphu_unwrap_batch_device) and replays of its CUDA graph
    (cuphu_batch_graph_*), with the outputs of the three compared."""
    import torch
    from cuphu_b200 import synthetic as S
    from cuphu_b200.replicas import max_over_ranks, shard_scenes
    torch.cuda.set_device(local_rank)
    data = S.batch_scenes(48, seed=args.seed)
    total_px = sum(int(g.size) for _, g, _ in data)
    # N GPUs: the same 48 scenes, split by scene (no data-path collective)
    mine = shard_scenes([int(g.size) for _, g, _ in data], rank, world)
    data = [data[i] for i in mine]

    def sync():
        if world > 1:
            import torch.distributed as tdist
            tdist.barrier()

    clocks = ClockSampler(local_rank)
    clocks.start()
    nloc = len(data)
    r = _batch_core(data, reps=args.steps, warm_each=True, sync_ranks=sync)
    del data
    clk = clocks.stop()
    (ms_ind, wall_ind), (ms_bat, wall_bat), (ms_gr, wall_gr) = (r["individual"], r["batched"],
                                                                r["graph"])
    ms_ind, ms_bat, ms_gr = (max_over_ranks(x) for x in (ms_ind, ms_bat, ms_gr))
    same_flags = r["identical"]
    mp = total_px / 1e6
    line = {"metric": "Mpix/s unwrapped, 48-interferogram uneven batch (mixed-precision Laplace PCG)",
            "value": mp / (ms_gr * 1e-3), "unit": "Mpix/s", "n_gpus": world,
            "steps": args.steps, "warmup": 1, "ms_per_step": ms_gr, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "c3_batch48", "scenes": 48, "pixels": total_px,
                       "scenes_per_rank": nloc,
                       "cost": "defo", "nlooks": 5.0, "n_irls": r["n_irls"],
                       "tiles": "auto (target 1024, overlap 64)"},
            "individual_calls": {"ms": ms_ind, "wall_ms": wall_ind, "mpix_s": mp / (ms_ind * 1e-3)},
            "batched_launch": {"ms": ms_bat, "wall_ms": wall_bat, "mpix_s": mp / (ms_bat * 1e-3)},
            "graph_replay": {"ms": ms_gr, "wall_ms": wall_gr, "mpix_s": mp / (ms_gr * 1e-3)},
            "outputs_identical": same_flags,
            "clocks": clk}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    ig, g, ex = make_scene(args.workload, args.seed)
    mode = {"smooth": 0, "defo": 1, "topo": 2}[ex["cost"]]
    n_irls = ex.get("n_irls", 16)
    vals = []
    for i in range(args.warmup + args.steps):
        v, dt, iters, n = cpu_baseline(ig, g, ex["nlooks"], mode, n_irls)
        if i >= args.warmup:
            vals.append((v, dt))
    v = float(np.mean([x[0] for x in vals]))
    ms = float(np.mean([x[1] for x in vals])) * 1e3
    cores = os.cpu_count()
    nrow, ncol = g.shape
    ntr, ntc = tiles_for(nrow, ncol)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpix/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "shape": [nrow, ncol], "tiles": [ntr, ntc],
                       "overlap": 64, "n_irls": n_irls, "max_iter": 1000, "tol": 1e-3,
                       "precision": "fp64", "parallelism": f"cpu{cores}",
                       "sample": f"{n}x{n} crop, full pipeline"},
            "cpu_baseline": {"value": v, "unit": "Mpix/s", "cores": cores, "kind": "port",
                             "sample": f"{n}x{n} crop of the {args.workload} scene: cost build "
                                       f"+ FP64 Jacobi-PCG ({n_irls} IRLS passes) + conncomp, "
                                       f"OpenMP on {cores} threads"},
            "e2e": {"value": v, "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    from cuphu_b200.replicas import max_over_ranks
    from cuphu_b200._lib import (CuPhuSolveStats, check, default_params, default_solve_options,
                                 default_tile_params, lib)
    torch.cuda.set_device(local_rank)
    L = lib()
    ig, g, ex = make_scene(args.workload, args.seed, args.scale)
    nrow, ncol = g.shape
    npix = nrow * ncol
    mode = {"smooth": 0, "defo": 1, "topo": 2}[ex["cost"]]
    nlooks = float(ex["nlooks"])
    ntr, ntc = tiles_for(nrow, ncol)
    params = default_params(nlooks=nlooks, ncorrlooks=nlooks)
    tile = default_tile_params(ntilerow=ntr, ntilecol=ntc, rowovrlp=64, colovrlp=64)
    prec = {"mixed": 0, "fp64": 1}[args.precision]
    opts = default_solve_options(precision=prec, ref_row=0, ref_col=0)
    if "n_irls" in ex:
        opts.n_irls = int(ex["n_irls"])

    tuned = None
    if not (args.profile or args.cost_only or args.no_autotune):
        import cuphu_b200
        tuned = cuphu_b200.autotune(ig, g, nlooks, cost=ex["cost"], ntiles=(ntr, ntc),
                                    tile_overlap=(64, 64), gpu_id=local_rank)
    d_ig = torch.from_numpy(ig.view(np.float32)).cuda()
    d_g = torch.from_numpy(g).cuda()
    d_u = torch.empty((nrow, ncol), dtype=torch.float32, device="cuda")
    d_c = torch.empty((nrow, ncol), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    sptr = C.c_void_p(stream.cuda_stream)

    def step(o, stats=None):
        check(L.cuphu_unwrap_device(C.c_void_p(d_ig.data_ptr()), None, C.c_void_p(d_g.data_ptr()),
                                    None, None, nrow, ncol, mode, C.byref(params),
                                    C.byref(tile), C.byref(o), C.c_void_p(d_u.data_ptr()),
                                    C.c_void_p(d_c.data_ptr()), None,
                                    C.byref(stats) if stats is not None else None, sptr))

    dist = world > 1
    if dist:
        import torch.distributed as tdist
    st = CuPhuSolveStats()
    if args.cost_only:
        # one DEFO cost build from the wrapped phase (for ncu captures)
        d_ph = torch.empty((nrow, ncol), dtype=torch.float32, device="cuda")
        check(L.cuphu_phase_gpu(C.c_void_p(d_ig.data_ptr()), C.c_longlong(npix),
                                C.c_void_p(d_ph.data_ptr()), sptr))
        narcs = (nrow - 1) * ncol + nrow * (ncol - 1)
        d_cost = torch.empty((narcs, 4), dtype=torch.int16, device="cuda")
        pc = default_params(nlooks=nlooks, ncorrlooks=nlooks)
        check(L.cuphu_build_costs_device(C.c_void_p(d_ph.data_ptr()), C.c_void_p(d_g.data_ptr()),
                                         None, nrow, ncol, 1, C.byref(pc),
                                         C.c_void_p(d_cost.data_ptr()), None, sptr))
        torch.cuda.synchronize()
        print(json.dumps({"cost_case": args.workload, "shape": [nrow, ncol]}), flush=True)
        return
    if args.profile:
        # one warm-up and one device step, nothing else (for ncu captures)
        for _ in range(args.warmup + 1):
            step(opts, st)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": args.workload, "solve_ms": st.solve_ms,
                          "total_ms": st.total_ms, "pcg_iterations": st.total_iters,
                          "px_iterations": st.px_iters, "ntiles": st.ntiles}), flush=True)
        return
    for _ in range(args.warmup):
        step(opts, st)
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step(opts)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        tdist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()
    ms = max_over_ranks(ms)
    value = world * npix / (ms * 1e-3) / 1e6

    # solver statistics of one more run (stats make the call synchronous)
    st = CuPhuSolveStats()
    step(opts, st)
    unw_mixed = d_u.cpu().numpy()

    # roofline of the dominant kernel (the persistent solve): algorithmic
    # bytes = tile pixels x (36 B per PCG iteration x iterations of the
    # active tiles + 38 B per IRLS pass for assemble and reweight + 12 B per
    # true-residual replacement, one SpMV read of x and the weights)
    peak, peak_kind = hbm_peak()
    # tile extents of the reference's tile geometry (cuphu_solver.cpp:1753-1791)
    tr_f = [(int(t * (nrow - 64) / ntr), (nrow if t == ntr - 1 else int((t + 1) * (nrow - 64) / ntr) + 64)) for t in range(ntr)]
    tc_f = [(int(t * (ncol - 64) / ntc), (ncol if t == ntc - 1 else int((t + 1) * (ncol - 64) / ntc) + 64)) for t in range(ntc)]
    tile_px = sum((b - a) for a, b in tr_f) * sum((b - a) for a, b in tc_f)
    px_iters = st.px_iters                # iterations x pixels of the active tiles
    bpi = 36 if prec == 0 else 64
    # pixels of the replacements: every tile replaces its residual once per
    # replace_every of its iterations (mixed precision only)
    repl_px = px_iters / opts.replace_every if prec == 0 and opts.replace_every > 0 else 0.0
    alg_bytes = px_iters * bpi + (opts.n_irls + 1) * tile_px * 38 + repl_px * 12
    achieved = alg_bytes / (st.solve_ms * 1e-3) / 1e9
    # DRAM traffic per launch, scaled from ncu captures of the 4096^2 case
    # (dram__bytes_read.sum + dram__bytes_write.sum at 20, 40 and 60
    # iterations): the marginal bytes per active-tile pixel-iteration, the
    # fixed bytes per tile pixel of each IRLS pass (assemble/INIT and final)
    # and the bytes per pixel of a true-residual replacement
    traffic = (px_iters * TRAFFIC_PER_PX_ITER + (opts.n_irls + 1) * tile_px * TRAFFIC_PER_PASS_PX
               + repl_px * TRAFFIC_PER_REPL_PX if prec == 0 else None)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "kernel": "k_solve", "solve_ms": st.solve_ms, "pcg_iterations": st.total_iters,
                "px_iterations": st.px_iters, "tile_px": tile_px,
                "bytes_per_px_iter": bpi}

    result = {}
    if rank == 0 and not args.skip_fp64 and prec == 0:
        o64 = default_solve_options(precision=1, ref_row=0, ref_col=0)
        o64.n_irls = opts.n_irls
        st64 = CuPhuSolveStats()
        step(o64, st64)
        torch.cuda.synchronize()
        ee0 = torch.cuda.Event(enable_timing=True)
        ee1 = torch.cuda.Event(enable_timing=True)
        ee0.record(stream)
        step(o64)
        ee1.record(stream)
        torch.cuda.synchronize()
        ms64 = ee0.elapsed_time(ee1)
        unw64 = d_u.cpu().numpy()
        diff = unw_mixed.astype(np.float64) - unw64
        flip = np.abs(diff) > np.pi
        flips = [tuple(x) for x in np.argwhere(flip)]
        d_ph = torch.empty((nrow, ncol), dtype=torch.float32, device="cuda")
        check(L.cuphu_phase_gpu(C.c_void_p(d_ig.data_ptr()), C.c_longlong(npix),
                                C.c_void_p(d_ph.data_ptr()), sptr))
        ph_dev = d_ph.cpu().numpy()
        del d_ph
        result["fp64"] = {"value": npix / (ms64 * 1e-3) / 1e6, "ms_per_step": ms64,
                          "speedup_mixed_vs_fp64": ms64 / ms,
                          "cycle_mismatches": int(flip.sum()),
                          "rms_rad": float(np.sqrt(np.mean(diff ** 2))),
                          "rms_rad_outside_flips": float(np.sqrt(np.mean(diff[~flip] ** 2))),
                          "max_abs_rad_outside_flips": float(np.abs(diff[~flip]).max()),
                          "pcg_iterations": st64.total_iters,
                          "mixed_pcg_iterations": st.total_iters,
                          "flips": flip_details(ph_dev, g, nlooks, mode, flips, (ntr, ntc), 64,
                                                opts.n_irls)}

    # cost-kernel bandwidth (DEFO costs from the wrapped phase, 8192^2)
    if rank == 0:
        d_ph = torch.empty((nrow, ncol), dtype=torch.float32, device="cuda")
        check(L.cuphu_phase_gpu(C.c_void_p(d_ig.data_ptr()), C.c_longlong(npix),
                                C.c_void_p(d_ph.data_ptr()), sptr))
        narcs = (nrow - 1) * ncol + nrow * (ncol - 1)
        d_cost = torch.empty((narcs, 4), dtype=torch.int16, device="cuda")
        pc = default_params(nlooks=nlooks, ncorrlooks=nlooks)
        for _ in range(3):
            check(L.cuphu_build_costs_device(C.c_void_p(d_ph.data_ptr()), C.c_void_p(d_g.data_ptr()),
                                             None, nrow, ncol, 1, C.byref(pc),
                                             C.c_void_p(d_cost.data_ptr()), None, sptr))
        ce0 = torch.cuda.Event(enable_timing=True)
        ce1 = torch.cuda.Event(enable_timing=True)
        reps = 10
        ce0.record(stream)
        for _ in range(reps):
            check(L.cuphu_build_costs_device(C.c_void_p(d_ph.data_ptr()), C.c_void_p(d_g.data_ptr()),
                                             None, nrow, ncol, 1, C.byref(pc),
                                             C.c_void_p(d_cost.data_ptr()), None, sptr))
        ce1.record(stream)
        torch.cuda.synchronize()
        cms = ce0.elapsed_time(ce1) / reps
        cbytes = npix * 4 + npix * 4 + narcs * 8
        result["cost_build"] = {"kernel": "k_costs7<DEFO>", "ms": cms,
                                "gbs": cbytes / (cms * 1e-3) / 1e9,
                                "frac": cbytes / (cms * 1e-3) / 1e9 / peak,
                                "bytes_per_px": cbytes / npix}
        del d_cost, d_ph

    if rank == 0 and not args.skip_adjoint:
        result["adjoint"] = adjoint_c4(args.seed, args.adjoint_fd, args.adjoint_fd_tol,
                                       args.adjoint_fd_iters)

    if rank == 0 and not args.skip_parity:
        result["parity"] = parity_crop(ig, g, nlooks, mode, n_irls=opts.n_irls)

    if rank == 0 and not args.skip_batch:
        result["batch"] = batch_c3(args.seed)

    # end to end through the C ABI with pinned host buffers
    h_ig = torch.from_numpy(ig.view(np.float32)).pin_memory()
    h_g = torch.from_numpy(g).pin_memory()
    h_u = torch.empty((nrow, ncol), dtype=torch.float32).pin_memory()
    h_c = torch.empty((nrow, ncol), dtype=torch.int32).pin_memory()

    def e2e_step():
        check(L.cuphu_unwrap_ex(C.c_void_p(h_ig.data_ptr()), C.c_void_p(h_g.data_ptr()), None,
                                None, nrow, ncol, mode, C.byref(params), C.byref(tile),
                                C.byref(opts), local_rank, C.c_void_p(h_u.data_ptr()),
                                C.c_void_p(h_c.data_ptr()), None))

    e2e_step()
    if dist:
        tdist.barrier()
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps)):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / max(1, args.steps)
    e2e_s = max_over_ranks(e2e_s)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        v, dt, iters, n = cpu_baseline(ig, g, nlooks, mode, opts.n_irls)
        cpu = {"value": v, "unit": "Mpix/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"{n}x{n} crop of the scene: cost build + FP64 Jacobi-PCG "
                         f"({opts.n_irls} IRLS passes, {iters} iterations) + conncomp, "
                         f"{dt:.1f} s"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if prec == 0 else "f64", "data": "synthetic",
                "config": {"workload": args.workload, "shape": [nrow, ncol],
                           "tiles": [ntr, ntc], "overlap": 64, "n_irls": opts.n_irls,
                           "max_iter": opts.max_iter, "tol": opts.tol,
                           "precision": args.precision, "parallelism": f"replicas{world}",
                           "l2": "inputs (805 MB) larger than L2", "autotune": tuned},
                "e2e": {"value": world * npix / e2e_s / 1e6, "unit": "Mpix/s",
                        "h2d_bytes_per_step": npix * 8, "d2h_bytes_per_step": npix * 8,
                        "phase": "host atan2f (the reference's), threaded and overlapped "
                                 "with its upload"},
                "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
                "gpu_launches": 14 * args.steps}
        line.update(result)
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2_8192_topo")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-adjoint", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--skip-parity", action="store_true",
                    help="skip the FP64-vs-oracle parity check on a 3x3-tile crop")
    ap.add_argument("--skip-batch", action="store_true",
                    help="skip the 48-interferogram batch measurement")
    ap.add_argument("--adjoint-fd", type=int, default=0,
                    help="finite-difference check of the adjoint on this many random arcs")
    ap.add_argument("--adjoint-fd-tol", type=float, default=1e-6,
                    help="relative solve tolerance of the finite-difference check")
    ap.add_argument("--adjoint-fd-iters", type=int, default=20000,
                    help="PCG iteration cap of the finite-difference check")
    ap.add_argument("--scale", type=int, default=None,
                    help="edge length override of the workload (small profiling cases)")
    ap.add_argument("--cost-only", action="store_true",
                    help="one DEFO cost build only (for ncu captures)")
    ap.add_argument("--profile", action="store_true",
                    help="warm-up + one device step only (for ncu captures)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.workload == "c3_batch48":
            run_batch(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as tdist
            tdist.destroy_process_group()


if __name__ == "__main__":
    main()
