"""Generate the golden fixtures that pin the CPU oracle to the reference.

Runs the reference cuPHU kernels (oracle/_ref/libcuphu_ref.so, compiled for
sm_100a from the reference sources by oracle/build.py) on small seeded
inputs and stores inputs and outputs as .npz files in this directory:

  costs_*.npz     cuphu_build_smooth/defo_costs_gpu (cuphu_cost.cu:339-479)
  conncomp_*.npz  cuphu_conncomp_gpu (cuphu_conncomp.cu:290-428)
  integrate.npz   cuphu_integrate_phase_gpu (cuphu_phase.cu:110-144)
  incrcost.npz    cuphu_incrcost_early_exit (cuphu_incrcost.cu:157-191)

The wrapped phase of every case is the host atan2f phase of the reference
(cuphu_solver.cpp:1706-1712), computed by the oracle.  Needs a CUDA GPU.

    python tests/golden/make_golden.py [outdir]
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from cuphu_b200 import synthetic as S  # noqa: E402


def scene(nr, nc, seed, nlooks=5.0):
    ig, g, t, _ = S.bumps(nr, nc, seed=seed, nbumps=3, amp_range=(5.0, 20.0),
                          sigma_range=(8.0, 20.0), nlooks=nlooks)
    return O.phase_from_igram(ig), g


def main(out):
    os.makedirs(out, exist_ok=True)
    if O.ref_lib() is None:
        raise SystemExit("oracle/_ref/libcuphu_ref.so is not built")
    cases = [(48, 64, 1, 5.0), (33, 70, 2, 9.0), (70, 41, 3, 20.0), (16, 16, 4, 1.5)]
    for nr, nc, seed, L in cases:
        ph, g = scene(nr, nc, seed, L)
        g = g.copy()
        g[: nr // 4, : nc // 3] *= 0.1          # a decorrelated patch
        rng = np.random.default_rng(seed)
        narcs = (nr - 1) * nc + nr * (nc - 1)
        w = (rng.random(narcs) > 0.1).astype(np.int16)
        for mode in (0, 1):
            for wname, wv in (("now", None), ("w", w)):
                c, _ = O.ref_build_costs(ph, g, L, mode=mode, weights=wv)
                np.savez_compressed(os.path.join(out, f"costs_m{mode}_{wname}_{nr}x{nc}.npz"),
                                    phase=ph, corr=g, nlooks=L, mode=mode,
                                    weights=wv if wv is not None else np.zeros(0, np.int16),
                                    costs=c)
    # conncomp: smooth field with a fringe break and a masked strip
    nr, nc = 40, 56
    rng = np.random.default_rng(7)
    unw = (0.1 * np.arange(nc)[None, :] + 0.05 * np.arange(nr)[:, None]).astype(np.float32)
    unw[:, 30:] += 9.0
    unw[15, 10] += 40.0
    corr = rng.uniform(0.0, 1.0, (nr, nc)).astype(np.float32)
    corr[corr < 0.1] = 0.02
    mask = np.ones((nr, nc), np.uint8)
    mask[:, 20:22] = 0
    narcs = (nr - 1) * nc + nr * (nc - 1)
    pos = rng.integers(-50, 600, narcs).astype(np.int16)
    neg = rng.integers(-50, 600, narcs).astype(np.int16)
    for name, kw in (("plain", {}), ("mask", dict(mask=mask)),
                     ("incr", dict(poscost=pos, negcost=neg)),
                     ("frac0", dict(minfrac=0.0, maxncomps=5))):
        lab = O.ref_conncomp(unw, corr, **kw)
        np.savez_compressed(os.path.join(out, f"conncomp_{name}.npz"), unw=unw, corr=corr,
                            mask=mask if "mask" in kw else np.zeros(0, np.uint8),
                            poscost=pos if "poscost" in kw else np.zeros(0, np.int16),
                            negcost=neg if "negcost" in kw else np.zeros(0, np.int16),
                            minfrac=kw.get("minfrac", 0.01), maxncomps=kw.get("maxncomps", 32),
                            labels=lab)
    # integration of random cycle counts
    ph, _ = scene(37, 45, 11)
    rng = np.random.default_rng(11)
    hf = rng.integers(-2, 3, (36, 45)).astype(np.int16)
    vf = rng.integers(-2, 3, (37, 44)).astype(np.int16)
    unw = O.ref_integrate(ph, hf, vf)
    np.savez_compressed(os.path.join(out, "integrate.npz"), phase=ph, hflows=hf, vflows=vf,
                        unw=unw)
    # incremental costs on smooth costs of a scene
    ph, g = scene(30, 38, 12)
    c, _ = O.ref_build_costs(ph, g, 5.0, mode=0)
    flows = np.random.default_rng(12).integers(-3, 4, c.shape[0]).astype(np.int16)
    p, n, ex = O.ref_incrcost(c, flows)
    np.savez_compressed(os.path.join(out, "incrcost.npz"), costs=c, flows=flows, pos=p, neg=n,
                        early_exit=ex)
    print("golden fixtures written to", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
