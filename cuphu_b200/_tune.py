"""Launch-shape autotuner (cuphu_autotune): picks, per device and job size,
the cost kernel's occupancy variant and the persistent solver's launch shape
(stages of each block's shared-memory ring x resident blocks per SM) by
timing the candidates on a representative scene."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, default_params, default_tile_params, lib, ptr

_COST = {"smooth": 0, "defo": 1, "topo": 2}
# the mixed-precision solver's launch shapes, in the library's index order
_SOLVE_SHAPES = ((3, 2), (2, 2), (6, 1))


def autotune(igram, corr, nlooks, cost="smooth", ntiles=(1, 1), tile_overlap=(0, 0), gpu_id=0):
    """Tune on this scene; the choices apply to later calls of similar size
    (same floor(log2) of the arc / work-item count) on this GPU.  Returns
    {"cost_blocks_per_sm": 3 | 4, "solver_stages": S, "solver_blocks_per_sm": B}
    for the mixed-precision solver's chosen shape."""
    ig = np.ascontiguousarray(igram, dtype=np.complex64)
    g = np.ascontiguousarray(corr, dtype=np.float32)
    nrow, ncol = g.shape
    if ig.shape != g.shape:
        raise ValueError("igram and corr must have the same shape")
    p = default_params(nlooks=float(nlooks), ncorrlooks=float(nlooks))
    t = default_tile_params(ntilerow=int(ntiles[0]), ntilecol=int(ntiles[1]),
                            rowovrlp=int(tile_overlap[0]), colovrlp=int(tile_overlap[1]))
    out = (C.c_int * 2)()
    check(lib().cuphu_autotune(ptr(ig.view(np.float32)), ptr(g), nrow, ncol, _COST[cost],
                               C.byref(p), C.byref(t), int(gpu_id), out))
    stages, blocks = _SOLVE_SHAPES[out[1]]
    return {"cost_blocks_per_sm": 3 + out[0], "solver_stages": stages,
            "solver_blocks_per_sm": blocks}
