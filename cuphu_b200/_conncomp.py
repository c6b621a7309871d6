"""Connected-component relabelling of an unwrapped phase.

``regrow_conncomp`` keeps the reference signature and semantics
(cuphu/_conncomp.py:12-119: valid = corr >= cost_thresh and mask != 0; 4-
neighbours join when |unw_a - unw_b| < pi; components of at least
max(1, int(min_conncomp_frac * npix)) pixels get labels 1..max_ncomps in
order of their smallest pixel index) but runs the GPU union-find of
libcuphu_b200 instead of scipy on the host.
"""
from __future__ import annotations

import numpy as np

from cuphu_b200._lib import check, lib, ptr

__all__ = ["regrow_conncomp"]


def regrow_conncomp(unw, corr, *, mask=None, cost_thresh=0.1, min_conncomp_frac=0.01,
                    max_ncomps=32, gpu_id=0):
    unw = np.ascontiguousarray(unw, dtype=np.float32)
    corr = np.ascontiguousarray(corr, dtype=np.float32)
    nrow, ncol = unw.shape
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    labels = np.zeros((nrow, ncol), dtype=np.uint32)
    check(lib().cuphu_conncomp_ex(ptr(unw), ptr(corr), ptr(m), nrow, ncol, float(cost_thresh),
                                  float(min_conncomp_frac), int(max_ncomps), int(gpu_id),
                                  ptr(labels)))
    return labels
