"""Bounded device waits: a solver block that never arrives at a grid barrier
(cuphu_test_skip_barrier_once) makes every other block's wait run out after
the configured limit; the kernel returns, the call reports CUPHU_ERR_TIMEOUT,
and the next call on the same device runs normally.  The failure is made on
the host side of the barrier protocol: no fault, trap or unbounded wait."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from cuphu_b200 import synthetic as S
from cuphu_b200._lib import (CuPhuError, CuPhuSolveStats, check, default_params,
                             default_solve_options, default_tile_params, lib)
from tests.devbuf import dptr, empty, to_dev, to_host

pytestmark = pytest.mark.gpu

TIMEOUT = -5


def _run(torch, ph, g, precision, timeout_ms, stats):
    nr, nc = ph.shape
    dph, dg = to_dev(ph), to_dev(g)
    du = empty((nr, nc), torch.float32)
    dc = empty((nr, nc), torch.int32)
    p = default_params(nlooks=5.0, ncorrlooks=5.0)
    t = default_tile_params(ntilerow=2, ntilecol=2, rowovrlp=12, colovrlp=12)
    o = default_solve_options(precision=precision, n_irls=2, timeout_ms=timeout_ms)
    st = CuPhuSolveStats()
    rc = lib().cuphu_unwrap_device(None, dptr(dph), dptr(dg), None, None, nr, nc, 0, C.byref(p),
                                   C.byref(t), C.byref(o), dptr(du), dptr(dc), None,
                                   C.byref(st) if stats else None, None)
    torch.cuda.synchronize()
    return rc, to_host(du)


@pytest.mark.parametrize("precision", [0, 1])
def test_skipped_barrier_times_out_and_device_recovers(torch_cuda, precision):
    ig, g, _, _ = S.bumps(120, 140, seed=51, nbumps=2)
    ph = O.phase_from_igram(ig)
    rc0, want = _run(torch_cuda, ph, g, precision, 5000, stats=True)
    check(rc0)
    # asynchronous call: enqueue succeeds, the device status carries the timeout
    check(lib().cuphu_test_skip_barrier_once(0, 0))
    rc, _ = _run(torch_cuda, ph, g, precision, 20, stats=False)
    assert rc == 0
    assert lib().cuphu_last_status(0) == TIMEOUT
    # a call that waits for its statistics returns the timeout itself
    check(lib().cuphu_test_skip_barrier_once(0, 1))
    rc, _ = _run(torch_cuda, ph, g, precision, 20, stats=True)
    assert rc == TIMEOUT
    with pytest.raises(CuPhuError):
        check(rc)
    # the switch is one-shot: the next call is normal and bit-identical
    rc, got = _run(torch_cuda, ph, g, precision, 5000, stats=True)
    check(rc)
    assert lib().cuphu_last_status(0) == 0
    assert np.array_equal(got.view(np.int32), want.view(np.int32))
