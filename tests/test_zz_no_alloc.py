"""cuphu_integrate_phase_noalloc (the integration entry point that allocates
no device memory) against cuphu_integrate_phase_gpu, through the C ABI.

Collected last so it also runs after every other test has used the device;
it must pass in a fresh process too.  Integration is compared bit for bit,
the tolerance every integration test here uses.
"""
import ctypes as C

import numpy as np
import pytest

from cuphu_b200._lib import CuPhuError, check, lib
from tests.devbuf import dptr, empty, to_dev, to_host

pytestmark = pytest.mark.gpu

MAX_ROWS = 65536  # CUPHU_NOALLOC_MAX_ROWS


def _inputs(nr, nc, seed):
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0.0, 2 * np.pi, (nr, nc)).astype(np.float32)
    hf = rng.integers(-3, 4, (max(nr - 1, 1), nc)).astype(np.int16)
    vf = rng.integers(-3, 4, (nr, max(nc - 1, 1))).astype(np.int16)
    return ph, hf, vf


def _allocating(torch, ph, hf, vf):
    nr, nc = ph.shape
    dph, dh, dv = to_dev(ph), to_dev(hf), to_dev(vf)
    du = empty((nr, nc), torch.float32)
    check(lib().cuphu_integrate_phase_gpu(dptr(dph), dptr(dh), dptr(dv), nr, nc,
                                          torch.cuda.current_device(), dptr(du)))
    return to_host(du)


def _noalloc(torch, ph, hf, vf):
    nr, nc = ph.shape
    dph, dh, dv = to_dev(ph), to_dev(hf), to_dev(vf)
    du = empty((nr, nc), torch.float32)
    du.fill_(float("nan"))
    stream = torch.cuda.current_stream().cuda_stream
    check(lib().cuphu_integrate_phase_noalloc(dptr(dph), dptr(dh), dptr(dv), nr, nc, dptr(du),
                                              C.c_void_p(stream)))
    return to_host(du)


def test_noalloc_matches_allocating_entry_point_on_two_calls(torch_cuda):
    # the second call is smaller than the first, so it runs over the scratch
    # rows the first call left behind
    for shape, seed in (((1031, 517), 1), ((300, 129), 2)):
        ph, hf, vf = _inputs(*shape, seed)
        want = _allocating(torch_cuda, ph, hf, vf)
        got = _noalloc(torch_cuda, ph, hf, vf)
        assert np.isfinite(got).all()
        assert np.array_equal(got.view(np.int32), want.view(np.int32))


def test_noalloc_handles_limit_and_rejects_beyond(torch_cuda):
    ph, hf, vf = _inputs(MAX_ROWS, 2, 3)
    want = _allocating(torch_cuda, ph, hf, vf)
    got = _noalloc(torch_cuda, ph, hf, vf)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))

    nr = MAX_ROWS + 1
    ph, hf, vf = _inputs(nr, 1, 4)
    dph, dh, dv = to_dev(ph), to_dev(hf), to_dev(vf)
    du = empty((nr, 1), torch_cuda.float32)
    with pytest.raises(CuPhuError, match="exceeds the no-allocation limit of 65536 rows"):
        check(lib().cuphu_integrate_phase_noalloc(dptr(dph), dptr(dh), dptr(dv), nr, 1,
                                                  dptr(du), None))
