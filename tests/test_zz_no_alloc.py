"""cuphu_integrate_phase_noalloc (the integration entry point that allocates
no device memory) against cuphu_integrate_phase_gpu, through the C ABI.

Collected last so it also runs after every other test has used the device;
one test runs the entry point as the first and only library call of a fresh
process.  Integration is compared bit for bit, the tolerance every
integration test here uses.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from cuphu_b200._lib import CuPhuError, check, lib
from tests.devbuf import dptr, empty, to_dev, to_host

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

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


def _pool_state():
    """(used, reserved) bytes of the device's default memory pool and the
    device's free memory, through the CUDA runtime torch has loaded; the
    pool's used high-water mark is reset to its current value first."""
    rt = C.CDLL("libcudart.so.12")
    dev = C.c_int()
    assert rt.cudaGetDevice(C.byref(dev)) == 0
    pool = C.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(C.byref(pool), dev) == 0
    used, reserved, high = C.c_uint64(), C.c_uint64(), C.c_uint64()
    free_b, total_b = C.c_size_t(), C.c_size_t()
    # cudaMemPoolAttrReservedMemCurrent = 5, UsedMemCurrent = 7, UsedMemHigh = 8
    assert rt.cudaMemPoolGetAttribute(pool, 7, C.byref(used)) == 0
    assert rt.cudaMemPoolGetAttribute(pool, 5, C.byref(reserved)) == 0
    assert rt.cudaMemPoolGetAttribute(pool, 8, C.byref(high)) == 0
    assert rt.cudaMemGetInfo(C.byref(free_b), C.byref(total_b)) == 0
    return rt, pool, used.value, reserved.value, high.value, free_b.value


def test_noalloc_call_allocates_nothing(torch_cuda):
    """A warm call moves neither the default pool's used or reserved bytes
    nor its used high-water mark (a transient stream-ordered allocation would
    raise it), nor torch's allocator, nor the device's free memory."""
    ph, hf, vf = _inputs(700, 300, 5)
    nr, nc = ph.shape
    dph, dh, dv = to_dev(ph), to_dev(hf), to_dev(vf)
    du = empty((nr, nc), torch_cuda.float32)
    stream = C.c_void_p(torch_cuda.cuda.current_stream().cuda_stream)
    args = (dptr(dph), dptr(dh), dptr(dv), nr, nc, dptr(du), stream)
    check(lib().cuphu_integrate_phase_noalloc(*args))          # warm: symbol looked up
    torch_cuda.cuda.synchronize()
    rt, pool, used0, res0, _, free0 = _pool_state()
    zero = C.c_uint64(0)
    # the high-water mark can only be reset to zero; any allocation from the
    # pool after that raises it to at least the pool's usage at that moment
    assert rt.cudaMemPoolSetAttribute(pool, 8, C.byref(zero)) == 0
    torch0 = torch_cuda.cuda.memory_allocated()
    for _ in range(2):
        check(lib().cuphu_integrate_phase_noalloc(*args))
    torch_cuda.cuda.synchronize()
    _, _, used1, res1, high1, free1 = _pool_state()
    assert (used1, res1) == (used0, res0)
    assert high1 <= used0
    assert torch_cuda.cuda.memory_allocated() == torch0
    assert free1 == free0


_FRESH = r"""
import ctypes as C, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import oracle as O
from cuphu_b200._lib import check, lib
rng = np.random.default_rng(7)
nr, nc = 513, 257
ph = rng.uniform(0.0, 2 * np.pi, (nr, nc)).astype(np.float32)
hf = rng.integers(-3, 4, (nr - 1, nc)).astype(np.int16)
vf = rng.integers(-3, 4, (nr, nc - 1)).astype(np.int16)
d = [torch.from_numpy(a).cuda() for a in (ph, hf, vf)]
du = torch.empty((nr, nc), dtype=torch.float32, device="cuda")
check(lib().cuphu_integrate_phase_noalloc(*[C.c_void_p(t.data_ptr()) for t in d], nr, nc,
                                          C.c_void_p(du.data_ptr()), None))
torch.cuda.synchronize()
want = O.integrate_phase(ph, hf, vf)
got = du.cpu().numpy()
print("match", bool(np.array_equal(got.view(np.int32), want.view(np.int32))))
"""


def test_noalloc_first_call_in_a_fresh_process(torch_cuda):
    """The symbol lookup of the entry point's first call on a device, in a
    process where nothing else of the library has run, against the oracle's
    integration."""
    r = subprocess.run([sys.executable, "-c", _FRESH, ROOT], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "match True" in r.stdout, r.stdout + r.stderr[-2000:]
