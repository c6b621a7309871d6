"""Band-by-band input (cuphu_stream_*): a scene held in a dataset that is read
by row slices streams to the GPU without being read whole, and gives the
same output, bit for bit, as the same scene passed as arrays."""
import ctypes as C

import numpy as np
import pytest

import cuphu_b200
from cuphu_b200 import _unwrap as U
from cuphu_b200 import synthetic as S
from cuphu_b200._lib import CuPhuError, check, lib

pytestmark = pytest.mark.gpu


class RowDataset:
    """A read-only dataset in the manner of h5py: shape, ndim, dtype, row
    slicing; reading it whole through __array__ is counted."""

    def __init__(self, a):
        self._a = a
        self.shape, self.ndim, self.dtype = a.shape, a.ndim, a.dtype
        self.whole_reads = 0
        self.slices = 0

    def __getitem__(self, key):
        self.slices += 1
        return self._a[key]

    def __array__(self, dtype=None, copy=None):
        self.whole_reads += 1
        return np.asarray(self._a, dtype=dtype)


@pytest.mark.parametrize("shape,tiles,band", [((300, 260), (2, 2), 37), ((130, 517), None, 64)])
def test_streamed_equals_arrays(torch_cuda, monkeypatch, shape, tiles, band):
    ig, g, _, _ = S.bumps(*shape, seed=41, nbumps=3, amp_range=(8, 25), sigma_range=(10, 40))
    ig = ig.copy()
    ig[3, 4] = np.nan
    mask = np.ones(shape, np.uint8)
    mask[50:60, 30:200] = 0
    kw = dict(init="laplace", mask=mask, mask_pad_distance=1, reference_pixel=(7, 9), n_irls=3)
    if tiles:
        kw.update(ntiles=tiles, tile_overlap=20)
    want_u, want_c = cuphu_b200.unwrap(ig, g, 5.0, **kw)
    monkeypatch.setattr(U, "_BAND_BYTES", band * shape[1] * 8)   # several bands
    dig, dg = RowDataset(ig), RowDataset(g)
    got_u, got_c = cuphu_b200.unwrap(dig, dg, 5.0, **kw)
    assert dig.whole_reads == 0 and dg.whole_reads == 0
    assert dig.slices >= 3
    assert np.array_equal(got_u.view(np.int32), want_u.view(np.int32))
    assert np.array_equal(got_c, want_c)


def test_stream_rejects_incomplete_scene(torch_cuda):
    h = C.c_void_p()
    check(lib().cuphu_stream_create(10, 8, 0, 0, C.byref(h)))
    try:
        ig = np.ones((5, 8), np.complex64)
        g = np.full((5, 8), 0.5, np.float32)
        check(lib().cuphu_stream_put_rows(h, 0, 5, ig.ctypes.data, g.ctypes.data, None, None))
        from cuphu_b200._lib import CuPhuSolveOptions, default_params, default_tile_params
        p, t = default_params(), default_tile_params()
        o = CuPhuSolveOptions()
        lib().cuphu_default_solve_options(C.byref(o))
        with pytest.raises(CuPhuError, match="not every row"):
            check(lib().cuphu_stream_unwrap(h, 0, C.byref(p), C.byref(t), C.byref(o), None))
        with pytest.raises(CuPhuError, match="rows outside"):
            check(lib().cuphu_stream_put_rows(h, 8, 5, ig.ctypes.data, g.ctypes.data, None, None))
    finally:
        lib().cuphu_stream_destroy(h)
