"""The oracle's connected components on the behaviours the reference's own
conncomp tests check (test/test_conncomp.py:32-75 there, run on the
reference's CPU relabelling): two plateaus split by a phase jump, an
all-masked scene, the minimum-size filter and the label cap.  CPU only."""
import numpy as np

import oracle as O


def test_two_components():
    unw = np.zeros((20, 30), np.float32)
    unw[:, 15:] += 10.0
    corr = np.full((20, 30), 0.8, np.float32)
    lab = O.conncomp(unw, corr)
    assert set(np.unique(lab)) == {1, 2}
    assert (lab[:, :15] == 1).all() and (lab[:, 15:] == 2).all()


def test_all_masked_returns_zeros():
    unw = np.zeros((10, 10), np.float32)
    corr = np.full((10, 10), 0.8, np.float32)
    lab = O.conncomp(unw, corr, mask=np.zeros((10, 10), np.uint8), minfrac=0.0)
    assert (lab == 0).all()


def test_min_frac_filters_small_components():
    unw = np.zeros((20, 20), np.float32)
    unw[10, 10] = 100.0
    corr = np.full((20, 20), 0.9, np.float32)
    lab = O.conncomp(unw, corr, minfrac=0.05)      # min size 20 px
    assert lab[10, 10] == 0
    assert set(np.unique(lab)) == {0, 1}


def test_max_ncomps_limits_output():
    unw = np.zeros((20, 30), np.float32)
    unw[:, 10:20] += 20.0
    unw[:, 20:] += 40.0
    corr = np.full((20, 30), 0.9, np.float32)
    assert set(np.unique(O.conncomp(unw, corr, minfrac=0.0))) == {1, 2, 3}
    lab = O.conncomp(unw, corr, minfrac=0.0, maxncomps=1)
    assert set(np.unique(lab)) == {0, 1}
