"""Pins the CPU oracle to the reference: every golden fixture in
tests/golden/ was produced by the reference cuPHU kernels compiled for sm_100a
(tests/golden/make_golden.py); the oracle must reproduce each output bit for
bit from the stored inputs."""
import glob
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _files(pattern):
    fs = sorted(glob.glob(os.path.join(GOLD, pattern)))
    if not fs:
        pytest.skip(f"no golden fixtures {pattern}")
    return fs


def test_costs_fixtures():
    for f in _files("costs_*.npz"):
        d = np.load(f)
        w = d["weights"] if d["weights"].size else None
        got = O.build_costs(d["phase"], d["corr"], float(d["nlooks"]), mode=int(d["mode"]),
                            weights=w)
        assert np.array_equal(got, d["costs"]), os.path.basename(f)


def test_conncomp_fixtures():
    for f in _files("conncomp_*.npz"):
        d = np.load(f)
        kw = {}
        if d["mask"].size:
            kw["mask"] = d["mask"]
        if d["poscost"].size:
            kw["poscost"], kw["negcost"] = d["poscost"], d["negcost"]
        got = O.conncomp(d["unw"], d["corr"], minfrac=float(d["minfrac"]),
                         maxncomps=int(d["maxncomps"]), **kw)
        assert np.array_equal(got, d["labels"]), os.path.basename(f)


def test_integrate_fixture():
    f = _files("integrate.npz")[0]
    d = np.load(f)
    got = O.integrate_phase(d["phase"], d["hflows"], d["vflows"])
    assert np.array_equal(got.view(np.int32), d["unw"].view(np.int32))


def test_incrcost_fixture():
    f = _files("incrcost.npz")[0]
    d = np.load(f)
    p, n, ex = O.incrcost(d["costs"], d["flows"])
    assert np.array_equal(p, d["pos"]) and np.array_equal(n, d["neg"])
    assert ex == bool(d["early_exit"])
