"""Batched cavities (ixb_batch_*): instances of different sizes and
parameters advanced together, one launch per phase, against the same
instances run one at a time through the single-instance path."""
import numpy as np
import pytest

from ixchel2d_b200 import _ffi as F
from ixchel2d_b200 import cases
from ixchel2d_b200.batch import Batch
from ixchel2d_b200.simple import Simple2D

pytestmark = pytest.mark.gpu

STATE = ("u", "v", "p", "T")


@pytest.fixture(autouse=True)
def _need_gpu():
    if F.lib.ixb_device_count() < 1:
        pytest.skip("no CUDA device")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _mixed_cases():
    return [cases.natural_cavity(40, 40, Ra=1e4), cases.natural_cavity(72, 56, Ra=3e5),
            cases.lid_driven_mixed(45, 29), cases.natural_cavity(33, 65, Ra=1e3),
            cases.lid_driven_mixed(90, 61, Re=50.0, Ri=0.5)]


@pytest.mark.parametrize("prec", [F.PREC_FP64, F.PREC_FP32_REFINED])
def test_batch_matches_single_instances(prec):
    cs = _mixed_cases()
    # conv_paso = 0: no instance meets the outer test, every one runs the budget
    bt = Batch.from_cases(cs, prec=prec, conv_paso=0.0)
    singles = [Simple2D.from_case(c, prec=prec) for c in cs]
    for k in range(8):
        bt.set_sweep_shape(k, 2, 64)
        for s in singles:
            s.set_sweep_shape(k, 2, 64)
    assert bt.iterate(37) == len(cs)
    for i, (s, c) in enumerate(zip(singles, cs)):
        s.iterations(37)
        a, b = bt[i].download(), s.download()
        for k in STATE:
            assert rel(a[k], b[k]) < 1e-11, (i, k, rel(a[k], b[k]))
        rep = bt.report(i)
        assert rep["n_simple"] == 37 and rep["exit_code"] == 2 and rep["status"] == F.OK


def test_batch_instances_stop_on_their_own_outer_test():
    cs = [cases.natural_cavity(24, 24, Ra=1e3), cases.natural_cavity(48, 40, Ra=1e5)]
    bt = Batch.from_cases(cs, prec=F.PREC_FP64, conv_paso=1e-6, conv_resi=1e30)
    left = bt.iterate(20000)
    reps = [bt.report(i) for i in range(2)]
    assert left == 0
    for r in reps:
        assert r["exit_code"] == 1 and r["maxbo"] < 1e-6
    assert reps[0]["n_simple"] != reps[1]["n_simple"]
    # an instance that stopped keeps its state: one more call changes nothing
    before = bt[0].download()
    bt.iterate(5)
    after = bt[0].download()
    for k in STATE:
        assert np.array_equal(before[k], after[k])
    # the single-instance path reaches the same state in the same number of iterations
    s = Simple2D.from_case(cs[0])
    s.iterations(reps[0]["n_simple"])
    ref = s.download()
    for k in STATE:
        assert rel(before[k], ref[k]) < 1e-11, k


def test_batch_autotune_keeps_state_and_results():
    cs = _mixed_cases()[:3]
    bt = Batch.from_cases(cs, prec=F.PREC_FP32_REFINED, conv_paso=0.0)
    before = [bt[i].download() for i in range(3)]
    chosen = bt.autotune(reps=2)
    assert all((c[0], c[1]) in Simple2D.SHAPES for c in chosen.values())
    for i in range(3):
        after = bt[i].download()
        for k in STATE:
            assert np.array_equal(before[i][k], after[k])
    bt.iterate(10)
    for i in range(3):
        assert all(np.all(np.isfinite(bt[i].download()[k])) for k in STATE)


def test_batch_nonfinite_instance_is_reported_and_others_continue():
    cs = _mixed_cases()[:2]
    bad = cs[1].state
    bad["T"] = bad["T"].copy()
    bad["T"][5, 5] = np.nan
    bt = Batch.from_cases(cs, prec=F.PREC_FP64, conv_paso=0.0)
    bt.iterate(3)
    r0, r1 = bt.report(0), bt.report(1)
    assert r1["status"] == F.ENONFINITE and r1["exit_code"] == 3
    assert r0["status"] == F.OK and r0["n_simple"] == 3


def test_batch_rejects_bad_sizes():
    import ctypes as C
    mi = (C.c_int * 2)(64, 2000)
    nj = (C.c_int * 2)(64, 64)
    b = C.c_void_p()
    assert F.lib.ixb_batch_create(2, mi, nj, F.PREC_FP64, C.byref(b)) == F.EINVAL


def test_batch_host_driven_loop_matches_graph(monkeypatch):
    cs = _mixed_cases()[:3]
    g = Batch.from_cases(cs, prec=F.PREC_FP32_REFINED, conv_paso=0.0)
    monkeypatch.setenv("IXB_NO_GRAPH", "1")
    h = Batch.from_cases(cs, prec=F.PREC_FP32_REFINED, conv_paso=0.0)
    assert g.iterate(12) == 3 and h.iterate(12) == 3
    for i in range(3):
        a, b = g[i].download(), h[i].download()
        for k in STATE:
            assert np.array_equal(a[k], b[k]), (i, k)
        assert h.report(i)["n_simple"] == 12
