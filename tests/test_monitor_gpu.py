"""The on-device Nusselt monitor (ixb_simple_converge) against the oracle.

The monitor runs blocks of `every` outer iterations and evaluates the
wall-averaged Nusselt number after each block inside the loop graph; it stops
when the monitored wall's value changes by less than tol_dnu between two
evaluations (exit 3), when maxbo < tol_maxbo (exit 4) or at max_iters (exit
5).  The oracle replays the same rule on the host: blocks of `every`
iterations, its own Nusselt number after each, the same tests.

Tolerances: with IXB_SOLVER_EXACT the iteration stream is bit-identical to
the oracle's, so the monitor must stop at the same iteration and the Nusselt
numbers agree to 1e-12 relative (both evaluate the same panel terms and sum
them in panel order).
"""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from ixchel2d_b200 import IxbError, Simple2D, cases
from ixchel2d_b200 import _ffi as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(autouse=True)
def _need_gpu(has_gpu):
    if not has_gpu:
        pytest.skip("no CUDA device")


def _oracle_monitor(o, k0, k1, vertical, wall, every, tol_dnu, tol_maxbo, max_iters):
    """The monitor's rule on the oracle: returns (iterations, exit_code, nu pair, last dnu)."""
    its, prev, evals, dnu, code = 0, 0.0, 0, float("inf"), 0
    while True:
        rep = o.iterations(every)
        its += every
        nu = o.nusselt_x(k0, k1) if vertical else o.nusselt_y(k0, k1)
        v = nu[wall]
        dnu = abs(v - prev) if evals > 0 else float("inf")
        prev, evals = v, evals + 1
        if dnu < tol_dnu:
            code = 3
        elif rep["maxbo"] < tol_maxbo:
            code = 4
        elif its >= max_iters:
            code = 5
        if code:
            return its, code, nu, dnu


@pytest.mark.parametrize("every", [50, 36])  # a multiple of four (unrolled blocks) and one that is not
def test_monitor_stops_where_the_oracle_does(every):
    case = cases.natural_cavity(32, 32, Ra=1e4, T0=0.5)
    g = Simple2D.from_case(case, solver=F.SOLVER_EXACT)
    o = O.OracleCase(case, solver=F.SOLVER_EXACT)
    kw = dict(k0=2, k1=30, vertical=True, wall=0, every=every, tol_dnu=1e-6, tol_maxbo=0.0, max_iters=20000)
    r = g.converge(**kw)
    its, code, nu, dnu = _oracle_monitor(o, **kw)
    assert r["exit_code"] == code == 3
    assert r["n_simple"] == its
    assert abs(r["nu"][0] - nu[0]) <= 1e-12 * abs(nu[0]) and abs(r["nu"][1] - nu[1]) <= 1e-12 * abs(nu[1])
    assert r["dnu"] < 1e-6 and abs(r["dnu"] - dnu) <= 1e-9
    # the state after the monitored run is the oracle's after the same iterations
    gs, os_ = g.download(), o.get_state()
    for k in ("u", "v", "p", "T"):
        assert np.array_equal(gs[k], os_[k]), k
    # and the monitor's Nusselt numbers are those of ixb_nusselt_x on that state
    assert g.nusselt_x(2, 30) == r["nu"]


def test_monitor_horizontal_walls_and_maxbo_exit():
    case = cases.lid_driven_mixed(45, 29, Re=100.0, Ri=1.0)
    g = Simple2D.from_case(case, solver=F.SOLVER_EXACT)
    o = O.OracleCase(case, solver=F.SOLVER_EXACT)
    kw = dict(k0=3, k1=43, vertical=False, wall=0, every=40, tol_dnu=0.0, tol_maxbo=1e-3, max_iters=40000)
    r = g.converge(**kw)
    its, code, nu, _ = _oracle_monitor(o, **kw)
    assert r["exit_code"] == code == 4 and r["n_simple"] == its
    assert r["maxbo"] < 1e-3
    assert abs(r["nu"][0] - nu[0]) <= 1e-12 * abs(nu[0])


def test_monitor_cap_and_hybrid_solver():
    case = cases.natural_cavity(40, 36, Ra=1e5)
    g = Simple2D.from_case(case)
    r = g.converge(k0=2, k1=34, every=100, tol_dnu=0.0, max_iters=300)
    assert r["exit_code"] == 5 and r["n_simple"] == 300
    # the same state as 300 plain iterations (blocks change nothing)
    h = Simple2D.from_case(case)
    h.iterations(300)
    a, b = g.download(), h.download()
    for k in ("u", "v", "p", "T"):
        assert np.array_equal(a[k], b[k]), k
    assert np.isfinite(r["dnu"]) and r["dnu"] > 0.0


def test_monitor_rejects_bad_arguments():
    case = cases.natural_cavity(16, 16)
    g = Simple2D.from_case(case)
    for kw in (dict(every=0), dict(max_iters=0), dict(k0=0), dict(k1=16), dict(wall=2), dict(tol_dnu=-1.0)):
        args = dict(k0=2, k1=14, every=10, tol_dnu=1e-6, max_iters=100)
        args.update(kw)
        with pytest.raises(IxbError) as ei:
            g.converge(**args)
        assert ei.value.status == F.EINVAL, kw


def test_monitor_reports_nonfinite():
    case = cases.natural_cavity(16, 16)
    case.state["T"][5, 5] = np.nan
    g = Simple2D.from_case(case)
    with pytest.raises(IxbError) as ei:
        g.converge(k0=2, k1=14, every=8, tol_dnu=1e-6, max_iters=80)
    assert ei.value.status == F.ENONFINITE


_HOST_CHILD = """
import sys, json
sys.path.insert(0, sys.argv[1])
from ixchel2d_b200 import Simple2D, cases
from ixchel2d_b200 import _ffi as F
g = Simple2D.from_case(cases.natural_cavity(32, 32, Ra=1e4, T0=0.5), solver=F.SOLVER_EXACT)
r = g.converge(k0=2, k1=30, every=50, tol_dnu=1e-6, max_iters=20000)
print(json.dumps({"n": r["n_simple"], "code": r["exit_code"], "nu": r["nu"], "dnu": r["dnu"]}))
"""


def test_host_driven_monitor_matches_the_graph():
    import json
    g = Simple2D.from_case(cases.natural_cavity(32, 32, Ra=1e4, T0=0.5), solver=F.SOLVER_EXACT)
    r = g.converge(k0=2, k1=30, every=50, tol_dnu=1e-6, max_iters=20000)
    env = dict(os.environ, IXB_NO_GRAPH="1")
    out = subprocess.run([sys.executable, "-c", _HOST_CHILD, str(ROOT)], env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    h = json.loads(out.stdout.strip().splitlines()[-1])
    assert h["n"] == r["n_simple"] and h["code"] == r["exit_code"] == 3
    assert tuple(h["nu"]) == r["nu"] and h["dnu"] == r["dnu"]
