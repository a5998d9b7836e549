"""Parity at the benchmarked size: the heated lid-driven cavity in mixed
convection (Re 100, Ri 1, Pr 0.71) on the tanh-clustered 701x301 mesh
(mi=701, nj=301: 302 x-lines of 702 rows, 702 y-lines of 302 rows), and the
transposed orientation 301x701 (mi=301, nj=701: 702 x-lines of 302 rows, 302
y-lines of 702 rows), against the CPU oracle after 30 outer iterations from
rest.

Tolerances, as in the small-grid parity tests:
* IXB_SOLVER_EXACT: bit-identical on the seven state fields and on au, av,
  p' and the mass source b_o, and the five norms to 1e-12 relative;
* IXB_SOLVER_HYBRID (the benchmarked binary64 form, with Newton-refined
  reciprocals in the line solve): 1e-10 relative on every field;
* IXB_PREC_FP32_REFINED: before convergence the binary32 line solves of the
  defect corrections leave binary32-sized differences; u, v and T stay
  within 1e-4 relative L2 of the oracle.
"""
import numpy as np
import pytest

from ixchel2d_b200 import Simple2D, cases
from ixchel2d_b200 import _ffi as F
from oracle import oracle as O
from tests.conftest import relerr

pytestmark = pytest.mark.gpu

STATE = ("u", "v", "p", "T", "u_ant", "v_ant", "T_ant")
HYBRID_TOL = 1e-10
REFINED_L2_TOL = 1e-4
ITERS = 30
SIZES = {"701x301": (701, 301), "301x701": (301, 701)}


@pytest.fixture(autouse=True)
def _need_gpu(has_gpu):
    if not has_gpu:
        pytest.skip("no CUDA device")


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


_ORACLE = {}


def _oracle_run(name):
    """Oracle state, aux arrays and report after ITERS iterations (cached per size)."""
    if name not in _ORACLE:
        mi, nj = SIZES[name]
        case = cases.lid_driven_mixed(mi, nj, Re=100.0, Ri=1.0, Pr=0.71, beta=1.2)
        o = O.OracleCase(case)
        rep = o.iterations(ITERS)
        _ORACLE[name] = (case, o.get_state(), o.get_aux(), rep)
        o.close()
    return _ORACLE[name]


@pytest.mark.parametrize("name", list(SIZES))
def test_headline_exact_solver_bit_identical(name):
    case, os_, oa, ro = _oracle_run(name)
    g = Simple2D.from_case(case, solver=F.SOLVER_EXACT)
    rg = g.iterations(ITERS)
    gs, ga = g.download(), g.download_aux()
    g.close()
    for k in STATE:
        assert np.array_equal(gs[k], os_[k]), (k, relerr(gs[k], os_[k]))
    for k in ("au", "av", "corr_pres"):
        assert np.array_equal(ga[k], oa[k]), (k, relerr(ga[k], oa[k]))
    sl = (slice(1, -1), slice(1, -1))
    assert np.array_equal(ga["b_o"][sl], oa["b_o"][sl]), relerr(ga["b_o"], oa["b_o"])
    for k in ("maxbo", "residuo", "err_u", "err_p", "err_t"):
        assert abs(rg[k] - ro[k]) <= 1e-12 * abs(ro[k]), (k, rg[k], ro[k])
    assert rg["n_simple"] == ro["n_simple"] == ITERS


@pytest.mark.parametrize("name", list(SIZES))
def test_headline_hybrid_binary64_within_tolerance(name):
    case, os_, _, ro = _oracle_run(name)
    g = Simple2D.from_case(case)
    rg = g.iterations(ITERS)
    gs = g.download()
    g.close()
    for k in STATE:
        assert relerr(gs[k], os_[k]) < HYBRID_TOL, (k, relerr(gs[k], os_[k]))
    for k in ("maxbo", "residuo"):
        assert abs(rg[k] - ro[k]) <= 1e-9 * abs(ro[k]), (k, rg[k], ro[k])


@pytest.mark.parametrize("name", list(SIZES))
def test_headline_hybrid_binary64_in_autotuned_shapes(name):
    # the benchmark runs the shapes the autotuner picks; they must keep parity too
    case, os_, _, _ = _oracle_run(name)
    g = Simple2D.from_case(case)
    g.autotune(reps=2)
    g.upload(case.state)
    g.iterations(ITERS)
    gs = g.download()
    g.close()
    for k in STATE:
        assert relerr(gs[k], os_[k]) < HYBRID_TOL, (k, relerr(gs[k], os_[k]))


@pytest.mark.parametrize("name", list(SIZES))
def test_headline_refined_tracks_binary64(name):
    case, os_, _, ro = _oracle_run(name)
    g = Simple2D.from_case(case, prec=F.PREC_FP32_REFINED)
    rg = g.iterations(ITERS)
    gs = g.download()
    g.close()
    for k in ("u", "v", "T"):
        assert rel_l2(gs[k], os_[k]) < REFINED_L2_TOL, (k, rel_l2(gs[k], os_[k]))
    assert np.isfinite(rg["maxbo"]) and abs(rg["maxbo"] - ro["maxbo"]) <= 1e-3 * abs(ro["maxbo"])
