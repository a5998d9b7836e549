"""Known-answer tests that pin the CPU oracle (oracle/ixb_oracle.cpp).

The reference ships no golden vectors and cannot be compiled here (Fortran),
so the oracle is checked against mathematics: a dense solve, exact metric
formulas, the conduction limit of the cavity (linear profile, known Nusselt
number), the cavity's 180-degree rotation symmetry, and a vanishing
momentum residual at convergence.  CPU only.
"""
import numpy as np
import pytest

from ixchel2d_b200 import cases
from oracle import oracle as O
from tests.conftest import relerr


def _dd_system(n, rng):
    a = rng.uniform(-1, 0, n)
    c = rng.uniform(-1, 0, n)
    b = np.abs(a) + np.abs(c) + rng.uniform(0.1, 1, n)
    d = rng.uniform(-1, 1, n)
    return a, b, c, d


@pytest.mark.parametrize("n", [2, 3, 17, 64, 301])
def test_thomas_matches_dense_solve(n):
    rng = np.random.default_rng(1234 + n)
    a, b, c, d = _dd_system(n, rng)
    A = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
    x_ref = np.linalg.solve(A, d)
    x = O.tridiagonal(a, b, c, d)
    assert relerr(x, x_ref) < 1e-12


def test_thomas_batch_matches_single():
    rng = np.random.default_rng(7)
    sys = [_dd_system(40, rng) for _ in range(9)]
    A, B, Cc, D = (np.array([s[k] for s in sys]) for k in range(4))
    X = O.tridiagonal_batch(A, B, Cc, D)
    for k in range(9):
        assert np.array_equal(X[k], O.tridiagonal(*sys[k]))


def test_metrics_follow_mesh_formulas():
    c = cases.lid_driven_mixed(23, 17)
    o = O.OracleCase(c)
    xu, yv, xp, yp = c.xu, c.yv, c.xp, c.yp
    mi, nj = c.mi, c.nj
    # mod_malla.f90:167-218 (1-based -> 0-based shifts)
    assert np.array_equal(o.metric("deltaxp")[1:], xu[1:] - xu[:-1])
    assert o.metric("deltaxp")[0] == 0.0
    assert np.array_equal(o.metric("deltaxu"), xp[1:] - xp[:-1])
    assert np.array_equal(o.metric("deltayv"), yp[1:] - yp[:-1])
    assert np.array_equal(o.metric("fexp"), (xp[1:] - xu) / (xp[1:] - xp[:-1]))
    assert np.array_equal(o.metric("fexu")[: mi - 1], (xu[1:] - xp[1:mi]) / (xu[1:] - xu[:-1]))
    assert o.metric("fexu")[mi - 1] == 0.0  # never set: read as 0 by the energy assembly
    assert np.array_equal(o.metric("feyv")[: nj - 1], (yv[1:] - yp[1:nj]) / (yv[1:] - yv[:-1]))
    assert o.metric("feyv")[nj - 1] == 0.0


def test_conduction_limit_linear_profile_and_nusselt():
    # Ra -> 0: buoyancy-driven velocity ~ Ra, so T solves pure conduction
    # between T=1 at xp(1) and T=0 at xp(mi+1) with adiabatic top/bottom.
    mi = nj = 24
    c = cases.natural_cavity(mi, nj, Ra=1e-8, Pr=0.71, T0=0.5)
    o = O.OracleCase(c)
    o.iterations(400)
    st = o.get_state()
    T = st["T"]
    xp = c.xp
    lin = (xp[-1] - xp) / (xp[-1] - xp[0])
    for j in range(nj + 1):
        sl = slice(None) if 0 < j < nj else slice(1, -1)  # corner nodes are never swept
        assert np.max(np.abs(T[sl, j] - lin[sl])) < 1e-6
    assert np.max(np.abs(st["u"])) < 1e-6
    # Nu on the vertical walls: -dT/dx = 1/(xp(mi+1)-xp(1)) integrated over
    # the interior rows yp(2)..yp(nj) (corner nodes are never swept)
    nu0, nu1 = o.nusselt_x(2, nj - 2)
    expect = (c.yp[nj - 1] - c.yp[1]) / (xp[-1] - xp[0])
    assert abs(nu0 - expect) < 1e-5
    assert abs(nu1 - expect) < 1e-5


def test_natural_cavity_rotation_symmetry():
    # (x,y) -> (1-x,1-y), (u,v) -> (-u,-v), T -> 1-T maps the converged
    # differentially heated cavity onto itself (the uniform part of the
    # buoyancy goes into a hydrostatic pressure, so only the steady state,
    # not the transient from p=0, is symmetric).
    c = cases.natural_cavity(20, 20, Ra=1e4, T0=0.5)
    o = O.OracleCase(c)
    r = o.iterations(2500)
    assert r["residuo"] < 1e-11
    st = o.get_state()
    u, v, T = st["u"], st["v"], st["T"]
    scale = np.max(np.abs(u))
    assert scale > 1e-2
    # u(ii,jj) <-> u(mi+1-ii, nj+2-jj);  v(ii,jj) <-> v(mi+2-ii, nj+1-jj)
    assert np.max(np.abs(u + u[::-1, ::-1])) < 1e-8 * scale
    assert np.max(np.abs(v + v[::-1, ::-1])) < 1e-8 * np.max(np.abs(v))
    assert np.max(np.abs(T + T[::-1, ::-1] - 1.0)) < 1e-8


def test_residual_vanishes_at_convergence():
    c = cases.natural_cavity(16, 16, Ra=1e3, T0=0.5)
    o = O.OracleCase(c)
    r1 = o.iterations(20)["residuo"]
    r2 = o.iterations(3000)["residuo"]
    assert r2 < 1e-10 < r1


def test_simple_loop_counter_semantics():
    # a loop runs until counter > max: max+2 passes when it never converges
    c = cases.natural_cavity(12, 12)
    o = O.OracleCase(c, iter_simple_max=3, conv_paso=0.0, conv_resi=0.0, conv_u=0.0, conv_p=0.0, conv_t=0.0,
                     iter_ecuaci_max=1)
    r = o.loop()
    assert r["n_simple"] == 5 and r["exit_code"] == 2
    # every inner loop: iter_ecuaci_max + 2 = 3 passes per outer iteration
    assert r["n_momen"] == 15 and r["n_pres"] == 15 and r["n_ener"] == 15


def test_nusselt_y_reference_rule_uses_zero_derivative_past_range():
    # derivada beyond i_1o is 0 in the reference (mod_postproceso.f90:137-160):
    # with a field of uniform wall-normal gradient g, panels fully inside
    # the range integrate -g exactly; the last panel sees zeros.
    c = cases.natural_cavity(10, 10)
    o = O.OracleCase(c)
    T = np.zeros((11, 11), order="F")
    for j in range(11):
        T[:, j] = 2.0 * c.yp[j]
    st = dict(c.state)
    st["T"] = T
    o.set_state(st)
    nu0, _ = o.nusselt_y(1, 8)   # panels at 1,3,5,7: the last reads derivada(9)=0
    xp = c.xp
    inner = -2.0 * (xp[6] - xp[0])
    # last panel: quadratic through (x7,2),(x8,2),(x9,0)
    x0, x1, x2 = xp[6], xp[7], xp[8]
    y0, y1, y2 = 2.0, 2.0, 0.0
    al = ((y2 - y1) / (x2 - x1) - (y1 - y0) / (x1 - x0)) / (x2 - x0)
    be = (y2 - y1) / (x2 - x1) - al * (x1 + x2)
    ga = y0 - al * x0 * x0 - be * x0
    last = al / 3 * (x2 ** 3 - x0 ** 3) + be / 2 * (x2 ** 2 - x0 ** 2) + ga * (x2 - x0)
    assert abs(nu0 - (inner - last)) < 1e-12


def test_per_line_values_equal_to_the_segment_values_change_nothing():
    # the oracle's per-line extension with the values the segments already hold
    c = cases.lid_driven_forced(14, 12)
    a = O.OracleCase(c)
    b = O.OracleCase(c)
    b.set_bc_values(2, 0, np.ones(13))  # side a of T: Dirichlet 1 everywhere
    a.iterations(20)
    b.iterations(20)
    sa, sb = a.get_state(), b.get_state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k
