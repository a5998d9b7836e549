"""The discrete energy adjoints against central differences of the CPU oracle
(the restatement of the reference's own CPU path), not only of the GPU
forward path.

The per-line hot-wall values the adjoint differentiates with respect to are an
extension of the reference's boundary tables (at most 15 piecewise-constant
segments per side); the oracle carries the same extension (ixo_set_bc_values),
checked here bit for bit against the library's ixb_set_bc_values.

In both configurations the flow does not depend on T (held fixed, or evolving
with Ri = Riy = 0), so the objective is affine in the wall values and central
differences with a step of 1e-2 are exact up to rounding: the adjoint must
match them to 1e-8 relative."""
import numpy as np
import pytest

from ixchel2d_b200 import _ffi as F
from ixchel2d_b200 import cases
from ixchel2d_b200.adjoint import HotWallNusselt
from ixchel2d_b200.simple import Simple2D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

H = 1e-2
TOL = 1e-8
STATE = ("u", "v", "p", "T", "u_ant", "v_ant", "T_ant")


@pytest.fixture(autouse=True)
def _need_gpu(has_gpu):
    if not has_gpu:
        pytest.skip("no CUDA device")


MI_F, NJ_F = 40, 32


def _forced_case():
    return cases.lid_driven_forced(MI_F, NJ_F, Re=100.0, conv_t=1e-4, iter_ecuaci_max=3)


def _profile():
    jj = np.arange(NJ_F + 1)
    return 1.0 + 0.05 * np.sin(0.7 * jj)


def test_per_line_values_match_the_library_bit_for_bit():
    case = _forced_case()
    vals = _profile()
    g = Simple2D.from_case(case, solver=F.SOLVER_EXACT)
    o = O.OracleCase(case, solver=F.SOLVER_EXACT)
    g.set_bc_values(F.VAR_T, 0, vals)
    o.set_bc_values(F.VAR_T, 0, vals)
    g.iterations(30)
    o.iterations(30)
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert np.array_equal(gs[k], os_[k]), k


def test_coupled_adjoint_matches_oracle_central_differences():
    case = _forced_case()
    K, j0, j1 = 60, 2, NJ_F - 2
    vals = _profile()
    sim = Simple2D.from_case(case)
    sim.set_bc_values(F.VAR_T, 0, vals)
    g, _ = sim.adjoint_energy_coupled(K, 16, j0, j1)

    def J(v):
        o = O.OracleCase(case)
        o.set_bc_values(F.VAR_T, 0, v)
        o.iterations(K)
        return o.nusselt_x(j0, j1)[0]

    for L in (3, NJ_F // 2, NJ_F - 3):
        e = np.zeros(NJ_F + 1)
        e[L - 1] = H
        fd = (J(vals + e) - J(vals - e)) / (2 * H)
        assert abs(g[L - 1] - fd) <= TOL * max(abs(fd), 1e-3), (L, g[L - 1], fd)


def test_fixed_flow_adjoint_matches_oracle_central_differences():
    n, K, j0, j1, nodes = 32, 40, 2, 30, 16
    case = cases.natural_cavity(n, n, Ra=1e4, T0=0.5)
    sim = Simple2D.from_case(case)
    sim.iterations(150)  # a developed flow, then held fixed
    state = sim.download()
    J = HotWallNusselt(sim, state, case.yp, nodes, K, j0, j1)
    theta = 1.0 + np.random.default_rng(5).uniform(-0.05, 0.05, nodes)
    g = J.gradient(theta)

    def Jo(th):
        o = O.OracleCase(case)
        o.set_state(state)
        o.set_bc_values(F.VAR_T, 0, J.P @ th)
        o.energy_passes(K)
        return o.nusselt_x(j0, j1)[0]

    for k in (0, nodes // 2, nodes - 2):
        e = np.zeros(nodes)
        e[k] = H
        fd = (Jo(theta + e) - Jo(theta - e)) / (2 * H)
        assert abs(g[k] - fd) <= TOL * max(abs(fd), 1e-3), (k, g[k], fd)
