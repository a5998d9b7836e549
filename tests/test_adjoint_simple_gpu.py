"""Discrete adjoint of the full coupled SIMPLE iteration (ixb_adjoint_simple)
for a buoyant flow, against central differences.

In natural convection the flow depends on the wall temperature through the
buoyancy term of the v rows, so the gradient of the hot-wall Nusselt number
runs through the momentum, pressure-correction and energy sweeps and the
velocity/pressure update.  The objective is then nonlinear in the wall
values: central differences with step h carry an O(h^2) error, so the check
uses h = 1e-4 and h = 1e-5 and a tolerance of 1e-5 relative (worst line),
and also the forward of the same call against ixb_simple_iterations."""
import numpy as np
import pytest

from ixchel2d_b200 import _ffi as F
from ixchel2d_b200 import cases
from ixchel2d_b200.simple import Simple2D

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(autouse=True)
def _need_gpu(has_gpu):
    if not has_gpu:
        pytest.skip("no CUDA device")


MI, NJ = 24, 20


def _case():
    return cases.natural_cavity(MI, NJ, Ra=1e4, T0=0.5)


def _profile():
    jj = np.arange(NJ + 1)
    return 1.0 + 0.05 * np.sin(0.9 * jj)


def _nu(case, vals, K):
    sim = Simple2D.from_case(case)
    sim.set_bc_values(F.VAR_T, 0, vals)
    _, nu = sim.adjoint_simple(K, 7, 2, NJ - 2, gradient=False)
    sim.close()
    return nu


def test_forward_is_the_plain_iteration():
    case, vals, K = _case(), _profile(), 15
    a = Simple2D.from_case(case)
    a.set_bc_values(F.VAR_T, 0, vals)
    _, nu = a.adjoint_simple(K, 4, 2, NJ - 2, gradient=False)
    b = Simple2D.from_case(case)
    b.set_bc_values(F.VAR_T, 0, vals)
    b.iterations(K)
    assert abs(nu - b.nusselt_x(2, NJ - 2)[0]) <= 1e-13 * abs(nu)
    sa, sb = a.download(), b.download()
    for k in ("u", "v", "p", "T"):
        assert np.max(np.abs(sa[k] - sb[k])) <= 1e-13 * max(np.max(np.abs(sb[k])), 1e-300), k


def test_buoyant_adjoint_matches_central_differences():
    case, vals, K = _case(), _profile(), 15
    sim = Simple2D.from_case(case)
    sim.set_bc_values(F.VAR_T, 0, vals)
    g, nu = sim.adjoint_simple(K, 4, 2, NJ - 2)
    sim.close()
    assert np.all(np.isfinite(g)) and np.max(np.abs(g)) > 1e-3
    assert g[0] == 0.0 and g[NJ] == 0.0  # lines 1 and nj+1 are not solved
    worst = 0.0
    for L in (3, NJ // 2, NJ - 2):
        fds = []
        for h in (1e-4, 1e-5):
            e = np.zeros(NJ + 1)
            e[L - 1] = h
            fds.append((_nu(case, vals + e, K) - _nu(case, vals - e, K)) / (2 * h))
        fd = fds[1]
        assert abs(fds[0] - fds[1]) <= 1e-6 * abs(fd)  # the differences have settled
        worst = max(worst, abs(g[L - 1] - fd) / abs(fd))
    assert worst < TOL, worst


def test_adjoint_is_independent_of_the_checkpoint_interval():
    case, vals, K = _case(), _profile(), 12
    out = []
    for C_ in (1, 5, 12):
        sim = Simple2D.from_case(case)
        sim.set_bc_values(F.VAR_T, 0, vals)
        out.append(sim.adjoint_simple(K, C_, 2, NJ - 2)[0])
        sim.close()
    for g in out[1:]:
        assert np.max(np.abs(g - out[0])) <= 1e-12 * np.max(np.abs(out[0]))


def test_adjoint_refuses_the_refined_form():
    sim = Simple2D.from_case(_case(), prec=F.PREC_FP32_REFINED)
    with pytest.raises(Exception):
        sim.adjoint_simple(5, 2, 2, NJ - 2)


def test_buoyant_adjoint_matches_oracle_central_differences():
    # the CPU oracle runs the same iteration (one pass of each equation: the
    # default parameters' convergence thresholds end every inner loop after
    # its first pass) with the per-line wall values of ixo_set_bc_values
    from oracle import oracle as O
    case, vals, K = _case(), _profile(), 15
    sim = Simple2D.from_case(case)
    sim.set_bc_values(F.VAR_T, 0, vals)
    g, _ = sim.adjoint_simple(K, 5, 2, NJ - 2)
    sim.close()

    def J(v):
        o = O.OracleCase(case)
        o.set_bc_values(F.VAR_T, 0, v)
        o.iterations(K)
        return o.nusselt_x(2, NJ - 2)[0]

    h = 1e-5
    for L in (4, NJ - 4):
        e = np.zeros(NJ + 1)
        e[L - 1] = h
        fd = (J(vals + e) - J(vals - e)) / (2 * h)
        assert abs(g[L - 1] - fd) <= TOL * abs(fd), (L, g[L - 1], fd)


def test_autograd_function_of_the_full_adjoint():
    import torch
    from ixchel2d_b200.adjoint import HotWallNusseltSimple
    case = _case()
    sim = Simple2D.from_case(case)
    nodes, K = 6, 10
    J = HotWallNusseltSimple(sim, case.state, case.yp, nodes, K, 2, NJ - 2, ckpt=4)
    theta = torch.tensor(1.0 + 0.02 * np.arange(nodes), dtype=torch.float64, requires_grad=True)
    y = J.as_torch()(theta)
    y.backward()
    g = theta.grad.numpy()
    th = theta.detach().numpy()
    assert abs(y.item() - J.value(th)) <= 1e-13 * abs(y.item())
    h = 1e-5
    e = np.zeros(nodes)
    e[2] = h
    fd = (J.value(th + e) - J.value(th - e)) / (2 * h)
    assert abs(g[2] - fd) <= TOL * abs(fd)
    sim.close()
