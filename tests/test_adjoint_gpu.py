"""Discrete adjoint of the energy iteration (flow held fixed) against central
finite differences of the same GPU forward path."""
import numpy as np
import pytest

from ixchel2d_b200 import _ffi as F
from ixchel2d_b200 import cases
from ixchel2d_b200.adjoint import HotWallNusselt, profile_matrix
from ixchel2d_b200.simple import Simple2D

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative (norm-wise) difference adjoint vs central differences


@pytest.fixture(autouse=True)
def _need_gpu():
    if F.lib.ixb_device_count() < 1:
        pytest.skip("no CUDA device")


def _setup(n=32, Ra=1e4, warm=150):
    case = cases.natural_cavity(n, n, Ra=Ra, T0=0.5)
    sim = Simple2D.from_case(case)
    sim.iterations(warm)          # a developed flow, then held fixed
    state = sim.download()
    return case, sim, state


def test_profile_matrix_interpolates():
    yp = np.array([-0.01, 0.0, 0.25, 0.5, 1.0, 1.02])
    P = profile_matrix(yp, 5)
    th = np.array([1.0, 2.0, 3.0, 4.0, 5.0])
    assert np.allclose(P @ th, [1.0, 1.0, 2.0, 3.0, 5.0, 5.0])


def test_adjoint_matches_central_differences():
    case, sim, state = _setup()
    nodes, K, j0, j1 = 16, 40, 2, 30
    J = HotWallNusselt(sim, state, case.yp, nodes, K, j0, j1)
    rng = np.random.default_rng(5)
    theta = 1.0 + rng.uniform(-0.05, 0.05, nodes)
    g_adj = J.gradient(theta)
    h = 1e-6
    g_fd = np.zeros(nodes)
    for k in range(nodes):
        e = np.zeros(nodes)
        e[k] = h
        g_fd[k] = (J.value(theta + e) - J.value(theta - e)) / (2 * h)
    err = np.linalg.norm(g_adj - g_fd) / np.linalg.norm(g_fd)
    assert err < TOL, (err, g_adj, g_fd)
    assert np.linalg.norm(g_fd) > 1e-3
    # the objective is affine in theta (flow held fixed): a large step is
    # exact and free of the small step's rounding, so the match is far tighter
    H = 1e-2
    for k in (0, nodes // 2, nodes - 1):
        e = np.zeros(nodes)
        e[k] = H
        fd = (J.value(theta + e) - J.value(theta - e)) / (2 * H)
        assert abs(g_adj[k] - fd) <= 1e-7 * max(abs(fd), 1e-3), (k, g_adj[k], fd)


def test_adjoint_leaves_the_state_unchanged_and_torch_wrapper():
    import torch
    case, sim, state = _setup(n=24, warm=60)
    J = HotWallNusselt(sim, state, case.yp, 8, 10, 2, 22)
    sim.upload(state)
    before = sim.download()
    sim.adjoint_energy(10, 2, 22)
    after = sim.download()
    for k in ("u", "v", "p", "T"):
        assert np.array_equal(before[k], after[k])
    theta = torch.full((8,), 1.0, dtype=torch.float64, requires_grad=True)
    nu = J.as_torch()(theta)
    nu.backward()
    assert np.allclose(theta.grad.numpy(), J.gradient(np.ones(8)))
    assert abs(nu.item() - J.value(np.ones(8))) < 1e-12


# ---------------------------------------------------------------------------
# energy adjoint through K outer iterations of an evolving flow that does not
# depend on T (Ri = Riy = 0), with checkpoints every C iterations
# ---------------------------------------------------------------------------
MI_F, NJ_F = 40, 32


def _forced_case():
    """Lid-driven forced convection (Ri = Riy = 0); the T loop runs 1 to 5
    passes per outer iteration (conv_t = 1e-4, iter_ecuaci_max = 3)."""
    return cases.lid_driven_forced(MI_F, NJ_F, Re=100.0, conv_t=1e-4, iter_ecuaci_max=3)


def _profile():
    jj = np.arange(NJ_F + 1)
    return 1.0 + 0.05 * np.sin(0.7 * jj)


def _forward(case, values, K, j0, j1):
    sim = Simple2D.from_case(case)
    sim.set_bc_values(2, 0, values)
    sim.iterations(K)
    nu = sim.nusselt_x(j0, j1)[0]
    st = sim.download()
    sim.close()
    return nu, st


def test_coupled_adjoint_matches_central_differences():
    case = _forced_case()
    K, j0, j1 = 60, 2, NJ_F - 2
    vals = _profile()
    sim = Simple2D.from_case(case)
    sim.set_bc_values(2, 0, vals)
    g, nu = sim.adjoint_energy_coupled(K, 16, j0, j1)
    end = sim.download()
    sim.close()
    # the call leaves the state and objective of a plain K-iteration run
    nu_ref, st_ref = _forward(case, vals, K, j0, j1)
    assert abs(nu - nu_ref) <= 1e-13 * abs(nu_ref), (nu, nu_ref)
    for k in ("u", "v", "p", "T"):
        assert np.max(np.abs(end[k] - st_ref[k])) <= 1e-13 * max(np.max(np.abs(st_ref[k])), 1e-300), k
    # the flow does not depend on T, so nu is affine in the wall values:
    # central differences with a large step are exact
    H = 1e-2
    for L in (3, NJ_F // 2, NJ_F - 3, NJ_F - 1):
        e = np.zeros(NJ_F + 1)
        e[L - 1] = H
        fd = (_forward(case, vals + e, K, j0, j1)[0] - _forward(case, vals - e, K, j0, j1)[0]) / (2 * H)
        assert abs(g[L - 1] - fd) <= 1e-8 * max(abs(fd), 1e-3), (L, g[L - 1], fd)
    assert np.max(np.abs(g)) > 1e-3


def test_coupled_adjoint_is_independent_of_the_checkpoint_interval():
    case = _forced_case()
    K, j0, j1 = 45, 2, NJ_F - 2
    out = []
    for ckpt in (1, 16, 45):
        sim = Simple2D.from_case(case)
        sim.set_bc_values(2, 0, _profile())
        out.append(sim.adjoint_energy_coupled(K, ckpt, j0, j1))
        sim.close()
    for g, nu in out[1:]:
        assert np.array_equal(g, out[0][0]) and nu == out[0][1]


def test_coupled_adjoint_refuses_buoyant_flow():
    case = cases.natural_cavity(24, 24, Ra=1e4, T0=0.5)  # Riy = -1: the flow depends on T
    sim = Simple2D.from_case(case)
    with pytest.raises(Exception):
        sim.adjoint_energy_coupled(10, 5, 2, 20)
    g = np.zeros(25)
    assert F.lib.ixb_adjoint_energy_coupled(sim.h, 10, 5, 2, 20, F.dptr(g), None) == F.EINVAL
    sim.close()


def test_coupled_autograd_function_matches_adjoint():
    import torch
    from ixchel2d_b200.adjoint import HotWallNusseltCoupled
    case = _forced_case()
    sim = Simple2D.from_case(case)
    nodes, K = 12, 30
    J = HotWallNusseltCoupled(sim, case.state, case.yp, nodes, K, 2, NJ_F - 2, ckpt=8)
    theta = torch.tensor(1.0 + 0.02 * np.cos(np.arange(nodes)), dtype=torch.float64, requires_grad=True)
    y = J.as_torch()(theta)
    y.backward()
    g = J.gradient(theta.detach().numpy())
    assert np.allclose(theta.grad.numpy(), g, rtol=0, atol=1e-14 * np.max(np.abs(g)))
    assert float(y.detach()) == J.value(theta.detach().numpy())
    sim.close()
