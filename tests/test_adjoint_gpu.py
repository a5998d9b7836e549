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
