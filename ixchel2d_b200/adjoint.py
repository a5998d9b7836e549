"""Gradient of the hot-wall Nusselt number with respect to a piecewise-linear
hot-wall temperature profile: with the flow held fixed (HotWallNusselt, over
ixb_energy_iterations and ixb_adjoint_energy), through K outer SIMPLE
iterations of a flow that does not depend on T (HotWallNusseltCoupled, over
ixb_simple_iterations and ixb_adjoint_energy_coupled), or through K outer
iterations of any flow, buoyant included (HotWallNusseltSimple, over
ixb_adjoint_simple).  as_torch() wraps
either in a thin torch.autograd.Function, used to check the adjoint against
finite differences."""
from __future__ import annotations

import numpy as np

from .simple import Simple2D
from . import _ffi as F


def profile_matrix(yp: np.ndarray, nodes: int) -> np.ndarray:
    """P (len(yp) x nodes): value at yp[j] = sum_n P[j, n] theta_n, linear
    interpolation between `nodes` equally spaced nodes on [0, 1], constant
    beyond them."""
    s = np.clip(np.asarray(yp, dtype=np.float64), 0.0, 1.0) * (nodes - 1)
    k = np.minimum(np.floor(s).astype(int), nodes - 2)
    t = s - k
    P = np.zeros((len(s), nodes))
    P[np.arange(len(s)), k] = 1.0 - t
    P[np.arange(len(s)), k + 1] = t
    return P


class HotWallNusselt:
    """J(theta) = nu0 of ixb_nusselt_x(j0, j1) after K passes of the T sweeps
    from `state`, with the side-a T boundary values set to P theta."""

    def __init__(self, sim: Simple2D, state: dict, yp: np.ndarray, nodes: int, K: int, j0: int, j1: int):
        self.sim, self.state, self.K, self.j0, self.j1 = sim, state, K, j0, j1
        self.P = profile_matrix(yp, nodes)

    def value(self, theta: np.ndarray) -> float:
        self.sim.set_bc_values(F.VAR_T, 0, self.P @ np.asarray(theta, dtype=np.float64))
        self.sim.upload(self.state)
        self.sim.energy_iterations(self.K)
        return self.sim.nusselt_x(self.j0, self.j1)[0]

    def gradient(self, theta: np.ndarray) -> np.ndarray:
        self.sim.set_bc_values(F.VAR_T, 0, self.P @ np.asarray(theta, dtype=np.float64))
        self.sim.upload(self.state)
        return self.P.T @ self.sim.adjoint_energy(self.K, self.j0, self.j1)

    def as_torch(self):
        import torch

        outer = self

        class _Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, theta):
                th = theta.detach().cpu().double().numpy()
                ctx.save_for_backward(theta)
                return torch.tensor(outer.value(th), dtype=torch.float64)

            @staticmethod
            def backward(ctx, g):
                (theta,) = ctx.saved_tensors
                grad = outer.gradient(theta.detach().cpu().double().numpy())
                return g * torch.tensor(grad, dtype=theta.dtype, device=theta.device)

        return _Fn.apply


class HotWallNusseltCoupled(HotWallNusselt):
    """J(theta) = nu0 of ixb_nusselt_x(j0, j1) after K outer SIMPLE
    iterations from `state` (the flow evolves with them but does not depend
    on T: Ri = Riy = 0), with the side-a T boundary values set to P theta.
    The gradient comes from ixb_adjoint_energy_coupled with checkpoints every
    `ckpt` iterations."""

    def __init__(self, sim: Simple2D, state: dict, yp: np.ndarray, nodes: int, K: int, j0: int, j1: int,
                 ckpt: int = 50):
        super().__init__(sim, state, yp, nodes, K, j0, j1)
        self.ckpt = ckpt

    def value(self, theta: np.ndarray) -> float:
        self.sim.set_bc_values(F.VAR_T, 0, self.P @ np.asarray(theta, dtype=np.float64))
        self.sim.upload(self.state)
        self.sim.iterations(self.K)
        return self.sim.nusselt_x(self.j0, self.j1)[0]

    def gradient(self, theta: np.ndarray) -> np.ndarray:
        self.sim.set_bc_values(F.VAR_T, 0, self.P @ np.asarray(theta, dtype=np.float64))
        self.sim.upload(self.state)
        g, _ = self.sim.adjoint_energy_coupled(self.K, self.ckpt, self.j0, self.j1)
        return self.P.T @ g


class HotWallNusseltSimple(HotWallNusseltCoupled):
    """J(theta) = nu0 of ixb_nusselt_x(j0, j1) after K outer SIMPLE
    iterations from `state` (one pass of each equation), with the side-a T
    boundary values set to P theta, for any flow: the gradient comes from
    ixb_adjoint_simple, the adjoint of the full coupled iteration (momentum,
    pressure correction and energy), so buoyant flows are covered."""

    def value(self, theta: np.ndarray) -> float:
        self.sim.set_bc_values(F.VAR_T, 0, self.P @ np.asarray(theta, dtype=np.float64))
        self.sim.upload(self.state)
        return self.sim.adjoint_simple(self.K, self.ckpt, self.j0, self.j1, gradient=False)[1]

    def gradient(self, theta: np.ndarray) -> np.ndarray:
        self.sim.set_bc_values(F.VAR_T, 0, self.P @ np.asarray(theta, dtype=np.float64))
        self.sim.upload(self.state)
        g, _ = self.sim.adjoint_simple(self.K, self.ckpt, self.j0, self.j1)
        return self.P.T @ g
