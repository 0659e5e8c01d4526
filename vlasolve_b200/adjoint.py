"""Gradients of a final radial-density loss with respect to initial-condition
parameters, through the hand-written adjoint of the step.

The reference has no derivative code.  The adjoint of the N linked steps runs
in the CUDA library (vls_adjoint_forward / vls_adjoint_backward: transposed
drift and chain-tail gathers, transposed natural-BC prefilter, transposed
kick with its shift derivative, transposed enclosed-mass scan and moment),
with checkpoints every K steps and recomputation of each segment.  It yields
dL/df0 and dL/d(initial chain values).  The map from the parameters theta to
the initial state (the analytic distribution function and its
renormalisation, vlasovSolver21::renormalize) is differentiated by central
differences of that map alone, in FP64, with no time steps: the two grids
of each parameter are evaluated on the device and contracted there with
dL/df0 (vls_adjoint_init_dot).

FinalDensity wraps this as a torch.autograd.Function: forward(theta) returns
the radial density of the final state, backward(grad) returns grad_theta.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import VlasovSolver21Spline


class DensityProblem:
    """A forward run of `nsteps` linked steps from the initial state generated
    with parameters `params` (init.* names) = theta."""

    def __init__(self, cfg, precision: str = "fp64", nsteps: int = 1,
                 checkpoint_every: int = 1, params=("R0", "alpha", "smoothingRadius"),
                 ic_step: float = 1e-6, device: int = 0, inner_every: int = 0,
                 layout: dict | None = None):
        self.solver = VlasovSolver21Spline(cfg, precision=precision, device=device, init=False,
                                           layout=layout)
        # second-level checkpoint spacing of the backward pass (0: chosen from
        # free device memory)
        self.solver.adjoint_set_inner(inner_every)
        # initial_state() makes FP64 grids whatever the storage precision: an
        # FP64 handle of its own for FP32 storage, created on first use
        self._cfg, self._device, self._precision = cfg, device, precision
        self._ic = self.solver if precision == "fp64" else None
        self.nsteps, self.K = int(nsteps), int(checkpoint_every)
        self.params = tuple(params)
        self.ic_step = ic_step
        self.vol = None
        self.theta = None

    @property
    def ic(self) -> VlasovSolver21Spline:
        """The FP64 handle initial_state() evaluates on."""
        if self._ic is None:
            self._ic = VlasovSolver21Spline(self._cfg, precision="fp64", device=self._device,
                                            init=False)
        return self._ic

    def close(self):
        """Frees the device memory of the handles."""
        if self._ic is not None and self._ic is not self.solver:
            self._ic.close()
        self._ic = None
        self.solver.close()

    def initial_state(self, theta):
        """FP64 initial grid and chain values for parameters theta."""
        self.ic.set_init_params(**dict(zip(self.params, map(float, theta))))
        return self.ic.f, self.ic.chains()["val"]

    def run(self, theta) -> np.ndarray:
        """Radial density of the final state for parameters theta."""
        self.theta = np.asarray(theta, dtype=np.float64).copy()
        self.solver.set_init_params(**dict(zip(self.params, map(float, self.theta))))
        self.solver.set_time(0.0, 0)
        self.solver.adjoint_forward(self.nsteps, self.K)
        if self.vol is None:
            self.vol = self.solver.shell_volumes()
        return self.solver.radial_density()

    def vjp(self, grad_rho) -> np.ndarray:
        """grad_theta = (d rho / d theta)^T grad_rho at the last run's theta."""
        g = np.asarray(grad_rho, dtype=np.float64)
        dbins = np.zeros(self.solver.nr)
        dbins[:-1] = g / self.vol
        self.solver.adjoint_backward(dbins)
        out = np.zeros(len(self.params))
        for k in range(len(self.params)):
            h = self.ic_step * max(1.0, abs(self.theta[k]))
            tp, tm = self.theta.copy(), self.theta.copy()
            tp[k] += h
            tm[k] -= h
            dg, dc = self.solver.adjoint_init_dot(dict(zip(self.params, map(float, tp))),
                                                  dict(zip(self.params, map(float, tm))))
            out[k] = (dg + dc) / (2 * h)
        return out


class FinalDensity(torch.autograd.Function):
    """theta (float64 tensor of the problem's parameters) -> final radial
    density (float64 tensor of N_r - 1 shells)."""

    @staticmethod
    def forward(ctx, theta, problem: DensityProblem):
        rho = problem.run(theta.detach().cpu().numpy())
        ctx.problem = problem
        return torch.as_tensor(rho, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_rho):
        g = ctx.problem.vjp(grad_rho.detach().cpu().numpy())
        return torch.as_tensor(g, dtype=torch.float64), None


def final_density(theta: torch.Tensor, problem: DensityProblem) -> torch.Tensor:
    return FinalDensity.apply(theta, problem)
