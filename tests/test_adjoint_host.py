"""The torch.autograd plumbing of the adjoint (vlasolve_b200.adjoint) with a
stand-in problem on the CPU: FinalDensity must hand the problem's
vector-Jacobian product to autograd unchanged."""
import numpy as np
import torch

from vlasolve_b200.adjoint import FinalDensity


class LinearProblem:
    """rho(theta) = A theta + c, an exactly known Jacobian."""

    def __init__(self):
        rng = np.random.default_rng(20261203)
        self.A = rng.standard_normal((7, 3))
        self.c = rng.standard_normal(7)
        self.calls = []

    def run(self, theta):
        self.calls.append(("run", np.array(theta)))
        return self.A @ np.asarray(theta) + self.c

    def vjp(self, g):
        self.calls.append(("vjp", np.array(g)))
        return self.A.T @ np.asarray(g)


def test_final_density_gradient_is_the_problem_vjp():
    p = LinearProblem()
    th = torch.tensor([2.0, 0.5, 0.5], dtype=torch.float64, requires_grad=True)
    target = torch.zeros(7, dtype=torch.float64)
    rho = FinalDensity.apply(th, p)
    L = ((rho - target) ** 2).sum()
    L.backward()
    expect = 2 * p.A.T @ (p.A @ th.detach().numpy() + p.c)
    np.testing.assert_allclose(th.grad.numpy(), expect, rtol=1e-14)
    assert [c[0] for c in p.calls] == ["run", "vjp"]


def test_final_density_gradcheck():
    p = LinearProblem()
    th = torch.tensor([1.0, -0.3, 0.7], dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda t: FinalDensity.apply(t, p), (th,))
