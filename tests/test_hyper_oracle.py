"""The neo-Hookean oracle (oracle/hyper_oracle.py) pinned without jax: its
residual is the gradient of its energy and its tangent the derivative of its
residual (central differences), and its Newton iteration reproduces the
behaviour the reference's tests assert for the nonlinear Galerkin path
(tests/test_methods.py:106-126: at most 10 steps, quadratic convergence)."""

import numpy as np
import pytest

import jaxiga_b200 as jx
from oracle import hyper_oracle as H
from oracle import iga_oracle as O


def model(dim, rational=False, mu=384.6, lam=576.9):
    if dim == 2:
        base = jx.primitives.quarter_annulus(1.0, 2.0) if rational else jx.primitives.rectangle(0, 0, 1, 1)
        patch = base.elevate(2).refine(1)
    else:
        patch = jx.primitives.cuboid([0, 0, 0], [1.0, 0.8, 1.2]).elevate(1).refine(1)
    V = jx.FunctionSpace(patch, vec=dim)
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec)
    return V, H.NeoHookean(S, mu, lam)


@pytest.mark.parametrize("dim,rational", [(2, False), (2, True), (3, False)])
def test_residual_is_the_energy_gradient_and_tangent_its_derivative(dim, rational):
    V, M = model(dim, rational)
    rng = np.random.default_rng(dim)
    u = 0.03 * rng.standard_normal(V.n_dofs)
    v = rng.standard_normal(V.n_dofs)
    h = 1e-6
    fd = (M.energy(u + h * v) - M.energy(u - h * v)) / (2 * h)
    r = M.residual(u)
    assert abs(fd - r @ v) <= 1e-7 * max(abs(r @ v), np.abs(r).sum() * 1e-3)
    Kv = M.tangent(u) @ v
    fdr = (M.residual(u + h * v) - M.residual(u - h * v)) / (2 * h)
    assert np.abs(fdr - Kv).max() <= 1e-6 * np.abs(Kv).max()
    # symmetric, and the small-strain limit is linear elasticity with the same Lame pair
    K = M.tangent(u)
    assert abs(K - K.T).max() <= 1e-10 * abs(K).max()


def test_small_strain_limit_is_linear_elasticity():
    V, M = model(2, mu=1.0, lam=0.5)
    S = M.space
    lam, mu = 0.5, 1.0
    E = mu * (3 * lam + 2 * mu) / (lam + mu)
    nu = lam / (2 * (lam + mu))
    A = O.Assembled(S, "elasticity", {"E": E, "nu": nu, "plane": "strain"}, np.zeros(0, dtype=int), np.zeros(0))
    K0 = M.tangent(np.zeros(V.n_dofs))
    assert abs(K0 - A.K_full).max() <= 1e-12 * abs(A.K_full).max()


def test_newton_converges_quadratically():
    V, M = model(2)
    problem = jx.Hyperelasticity(V, dirichlet=[jx.DirichletBC([0.0, 0.0], where="bottom"),
                                               jx.DirichletBC([0.0, 0.2], where="top")])
    pres, vals = problem.resolve_dirichlet({"mu": 384.6, "lam": 576.9})
    u, st = H.newton(M, pres, vals, np.zeros(V.n_dofs))
    assert st["converged"] and st["iterations"] <= 10
    hist = st["history"]
    assert hist[-1] < 1e-9 and hist[-1] < hist[-2] ** 1.5
