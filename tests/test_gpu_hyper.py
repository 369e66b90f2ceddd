"""The nonlinear Galerkin path on the device (compressible neo-Hookean,
src/jaxiga/forms/library.py:206-225) against its oracle restatement
(oracle/hyper_oracle.py): the stored energy, the residual and the tangent
K(u) v and its diagonal at a deformed state, in 2D (polynomial and rational)
and 3D, to 1e-12; and Newton's method on the reference's own nonlinear test
cases (tests/test_methods.py:106-126, tests/test_implicit_diff.py:79-91):
converged in at most 10 steps, quadratically, to the oracle's solution."""

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200 import history_list
from oracle import hyper_oracle as H
from oracle import iga_oracle as O

pytestmark = pytest.mark.gpu


def space(dim, rational):
    if dim == 2:
        base = jx.primitives.quarter_annulus(1.0, 2.0) if rational else jx.primitives.rectangle(0, 0, 1, 1)
        patch = base.elevate(2).refine(3)
    else:
        patch = jx.primitives.cuboid([0, 0, 0], [1.0, 0.8, 1.2]).elevate(1).refine(2)
    return jx.FunctionSpace(patch, vec=dim)


@pytest.mark.parametrize("dim,rational", [(2, False), (2, True), (3, False)])
def test_state_residual_tangent_and_diagonal_match_oracle(dim, rational):
    V = space(dim, rational)
    mu, lam = 384.6, 576.9
    M = H.NeoHookean(O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec), mu, lam)
    rng = np.random.default_rng(10 * dim + rational)
    u = 0.02 * rng.standard_normal(V.n_dofs)
    x = rng.standard_normal(V.n_dofs)
    op = jx.Operator(V, "hyperelastic", (mu, lam))
    e = op.state(u, energy=True)
    assert abs(e - M.energy(u)) <= 1e-12 * abs(M.energy(u))
    r = op.residual().cpu().numpy()
    r_o = M.residual(u)
    assert np.abs(r - r_o).max() <= 1e-12 * np.abs(r_o).max()
    K = M.tangent(u)
    y = op.apply(x, masked=False).cpu().numpy()
    assert np.abs(y - K @ x).max() <= 1e-12 * np.abs(K @ x).max()
    d = op.diag().cpu().numpy()
    assert np.abs(d - K.diagonal()).max() <= 1e-12 * np.abs(K.diagonal()).max()
    # back to the undeformed state: the tangent is linear elasticity's (plane strain)
    op.state(np.zeros(V.n_dofs))
    E = mu * (3 * lam + 2 * mu) / (lam + mu)
    nu = lam / (2 * (lam + mu))
    lin = jx.Operator(V, "elasticity", (E, nu), plane_strain=True)
    y0, y1 = op.apply(x, masked=False).cpu().numpy(), lin.apply(x, masked=False).cpu().numpy()
    assert np.abs(y0 - y1).max() <= 1e-12 * np.abs(y1).max()
    assert np.abs(op.residual().cpu().numpy()).max() <= 1e-12 * mu
    op.close()
    lin.close()


def test_newton_matches_oracle_and_converges_quadratically():
    """tests/test_methods.py:106-126: a square pulled upward at the top."""
    V = jx.FunctionSpace(jx.primitives.rectangle(0, 0, 1, 1).elevate(2).refine(1), vec=2)
    problem = jx.Hyperelasticity(V, dirichlet=[jx.DirichletBC([0.0, 0.0], where="bottom"),
                                               jx.DirichletBC([0.0, 0.2], where="top")])
    params = {"mu": 384.6, "lam": 576.9}
    sol = jx.solve(problem, params=params)
    st = sol.stats
    assert st["converged"] and st["iterations"] <= 10 and not st["stalled"]
    hist = history_list(st)
    assert hist[-1] < 1e-9 and hist[-1] < hist[-2] ** 1.5
    M = H.NeoHookean(O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec), 384.6, 576.9)
    pres, vals = problem.resolve_dirichlet(params)
    u_o, st_o = H.newton(M, pres, vals, np.zeros(V.n_dofs))
    assert st_o["converged"]
    assert np.abs(sol.u - u_o).max() <= 1e-8 * np.abs(u_o).max()
    assert st["iterations"] == st_o["iterations"]


def test_newton_with_a_traction_and_the_lame_conversion():
    """tests/test_implicit_diff.py:79-91: clamped left edge, traction on the right."""
    V = jx.FunctionSpace(jx.primitives.rectangle(0, 0, 1, 1).elevate(2).refine(2), vec=2)
    problem = jx.Hyperelasticity(
        V, dirichlet=[jx.DirichletBC([0.0, 0.0], where="left")],
        neumann=[jx.Neumann(lambda x, n, p: np.stack([np.full(len(x), p["load"]), np.full(len(x), 0.3 * p["load"])],
                                                      axis=1), where="right")])
    params = {"E": 200.0, "nu": 0.3, "load": 5.0}
    sol = jx.solve(problem, params=params)
    assert sol.stats["converged"]
    lam, mu = H.lame(200.0, 0.3)
    M = H.NeoHookean(O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec), mu, lam)
    pres, vals = problem.resolve_dirichlet(params)
    # the same traction load, assembled by the oracle's boundary quadrature
    from jaxiga_b200.solve import _problem_operator  # noqa: F401  (the device load is checked through the solve)
    import torch

    op = jx.Operator(V, "hyperelastic", (mu, lam))
    from jaxiga_b200.newton import _external_loads

    f_ext = _external_loads(problem, params, op).cpu().numpy()
    u_o, st_o = H.newton(M, pres, vals, f_ext)
    assert st_o["converged"]
    assert np.abs(sol.u - u_o).max() <= 1e-8 * np.abs(u_o).max()
    # the residual at the solution, by the oracle, is at the tolerance
    free = np.setdiff1d(np.arange(V.n_dofs), pres)
    assert np.linalg.norm((M.residual(sol.u) - f_ext)[free]) <= 1e-8
    op.close()
    del torch


def test_a_failed_newton_solve_reports_it():
    """A displacement that inverts elements: Newton stalls or reports a
    non-finite state, with a warning, as the reference's diagnostics do."""
    V = jx.FunctionSpace(jx.primitives.rectangle(0, 0, 1, 1).elevate(2).refine(1), vec=2)
    problem = jx.Hyperelasticity(V, dirichlet=[jx.DirichletBC([0.0, 0.0], where="bottom"),
                                               jx.DirichletBC([0.0, -1.5], where="top")])
    with pytest.warns(RuntimeWarning, match="Newton did not reach"):
        sol = jx.solve(problem, params={"mu": 1.0, "lam": 1.0}, max_steps=3)
    assert not sol.stats["converged"]
