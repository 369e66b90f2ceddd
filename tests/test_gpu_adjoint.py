"""Gradients through the device solve: one forward and one adjoint solve
(src/jaxiga/solvers/linear.py:360-389, 414-442), checked against central
finite differences of the solve, and the solve counters of the reference's
tests/test_galerkin.py:264-274."""

from __future__ import annotations

import numpy as np
import pytest
from cases import build, with_fields

import jaxiga_b200 as jx
from jaxiga_b200.solve import geometry_operator

pytestmark = pytest.mark.gpu

LIN = jx.LinearOptions(tol=1e-13)


def _sq(u):
    return 0.5 * float(u @ u), u


def _J(problem, params):
    return _sq(jx.solve(problem, params=params, linear=LIN).u)[0]


def _fd(problem, params, name, h):
    p1, p2 = dict(params), dict(params)
    p1[name] = params[name] * (1 + h)
    p2[name] = params[name] * (1 - h)
    return (_J(problem, p1) - _J(problem, p2)) / (2 * h * params[name])


def test_poisson_a0_gradient_with_one_adjoint_solve():
    # nonzero Dirichlet data: the lift K_fp g depends on a0 too
    V = jx.FunctionSpace(jx.primitives.quadrilateral([[0, 0], [1, 0], [1, 1], [0, 1]]).elevate(2).refine(3))
    bc = jx.DirichletBC(lambda x, p: 1.0 + x[0] * x[1], where=lambda x: np.full(len(x), True))
    pr = jx.Poisson(V, dirichlet=[bc], source=lambda x, p: np.sin(3 * x[0]))
    params = {"a0": 1.7}
    jx.reset_solve_counter()
    J, g, sol = jx.value_and_grad(pr, params, _sq, ["a0"], linear=LIN)
    assert jx.SOLVE_COUNTER == {"forward": 1, "adjoint": 1}
    fd = _fd(pr, params, "a0", 1e-5)
    assert abs(g["a0"] - fd) < 1e-6 * abs(fd), (g["a0"], fd)


def test_pointfield_coefficient_gradient_matches_directional_difference():
    V, problem, params = build("darcy3d")
    interp = lambda c: geometry_operator(V).interpolate(c).cpu().numpy()  # noqa: E731
    params = with_fields("darcy3d", V, params, interp)
    a = np.asarray(params["a0"].values)
    J, g, _ = jx.value_and_grad(problem, params, _sq, ["a0"], linear=LIN)
    assert g["a0"].shape == a.shape
    d = np.random.default_rng(5).standard_normal(a.shape) * a
    h = 1e-6
    Jp = _J(problem, {**params, "a0": jx.PointField(a + h * d)})
    Jm = _J(problem, {**params, "a0": jx.PointField(a - h * d)})
    fd = (Jp - Jm) / (2 * h)
    assert abs(float(np.sum(g["a0"] * d)) - fd) < 1e-6 * abs(fd)


def test_elasticity_E_nu_gradients():
    V, problem, params = build("elast3d")
    params = with_fields("elast3d", V, params, lambda c: geometry_operator(V).interpolate(c).cpu().numpy())
    jx.reset_solve_counter()
    J, g, _ = jx.value_and_grad(problem, params, _sq, ["E", "nu"], linear=LIN)
    assert jx.SOLVE_COUNTER == {"forward": 1, "adjoint": 1}
    for name in ("E", "nu"):
        fd = _fd(problem, params, name, 1e-5)
        assert abs(g[name] - fd) < 1e-6 * abs(fd), (name, g[name], fd)


def test_plate_E_t_gradients():
    V, problem, params = build("plate2d")
    J, g, _ = jx.value_and_grad(problem, params, _sq, ["E", "t"], linear=LIN)
    for name in ("E", "t"):
        fd = _fd(problem, params, name, 1e-5)
        assert abs(g[name] - fd) < 1e-6 * abs(fd), (name, g[name], fd)
    with pytest.raises(NotImplementedError):
        jx.value_and_grad(problem, params, _sq, ["nu"], linear=LIN)
