"""Post-processing on the device against the oracle: gradients at the Gauss
points (Solution.grad), evaluation at arbitrary reference points of a
PointSet (Solution.at / grad on any point set, src/jaxiga/post/solution.py:39-54),
and the L2 / H1 / energy error norms and the H1 norm (src/jaxiga/post/norms.py:43-140)."""

from __future__ import annotations

import numpy as np
import pytest
from cases import build, with_fields

import jaxiga_b200 as jx
from jaxiga_b200.solve import geometry_operator
from oracle import iga_oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def _oracle_space(V):
    return O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec)


def _field(S, rng):
    return rng.standard_normal((S.n_scalar, S.vec))


@pytest.mark.parametrize("tag", ["annulus2d", "elast3d", "plate2d"])
def test_gradients_at_gauss_points_match_oracle(tag):
    V, _, _ = build(tag)
    S = _oracle_space(V)
    c = _field(S, np.random.default_rng(3))
    g = geometry_operator(V).interpolate_grad(c.reshape(-1)).cpu().numpy()
    el = np.arange(S.n_elems)
    basis = O.evaluate(S, el)
    ref = np.einsum("eqdn,enc->eqcd", basis["dR"], c[basis["dofs"]])
    assert g.shape == ref.shape
    assert _rel(g, ref) < 1e-12


@pytest.mark.parametrize("tag", ["annulus2d", "darcy3d", "elast3d"])
def test_eval_points_match_oracle(tag):
    V, _, _ = build(tag)
    S = _oracle_space(V)
    rng = np.random.default_rng(11)
    c = _field(S, rng)
    elems = rng.choice(S.n_elems, size=min(S.n_elems, 24), replace=False)
    ref = rng.uniform(-1.0, 1.0, size=(5, S.dim))
    ref[0] = -1.0  # element corner: the knot itself
    ps = jx.PointSet(elems=elems, ref=ref)
    e_flat, r_flat = ps.flat()
    out = geometry_operator(V).eval_points(e_flat, r_flat, c.reshape(-1), val=True, grad=True, x=True, jac=True)
    basis = O.evaluate(S, elems, ref=ref)
    val = np.einsum("eqn,enc->eqc", basis["R"], c[basis["dofs"]]).reshape(-1, S.vec)
    grad = np.einsum("eqdn,enc->eqcd", basis["dR"], c[basis["dofs"]]).reshape(-1, S.vec, S.dim)
    assert _rel(out["val"].cpu().numpy(), val) < 1e-12
    assert _rel(out["grad"].cpu().numpy(), grad) < 1e-12
    assert _rel(out["x"].cpu().numpy(), basis["x"].reshape(-1, S.dim)) < 1e-13
    assert _rel(out["jac"].cpu().numpy(), basis["w"].reshape(-1)) < 1e-12  # unit reference weights


def test_point_set_on_the_gauss_rule_equals_the_gauss_kernels():
    V, problem, params = build("poisson2d")
    sol = jx.solve(problem, params=params, linear=jx.LinearOptions(tol=1e-12))
    ps = jx.gauss(V)
    assert _rel(sol.at(ps), sol.at()) < 1e-13
    assert _rel(sol.grad(ps), sol.grad()) < 1e-12


def test_out_of_range_element_gives_nan():
    V, _, _ = build("poisson2d")
    out = geometry_operator(V).eval_points([0, V.n_elems], [[0.0, 0.0], [0.0, 0.0]], np.ones(V.n_scalar_basis),
                                           x=True, jac=True)
    v = out["val"].cpu().numpy()
    assert np.isfinite(v[0]).all() and np.isnan(v[1]).all()


def _sin(x):
    return np.sin(2 * np.pi * x[:, 0]) * np.sin(2 * np.pi * x[:, 1])


def _sin_grad(x):
    s, c = np.sin(2 * np.pi * x), np.cos(2 * np.pi * x)
    return (2 * np.pi * np.stack([c[:, 0] * s[:, 1], s[:, 0] * c[:, 1]], axis=1))[:, None, :]


def test_h1_error_matches_oracle_and_converges():
    errs = []
    for r in (4, 5):
        V = jx.FunctionSpace(jx.primitives.quadrilateral([[0, 0], [1, 0], [1, 1], [0, 1]]).elevate(3).refine(r))
        f = lambda x, p: 8 * np.pi**2 * np.sin(2 * np.pi * x[0]) * np.sin(2 * np.pi * x[1])  # noqa: E731
        pr = jx.Poisson(V, dirichlet=[jx.DirichletBC(0.0, where=lambda x: np.full(len(x), True))], source=f)
        sol = jx.solve(pr, params={"a0": 1.0}, linear=jx.LinearOptions(tol=1e-13))
        h1 = jx.errornorm(sol, _sin, "H1", exact_grad=_sin_grad)
        # oracle: the same u on the same Gauss set
        S = _oracle_space(V)
        b = O.evaluate(S, np.arange(S.n_elems))
        gh = np.einsum("eqdn,en->eqd", b["dR"], sol.u[b["dofs"]]).reshape(-1, 2)
        ge = _sin_grad(b["x"].reshape(-1, 2))[:, 0]
        w = b["w"].reshape(-1)
        ref = np.sqrt(np.sum(w * np.sum((gh - ge) ** 2, -1)) / np.sum(w * np.sum(ge**2, -1)))
        assert abs(h1 - ref) < 1e-10 * ref
        # a finer Gauss rule through the point-set path agrees to quadrature accuracy
        h1q = jx.errornorm(sol, _sin, "H1", exact_grad=_sin_grad, quad=6)
        assert abs(h1q - h1) < 1e-3 * h1
        errs.append(h1)
    rate = np.log2(errs[0] / errs[1])
    assert rate > 3 - 0.5, rate  # H1 rate p for p = 3 (the L2 rate test is tests/test_galerkin.py:59-65)


def test_energy_norm_matches_oracle():
    V, problem, params = build("elast3d")
    params = with_fields("elast3d", V, params, lambda c: geometry_operator(V).interpolate(c).cpu().numpy())
    sol = jx.solve(problem, params=params, linear=jx.LinearOptions(tol=1e-12))
    C = problem.C(params)

    def exact(x):
        return np.stack([0.01 * x[:, 0] ** 2, 0.02 * x[:, 0] * x[:, 1], -0.01 * x[:, 2]], axis=1)

    def stress(x):
        g = np.zeros((len(x), 3, 3))
        g[:, 0, 0] = 0.02 * x[:, 0]
        g[:, 1, 0] = 0.02 * x[:, 1]
        g[:, 1, 1] = 0.02 * x[:, 0]
        g[:, 2, 2] = -0.01
        eps = np.stack([g[:, 0, 0], g[:, 1, 1], g[:, 2, 2], g[:, 1, 2] + g[:, 2, 1], g[:, 0, 2] + g[:, 2, 0],
                        g[:, 0, 1] + g[:, 1, 0]], axis=1)
        return eps @ C.T

    en = jx.errornorm(sol, exact, "energy", exact_grad=stress)
    S = _oracle_space(V)
    b = O.evaluate(S, np.arange(S.n_elems))
    B = O.strain_displacement(b["dR"])
    ue = sol.u[S.expand(b["dofs"])]
    sh = np.einsum("st,eqtj,ej->eqs", C, B, ue).reshape(-1, 6)
    se = stress(b["x"].reshape(-1, 3))
    Ci = np.linalg.inv(C)
    w = b["w"].reshape(-1)
    d = sh - se
    ref = np.sqrt(np.sum(w * np.einsum("ni,ij,nj->n", d, Ci, d)) / np.sum(w * np.einsum("ni,ij,nj->n", se, Ci, se)))
    assert abs(en - ref) < 1e-10 * ref
    with pytest.raises(ValueError, match="constitutive"):
        p2d, pr2d, pa2d = build("poisson2d")
        s2 = jx.solve(pr2d, params=pa2d)
        jx.errornorm(s2, _sin, "energy", exact_grad=_sin_grad)


def test_h1_norm_and_integrate_with_quad():
    V, problem, params = build("annulus2d")
    params = with_fields("annulus2d", V, params, lambda c: geometry_operator(V).interpolate(c).cpu().numpy())
    sol = jx.solve(problem, params=params, linear=jx.LinearOptions(tol=1e-12))
    S = _oracle_space(V)
    b = O.evaluate(S, np.arange(S.n_elems))
    u = np.einsum("eqn,en->eq", b["R"], sol.u[b["dofs"]])
    g = np.einsum("eqdn,en->eqd", b["dR"], sol.u[b["dofs"]])
    ref = np.sqrt(np.sum(b["w"] * (u**2 + np.sum(g**2, -1))))
    assert abs(jx.norm(sol, "H1") - ref) < 1e-11 * ref
    # annulus area pi/4 (r_o^2 - r_i^2) = 3 pi / 4, tests/test_evaluation.py:32-36 of the reference
    for q in (None, 5, 7):
        assert abs(jx.integrate(lambda x: np.ones(len(x)), V, quad=q) - 0.75 * np.pi) < 1e-12
