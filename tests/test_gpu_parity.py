"""Parity of the CUDA path (through the libjxb C ABI) with the reference fixtures and the oracle.

Tolerances: operator quantities (K.v, diag K, load vector, Gauss-point
geometry) agree with the reference to 1e-12 relative (FP64, different
summation order); solutions to 1e-10 relative L2 (the FP64 bar); CG
iteration counts with the oracle's restatement of jax's CG to +-1.
"""

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200.solve import geometry_operator, qp_points
from oracle import iga_oracle as O
from tests.cases import CASES, OPS, build, golden, with_fields

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def device_interp(V):
    geo = geometry_operator(V)
    return lambda c: geo.interpolate(c).cpu().numpy()


def source_qp(tag, V, params):
    x = qp_points(V)
    n = x.shape[0]
    if tag == "poisson2d":
        return 8 * np.pi**2 * np.sin(2 * np.pi * x[:, 0]) * np.sin(2 * np.pi * x[:, 1])
    if tag == "patch2d":
        return np.zeros(n)
    if tag in ("annulus2d", "elast3d"):
        return np.asarray(params["f"].values).reshape(n, -1)
    return np.ones(n)


def make_operator(tag):
    V, problem, params = build(tag)
    params = with_fields(tag, V, params, device_interp(V))
    pres, vals = problem.resolve_dirichlet(params)
    mask = np.zeros(V.n_dofs, bool)
    mask[pres] = True
    coef, field = problem.operator_coefficients(params)
    coef_qp = None if field is None else np.asarray(field.values)
    op = jx.Operator(V, OPS[tag], coef, prescribed=mask, coef_qp=coef_qp)
    return V, problem, params, op, pres, vals


@pytest.mark.parametrize("tag", CASES)
def test_dirichlet_partition_matches_reference(tag):
    g = golden()
    V, problem, params = build(tag)
    pres, vals = problem.resolve_dirichlet(params)
    np.testing.assert_array_equal(pres, g[f"{tag}/prescribed"])
    np.testing.assert_allclose(vals, g[f"{tag}/prescribed_values"], rtol=0, atol=1e-14)


@pytest.mark.parametrize("tag", CASES)
def test_operator_matches_reference(tag):
    g = golden()
    V, problem, params, op, pres, vals = make_operator(tag)
    free = np.setdiff1d(np.arange(V.n_dofs), pres)
    x = np.full(V.n_dofs, 123.0)  # prescribed entries must be ignored by the masked operator
    x[free] = g[f"{tag}/v"]
    y = op.apply(x).cpu().numpy()
    assert rel(y[free], g[f"{tag}/Kv"]) < 1e-12
    assert np.all(y[pres] == 0.0)
    d = op.diag().cpu().numpy()
    assert rel(d[free], g[f"{tag}/diag"]) < 1e-12
    F = op.load(source_qp(tag, V, params)).cpu().numpy()
    assert rel(F, g[f"{tag}/load_F"]) < 1e-12
    sample = g[f"{tag}/sample"]
    xq = op.qp_coords().cpu().numpy()[sample]
    np.testing.assert_allclose(xq, g[f"{tag}/basis_x"], rtol=0, atol=1e-14)
    w = op.qp_weights().cpu().numpy()
    np.testing.assert_allclose(w[sample], g[f"{tag}/basis_w"], rtol=1e-13, atol=1e-18)
    assert abs(w.sum() - float(g[f"{tag}/wsum"])) < 1e-12 * abs(float(g[f"{tag}/wsum"]))
    op.close()


@pytest.mark.parametrize("tag", CASES)
def test_solve_matches_reference(tag):
    g = golden()
    V, problem, params = build(tag)
    params = with_fields(tag, V, params, device_interp(V))
    sol = jx.solve(problem, params=params, linear=jx.LinearOptions(tol=1e-13))
    # 1e-13 is at the attainable accuracy of FP64 CG for these problems: the
    # recursive residual meets it, the recomputed true residual may land a few
    # percent above (then the stats report converged = False, as the reference's
    # diagnostics would); the check that matters is the solution's
    assert sol.stats["finite"] and sol.stats["relative_residual"] < 2e-13
    assert rel_l2(sol.u, g[f"{tag}/u"]) < 1e-10
    # energy u_f^T K_ff u_f of the discrete solution
    free = np.setdiff1d(np.arange(V.n_dofs), g[f"{tag}/prescribed"])
    geo = jx.Operator(V, OPS[tag], problem.operator_coefficients(params)[0],
                      prescribed=np.isin(np.arange(V.n_dofs), g[f"{tag}/prescribed"]),
                      coef_qp=None if problem.operator_coefficients(params)[1] is None
                      else np.asarray(problem.operator_coefficients(params)[1].values))
    uf = np.zeros(V.n_dofs)
    uf[free] = sol.u[free]
    energy = float(uf @ geo.apply(uf).cpu().numpy())
    assert abs(energy - float(g[f"{tag}/energy"])) < 1e-10 * abs(float(g[f"{tag}/energy"]))
    geo.close()


def test_poisson_error_norm_matches_reference():
    g = golden()
    V, problem, params = build("poisson2d")
    sol = jx.solve(problem, params=params, linear=jx.LinearOptions(tol=1e-13))
    exact = lambda x: np.sin(2 * np.pi * x[:, 0]) * np.sin(2 * np.pi * x[:, 1])  # noqa: E731
    err = jx.errornorm(sol, exact, "L2")
    assert abs(err - float(g["poisson2d/errornorm_L2"])) < 1e-8 * float(g["poisson2d/errornorm_L2"])


def test_patch_test_reproduces_linear_field():
    """tests/test_galerkin.py:35-47 of the reference: a field in the space is recovered exactly."""
    V, problem, params = build("patch2d")
    sol = jx.solve(problem, params=params, linear=jx.LinearOptions(tol=1e-14))
    assert jx.errornorm(sol, lambda x: 1.0 + 2.0 * x[:, 0] - 3.0 * x[:, 1], "L2") < 1e-12


@pytest.mark.parametrize("tag", ["poisson2d", "annulus2d", "elast3d", "darcy3d", "plate2d"])
def test_pcg_iterations_match_jax_cg(tag):
    """Same operator, same Jacobi preconditioner, same stopping rule -> same CG history."""
    g = golden()
    V, problem, params, op, pres, vals = make_operator(tag)
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec)
    coef, field = problem.operator_coefficients(params)
    names = {"poisson": ("a0",), "elasticity": ("E", "nu"), "plate": ("E", "nu", "t")}[OPS[tag]]
    oparams = dict(zip(names, coef))
    if field is not None:
        oparams["a0_qp"] = np.asarray(field.values)
    A = O.Assembled(S, OPS[tag], oparams, pres, vals, need_full=False)
    b = g[f"{tag}/rhs"]
    tol = 1e-10
    x_o, k_o = O.jax_cg(lambda v: A.K @ v, b, tol, inv_diag=O.jacobi_inverse(A.diag))
    bf = np.zeros(V.n_dofs)
    bf[A.free] = b
    x, st = op.pcg(bf, tol=tol, preconditioner="jacobi")
    assert abs(st["iterations"] - k_o) <= 1, (st["iterations"], k_o)
    assert rel_l2(x.cpu().numpy()[A.free], x_o) < 1e-7
    op.close()


def test_apply_and_pcg_are_bitwise_deterministic():
    V, problem, params, op, pres, vals = make_operator("elast3d")
    rng = np.random.default_rng(7)
    x = rng.standard_normal(V.n_dofs)
    y1 = op.apply(x).cpu().numpy()
    y2 = op.apply(x).cpu().numpy()
    assert np.array_equal(y1, y2)
    s1, _ = op.pcg(x, tol=1e-8)
    s2, _ = op.pcg(x, tol=1e-8)
    assert np.array_equal(s1.cpu().numpy(), s2.cpu().numpy())
    op.close()
