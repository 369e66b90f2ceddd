"""Operator parity at the full sizes of the benchmark workloads.

The golden fixtures are small (4^3 .. 8^2 elements). Here the device K.u,
diag K and load vector of the full-size workloads -- 3D elasticity 64^3
(902,289 DOFs), Darcy 96^3 with its Gaussian-random-field coefficient
(970,299 DOFs) and the clamped plate 256^2 (67,600 DOFs) -- are compared on
a seeded sample of control points with the oracle: the NumPy restatement of
evaluation.py / library.py evaluated on exactly the elements that support
those points, so each sampled row of K.u is complete. This is the
matrix-free-against-assembled check of the reference's
tests/test_advanced.py:123-132 (relative difference below 1e-12), taken at
the benchmark sizes instead of fixture sizes.
"""

from __future__ import annotations

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200 import workloads
from jaxiga_b200.solve import geometry_operator
from oracle import iga_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _control_index(S, i):
    """Per-direction indices of scalar control point i (first direction fastest)."""
    out = []
    for n in S.n_cp:
        out.append(i % n)
        i //= n
    return out


def _support(S, i):
    """Elements (first direction fastest) whose span has basis function i."""
    idx = _control_index(S, int(i))
    per_dir = []
    for d in range(S.dim):
        first = S.spans[d][2]
        per_dir.append(np.nonzero((first <= idx[d]) & (idx[d] <= first + S.degree[d]))[0])
    strides = np.array([1, *np.cumprod(S.n_span[:-1])])
    mesh = np.meshgrid(*per_dir, indexing="ij")
    return sum(m.ravel() * strides[d] for d, m in enumerate(mesh))


def _sample_points(S, rng, n, margin):
    """n distinct scalar control points at least ``margin`` layers from every
    face (so that every component is free under the workloads' conditions)."""
    lo = [margin] * S.dim
    hi = [S.n_cp[d] - 1 - margin for d in range(S.dim)]
    idx = [rng.integers(lo[d], hi[d] + 1, size=4 * n) for d in range(S.dim)]
    strides = np.array([1, *np.cumprod(S.n_cp[:-1])])
    pts = np.unique(sum(idx[d] * strides[d] for d in range(S.dim)))
    return rng.permutation(pts)[:n]


def _oracle_rows(S, op, params_of, x, pts, source_of=None, chunk=256):
    """K x, diag K and the load vector, complete on the rows of ``pts``.

    params_of(elems, basis) -> element-tangent parameters of those elements;
    source_of(elems, basis) -> source values (n_e, n_q, vec) or None.
    """
    vec = S.vec
    elems = np.unique(np.concatenate([_support(S, i) for i in pts]))
    y = np.zeros(S.n_dofs)
    d = np.zeros(S.n_dofs)
    F = np.zeros(S.n_dofs)
    order = 2 if op == "plate" else 1
    for lo in range(0, len(elems), chunk):
        el = elems[lo:lo + chunk]
        basis = O.evaluate(S, el, order=order)
        Ke = O.element_tangents(op, basis, params_of(el, basis), vec)
        gd = S.expand(S.elem_dofs[el])
        np.add.at(y, gd, np.einsum("eij,ej->ei", Ke, x[gd]))
        np.add.at(d, gd, np.diagonal(Ke, axis1=1, axis2=2))
        if source_of is not None:
            fq = source_of(el, basis)
            Fe = np.einsum("eq,eqc,eqi->eic", basis["w"], fq, basis["R"]).reshape(len(el), -1)
            np.add.at(F, gd, Fe)
    rows = S.expand(np.asarray(pts)[None, :])[0]
    return y[rows], d[rows], F[rows], rows, len(elems)


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def _operator(V, problem, params, op_name, coef, coef_qp=None):
    pres, vals = problem.resolve_dirichlet(params)
    mask = np.zeros(V.n_dofs, bool)
    mask[pres] = True
    return jx.Operator(V, op_name, coef, prescribed=mask, coef_qp=coef_qp), mask


def test_elasticity_64_matches_oracle_on_sampled_rows():
    V, problem, params = workloads.config2(n=64)
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 3)
    op, mask = _operator(V, problem, params, "elasticity", (1.0, 0.3))
    rng = np.random.default_rng([20260901, 102])
    x = rng.standard_normal(V.n_dofs)
    xm = np.where(mask, 0.0, x)
    eta = params["eta"]
    fq_dev = geometry_operator(V).interpolate(eta)
    fq_dev[..., 2] -= 1.0
    y_dev = op.apply(x).cpu().numpy()
    d_dev = op.diag().cpu().numpy()
    F_dev = op.load(fq_dev).cpu().numpy()
    pts = _sample_points(S, rng, 40, margin=1)

    def source_of(el, basis):
        return np.einsum("eqn,enc->eqc", basis["R"], eta[S.elem_dofs[el]]) + np.array([0.0, 0.0, -1.0])

    y, d, F, rows, n_el = _oracle_rows(S, "elasticity", lambda el, b: {"E": 1.0, "nu": 0.3}, xm, pts, source_of)
    assert n_el > 1000
    assert _rel(y_dev[rows], y) < TOL
    assert _rel(d_dev[rows], d) < TOL
    assert _rel(F_dev[rows], F) < TOL
    op.close()


def test_darcy_96_matches_oracle_on_sampled_rows():
    V, problem, params = workloads.config4(n=96)
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 1)
    loga = params["loga"]
    a_qp = np.exp(geometry_operator(V).interpolate(loga)[..., 0].cpu().numpy())
    op, mask = _operator(V, problem, params, "poisson", (1.0,), coef_qp=a_qp)
    rng = np.random.default_rng([20260901, 104])
    x = rng.standard_normal(V.n_dofs)
    xm = np.where(mask, 0.0, x)
    y_dev = op.apply(x).cpu().numpy()
    d_dev = op.diag().cpu().numpy()
    nq = a_qp.shape[1]
    F_dev = op.load(np.ones(V.n_elems * nq)).cpu().numpy()
    pts = _sample_points(S, rng, 48, margin=1)
    coef_err = []

    def params_of(el, basis):
        # the coefficient at the Gauss points from the oracle's own interpolation
        a = np.exp(np.einsum("eqn,en->eq", basis["R"], loga[S.elem_dofs[el]]))
        coef_err.append(_rel(a_qp[el], a))
        return {"a0": a}

    y, d, F, rows, n_el = _oracle_rows(S, "poisson", params_of, xm, pts,
                                       lambda el, b: np.ones(b["w"].shape + (1,)))
    assert n_el > 1000
    assert max(coef_err) < TOL
    assert _rel(y_dev[rows], y) < TOL
    assert _rel(d_dev[rows], d) < TOL
    assert _rel(F_dev[rows], F) < TOL
    op.close()


def test_plate_256_matches_oracle_on_sampled_rows():
    V, problem, params = workloads.config5(n=256)
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 1)
    coef = problem.operator_coefficients(params)[0]
    op, mask = _operator(V, problem, params, "plate", coef)
    rng = np.random.default_rng([20260901, 105])
    x = rng.standard_normal(V.n_dofs)
    xm = np.where(mask, 0.0, x)
    y_dev = op.apply(x).cpu().numpy()
    d_dev = op.diag().cpu().numpy()
    F_dev = op.load(np.ones(V.n_elems * 25)).cpu().numpy()
    pts = _sample_points(S, rng, 200, margin=2)
    y, d, F, rows, n_el = _oracle_rows(S, "plate", lambda el, b: dict(params), xm, pts,
                                       lambda el, b: np.ones(b["w"].shape + (1,)))
    assert n_el > 2000
    assert _rel(y_dev[rows], y) < TOL
    assert _rel(d_dev[rows], d) < TOL
    assert _rel(F_dev[rows], F) < TOL
    op.close()
