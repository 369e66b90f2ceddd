"""Neumann loads on the device against the oracle, and the reference's
pressure-loaded thick cylinder (Lame) solved end to end
(tests/test_examples.py:22-60 of the reference)."""

from __future__ import annotations

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200.neumann import boundary_points, neumann_load, resolve_set
from jaxiga_b200.pointset import boundary_gauss
from oracle import iga_oracle as O

pytestmark = pytest.mark.gpu


def _annulus(vec=1):
    return jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 4.0).elevate(3).refine(3), vec=vec)


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("label", ["inner", "outer", "sym_x"])
def test_boundary_points_match_oracle(label):
    V = _annulus()
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 1)
    op = jx.Operator(V, "poisson", (1.0,))
    ps = boundary_gauss(V, V.boundary(label))
    x, n, w, _ = boundary_points(op, ps)
    b = O.evaluate_boundary(S, ps.elems, ps.sides, ps.ref, ps.weights)
    assert _rel(x.cpu().numpy(), b["x"].reshape(-1, 2)) < 1e-14
    assert np.abs(n.cpu().numpy() - b["normal"].reshape(-1, 2)).max() < 1e-13
    assert _rel(w.cpu().numpy(), b["w"].reshape(-1)) < 1e-13
    op.close()


def test_traction_load_matches_oracle_2d_and_3d():
    # 2D elasticity, pressure on the inner arc plus a shear on the outer arc
    V = _annulus(vec=2)
    pr = jx.LinearElasticity(V, neumann=[jx.Neumann(lambda x, n, p: -p["q"] * n, where="inner"),
                                         jx.Neumann(lambda x, n, p: np.stack([-n[:, 1], n[:, 0]], 1) * x[:, :1],
                                                    where="outer")])
    params = {"E": 1.0, "nu": 0.3, "q": 2.5}
    op = jx.Operator(V, "elasticity", (1.0, 0.3))
    F = neumann_load(op, pr, params).cpu().numpy()
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 2)
    ref = np.zeros(V.n_dofs)
    for bc, label in zip(pr.neumann, ("inner", "outer")):
        ps = boundary_gauss(V, V.boundary(label))
        ref += O.neumann_load(S, ps.elems, ps.sides, ps.ref, ps.weights, lambda x, n, bc=bc: bc.value(x, n, params))
    assert _rel(F, ref) < 1e-13
    op.close()
    # 3D: a flux on the elements of the x = 1 face selected by a predicate on side centres
    kn = np.linspace(0, 1, 4)[1:-1]
    V3 = jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(2).insert_knots(kn, kn, kn))
    pred = lambda c: np.isclose(c[:, 0], 1.0) & (c[:, 1] < 0.4)  # noqa: E731
    pr3 = jx.Poisson(V3, neumann=[jx.Neumann(lambda x, n, p: np.sin(x[:, 1:2]) * n[:, :1], where=pred)])
    op3 = jx.Operator(V3, "poisson", (1.0,))
    F3 = neumann_load(op3, pr3, {}).cpu().numpy()
    bset = resolve_set(V3, pred)
    assert len(bset.elems) == 3  # of the 3 x 3 face elements, the row with centre y = 1/6
    S3 = O.Space(V3.knots, V3.degree, V3.cpts, V3.wgts, 1)
    ps = boundary_gauss(V3, bset)
    ref3 = O.neumann_load(S3, ps.elems, ps.sides, ps.ref, ps.weights, lambda x, n: np.sin(x[:, 1:2]) * n[:, :1])
    assert _rel(F3, ref3) < 1e-13
    op3.close()


def _lame(r_int=1.0, r_ext=4.0, pressure=10.0, E=1e5, nu=0.3):
    a2, b2 = r_int**2, r_ext**2

    def disp(pts):
        r, th = np.hypot(pts[:, 0], pts[:, 1]), np.arctan2(pts[:, 1], pts[:, 0])
        ur = pressure * a2 * r / (E * (b2 - a2)) * ((1 - nu) + (1 + nu) * b2 / r**2)
        return np.stack([ur * np.cos(th), ur * np.sin(th)], axis=1)

    def stress(pts):
        r, th = np.hypot(pts[:, 0], pts[:, 1]), np.arctan2(pts[:, 1], pts[:, 0])
        srr = pressure * a2 / (b2 - a2) * (1 - b2 / r**2)
        stt = pressure * a2 / (b2 - a2) * (1 + b2 / r**2)
        c, s = np.cos(th), np.sin(th)
        return np.stack([srr * c**2 + stt * s**2, srr * s**2 + stt * c**2, (srr - stt) * s * c], axis=1)

    return disp, stress


def test_pressurised_thick_cylinder_recovers_the_lame_solution():
    disp, stress = _lame()
    V = jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 4.0).elevate(4).refine(3), vec=2)
    pr = jx.LinearElasticity(V, plane="stress",
                             dirichlet=[jx.DirichletBC(0.0, where="sym_y", component=1),
                                        jx.DirichletBC(0.0, where="sym_x", component=0)],
                             neumann=[jx.Neumann(lambda x, n, p: -10.0 * n, where="inner")])
    sol = jx.solve(pr, params={"E": 1e5, "nu": 0.3})
    assert sol.stats["converged"]
    assert jx.errornorm(sol, disp, "L2") < 5e-5
    assert jx.errornorm(sol, disp, "energy", exact_grad=stress) < 5e-4
