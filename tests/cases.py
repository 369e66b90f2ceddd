"""The golden cases, built through the product API and through the oracle.

Each case mirrors one block of tests/golden/make_golden.py: the same geometry
construction, boundary conditions, coefficients and source, so the GPU path,
the oracle and the reference fixtures are compared on identical inputs.
"""

from __future__ import annotations

import os

import numpy as np

import jaxiga_b200 as jx

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")
_cache = {}


def golden():
    if "g" not in _cache:
        _cache["g"] = np.load(GOLDEN)
    return _cache["g"]


ALL = lambda x: np.full(x.shape[0], True)  # noqa: E731
PLATE = {"E": 12 * (1 - 0.3**2), "nu": 0.3, "t": 1.0}


def build(tag):
    """(space, problem, params, source_kind) through the product API."""
    g = golden()
    P = jx.primitives
    if tag == "poisson2d":
        V = jx.FunctionSpace(P.quadrilateral([[0, 0], [1, 0], [1, 1], [0, 1]]).elevate(3).refine(5))
        f = lambda x, p: 8 * np.pi**2 * np.sin(2 * np.pi * x[0]) * np.sin(2 * np.pi * x[1])  # noqa: E731
        return V, jx.Poisson(V, dirichlet=[jx.DirichletBC(0.0, where=ALL)], source=f), {"a0": 1.0}
    if tag == "patch2d":
        V = jx.FunctionSpace(P.quadrilateral([[0, 0], [1, 0], [1, 1], [0, 1]]).elevate(2).refine(2))
        bc = jx.DirichletBC(lambda x, p: 1.0 + 2.0 * x[0] - 3.0 * x[1], where=ALL)
        return V, jx.Poisson(V, dirichlet=[bc], source=lambda x, p: 0.0), {"a0": 1.0}
    if tag == "annulus2d":
        kn = np.linspace(0, 1, 9)[1:-1]
        V = jx.FunctionSpace(P.quarter_annulus(1.0, 2.0).elevate(3).insert_knots(kn, kn))
        bcs = [jx.DirichletBC(0.0, where=s) for s in ("inner", "outer", "sym_y", "sym_x")]
        return V, jx.Poisson(V, dirichlet=bcs, source=lambda x, p: p["f"]), {"a0": float(g["annulus2d/a0"])}
    if tag == "elast3d":
        kn = np.linspace(0, 1, 5)[1:-1]
        V = jx.FunctionSpace(P.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kn), vec=3)
        pr = jx.LinearElasticity(V, dirichlet=[jx.DirichletBC([0.0, 0.0, 0.0], where="left")],
                                 source=lambda x, p: p["f"])
        return V, pr, {"E": 1.0, "nu": 0.3}
    if tag == "darcy3d":
        kn = np.linspace(0, 1, 6)[1:-1]
        V = jx.FunctionSpace(P.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kn))
        return V, jx.Poisson(V, dirichlet=[jx.DirichletBC(0.0, where=ALL)], source=lambda x, p: 1.0), {}
    if tag == "plate2d":
        kn = np.linspace(0, 1, 9)[1:-1]
        V = jx.FunctionSpace(P.rectangle(0, 0, 1, 1).elevate(4).insert_knots(kn, kn))
        bcs = [jx.ClampedBC(where=s) for s in ("left", "right", "bottom", "top")]
        return V, jx.KirchhoffPlate(V, dirichlet=bcs, source=lambda x, p: 1.0), dict(PLATE)
    raise KeyError(tag)


def with_fields(tag, V, params, interpolate):
    """Add the PointField inputs (interpolated control-point fields) to params.

    ``interpolate(coef) -> (n_elem, n_q, ncomp)`` evaluates sum_i R_i c_i at the
    Gauss points (the device kernel on the GPU, the oracle on the CPU).
    """
    g = golden()
    params = dict(params)
    if tag == "annulus2d":
        params["f"] = jx.PointField(interpolate(g["annulus2d/source_coef"])[..., 0])
    elif tag == "elast3d":
        params["f"] = jx.PointField(interpolate(g["elast3d/eta"]) + np.array([0.0, 0.0, -1.0]))
    elif tag == "darcy3d":
        params["a0"] = jx.PointField(np.exp(interpolate(g["darcy3d/loga"])[..., 0]))
    return params


CASES = ["poisson2d", "patch2d", "annulus2d", "elast3d", "darcy3d", "plate2d"]
OPS = {"poisson2d": "poisson", "patch2d": "poisson", "annulus2d": "poisson", "elast3d": "elasticity",
       "darcy3d": "poisson", "plate2d": "plate"}


def make_operator_oracle(tag):
    """The oracle's assembled free-free operator of a golden case (no per-point fields)."""
    from oracle import iga_oracle as O

    V, problem, params = build(tag)
    pres, vals = problem.resolve_dirichlet(params)
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec)
    coef, field = problem.operator_coefficients(params)
    if field is not None:
        raise ValueError(f"{tag} has a per-point coefficient")
    names = {"poisson": ("a0",), "elasticity": ("E", "nu"), "plate": ("E", "nu", "t")}[OPS[tag]]
    return O.Assembled(S, OPS[tag], dict(zip(names, coef)), pres, vals, need_full=False)
