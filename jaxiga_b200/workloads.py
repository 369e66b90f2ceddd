"""The benchmark workloads: seeded synthetic problems with the sizes, geometry
and value distributions of the five solver configurations.

Every draw uses ``numpy.random.default_rng([20260901, k])`` with ``k`` the
configuration index (1..5), so inputs are reproducible across machines.

  1  2D Poisson, unit square, cubic, 32 x 32 spans, f = 8 pi^2 sin sin, u = 0 on the boundary
  2  3D elasticity, unit cube, cubic, 64^3 spans, E = 1, nu = 0.3, x = 0 clamped,
     body force (0, 0, -1) + sum_i R_i eta_i with eta ~ N(0, 0.1^2) per control point
  3  (batched quarter annuli: see the batch module)
  4  3D Darcy, unit cube, cubic, 96^3 spans, a = exp(GRF) with a squared-exponential
     covariance (length 0.1, sigma 1) sampled exactly at the control points, f = 1, u = 0
  5  Kirchhoff plate, unit square, quartic, 256^2 spans, clamped edges, D = 1, nu = 0.3, q = 1
"""

from __future__ import annotations

import numpy as np

from .forms import ClampedBC, DirichletBC, KirchhoffPlate, LinearElasticity, PointField, Poisson
from .geometry import primitives
from .space import FunctionSpace

SEED = 20260901


def rng(k):
    return np.random.default_rng([SEED, k])


def _all(x):
    return np.full(x.shape[0], True)


def uniform_knots(n):
    return np.linspace(0.0, 1.0, n + 1)[1:-1]


def se_factor(x, length, sigma=1.0):
    """Factor L with L L^T = sigma^2 exp(-(x_i - x_j)^2 / (2 length^2)) (eigen, clipped)."""
    K = sigma**2 * np.exp(-((x[:, None] - x[None, :]) ** 2) / (2.0 * length**2))
    w, U = np.linalg.eigh(K)
    return U * np.sqrt(np.clip(w, 0.0, None))[None, :]


def grf_on_grid(axes, length, sigma, gen):
    """Exact sample of a separable squared-exponential GRF on a tensor grid.

    ``axes`` are the per-direction coordinates; the result is flattened first
    direction fastest (the control-point order).
    """
    Ls = [se_factor(a, length, sigma if d == 0 else 1.0) for d, a in enumerate(axes)]
    xi = gen.standard_normal([len(a) for a in axes[::-1]])  # axes reversed: last direction slowest
    out = xi
    for d, L in enumerate(Ls):
        axis = len(axes) - 1 - d
        out = np.moveaxis(np.tensordot(L, np.moveaxis(out, axis, 0), axes=(1, 0)), 0, axis)
    return out.reshape(-1)


def config1():
    V = FunctionSpace(primitives.quadrilateral([[0, 0], [1, 0], [1, 1], [0, 1]]).elevate(3).refine(5))
    f = lambda x, p: 8 * np.pi**2 * np.sin(2 * np.pi * x[0]) * np.sin(2 * np.pi * x[1])  # noqa: E731
    return V, Poisson(V, dirichlet=[DirichletBC(0.0, where=_all)], source=f), {"a0": 1.0}


def config2(n=64, interpolate=None):
    """3D elasticity; ``interpolate(coef)`` evaluates a control-point field at the Gauss points."""
    kn = uniform_knots(n)
    V = FunctionSpace(primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kn), vec=3)
    eta = rng(2).normal(0.0, 0.1, size=(V.n_scalar_basis, 3))
    problem = LinearElasticity(V, dirichlet=[DirichletBC([0.0, 0.0, 0.0], where="left")], source=lambda x, p: p["f"])
    params = {"E": 1.0, "nu": 0.3, "eta": eta}
    if interpolate is not None:
        params["f"] = PointField(interpolate(eta) + np.array([0.0, 0.0, -1.0]))
    return V, problem, params


def config3(n_instances=256, interpolate=None, span_range=(8, 128)):
    """Quarter annuli (inner radius 1, outer 2): degree ~ U{2,3,4}, spans per
    direction log-uniform in span_range, a0 ~ LogNormal(0, 0.5), source
    sum_k c_k R_k with c ~ N(0, 1) per control point, u = 0 on all four sides.

    Returns (problems, params_list); params carry the source coefficients
    ("c") and, with ``interpolate(space, coef)``, the source as a PointField.
    """
    g = rng(3)
    problems, params = [], []
    lo, hi = np.log(span_range[0]), np.log(span_range[1])
    for _ in range(n_instances):
        p = int(g.integers(2, 5))
        n = [int(round(np.exp(g.uniform(lo, hi)))) for _ in range(2)]
        a0 = float(g.lognormal(0.0, 0.5))
        patch = primitives.quarter_annulus(1.0, 2.0).elevate(p).insert_knots(uniform_knots(n[0]), uniform_knots(n[1]))
        V = FunctionSpace(patch)
        c = g.standard_normal(V.n_scalar_basis)
        bcs = [DirichletBC(0.0, where=s) for s in ("inner", "outer", "sym_y", "sym_x")]
        pr = Poisson(V, dirichlet=bcs, source=lambda x, pa: pa["f"])
        pa = {"a0": a0, "c": c}
        if interpolate is not None:
            pa["f"] = PointField(interpolate(V, c)[..., 0])
        problems.append(pr)
        params.append(pa)
    return problems, params


def config4(n=96, interpolate=None):
    kn = uniform_knots(n)
    V = FunctionSpace(primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kn))
    nx, ny, nz = V.n_cp
    axes = [V.cpts[:nx, 0], V.cpts[: nx * ny: nx, 1], V.cpts[:: nx * ny, 2]]
    loga = grf_on_grid(axes, 0.1, 1.0, rng(4))
    problem = Poisson(V, dirichlet=[DirichletBC(0.0, where=_all)], source=lambda x, p: 1.0)
    params = {"loga": loga}
    if interpolate is not None:
        params["a0"] = PointField(np.exp(interpolate(loga)[..., 0]))
    return V, problem, params


def config5(n=256):
    kn = uniform_knots(n)
    V = FunctionSpace(primitives.rectangle(0, 0, 1, 1).elevate(4).insert_knots(kn, kn))
    bcs = [ClampedBC(where=s) for s in ("left", "right", "bottom", "top")]
    return V, KirchhoffPlate(V, dirichlet=bcs, source=lambda x, p: 1.0), {"E": 12 * (1 - 0.3**2), "nu": 0.3, "t": 1.0}
