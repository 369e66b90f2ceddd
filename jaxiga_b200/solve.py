"""``solve(problem, method="galerkin", ...)`` on the B200 device path.

Mirrors ``src/jaxiga/methods/__init__.py:11-64`` (``solve``),
``src/jaxiga/methods/galerkin.py:275-357`` (``solve_galerkin``, linear branch),
``src/jaxiga/solvers/linear.py:76-127`` (``LinearOptions``) and
``src/jaxiga/post/norms.py`` (``errornorm``/``norm``).

The linear branch of ``solve_galerkin`` becomes:

  1. Dirichlet partition (problem.resolve_dirichlet);
  2. one device plan: per-point geometry factors, the masked operator;
  3. b = F - K_fp g  (load vector from the source at the Gauss points, minus
     the unconstrained operator applied to the lifted Dirichlet data);
  4. device Jacobi-PCG in FP64 (jax CG semantics), or FP64 iterative
     refinement around FP32 inner PCG when ``precision="mixed"``;
  5. the FP64 true residual as the diagnostics of solvers/diagnostics.py:8-19.
"""

from __future__ import annotations

import dataclasses
import warnings

import numpy as np

from .forms import PointField, call_points, flat_params
from .operator import Operator


@dataclasses.dataclass(frozen=True)
class LinearOptions:
    """Linear-solver configuration (solvers/linear.py:76-127) plus the device fields.

    ``backend="b200"`` (the only backend here) runs matrix-free CG on the GPU;
    ``precision`` is ``"fp64"`` (plain) or ``"mixed"`` (FP32 iterations with
    FP64 corrections to ``tol``). ``refinement`` picks the mixed scheme:
    ``"reliable"`` (FP32 PCG whose iterate and residual are refreshed in FP64
    each time the residual has fallen by ``update_delta``, keeping the search
    direction) or ``"restart"`` (FP64 iterative refinement around FP32 inner
    solves to ``inner_tol``). ``check_every`` is the iterations per captured
    CUDA graph launch between host convergence checks.
    """

    method: str = "cg"
    matrix_free: bool = True
    preconditioner: str = "jacobi"
    tol: float = 1e-10
    maxiter: int | None = None
    superlu_ordering: str = "auto"
    backend: str = "b200"
    precision: str = "fp64"
    inner_tol: float = 1e-4
    check_every: int = 16
    refinement: str = "reliable"
    update_delta: float = 1e-2

    def __post_init__(self):
        if not np.isfinite(self.tol) or self.tol <= 0:
            raise ValueError("tol must be finite and positive")
        if self.maxiter is not None and (isinstance(self.maxiter, (bool, np.bool_))
                                         or not isinstance(self.maxiter, (int, np.integer)) or self.maxiter <= 0):
            raise ValueError("maxiter must be a positive integer or None")
        allowed = {"cg", "bicgstab", "gmres", "dense", "scipy"}
        if self.method not in allowed:
            raise ValueError(f"unknown linear method {self.method!r}; expected one of {allowed}")
        if self.preconditioner not in {"none", "jacobi"}:
            raise ValueError(f"unknown preconditioner {self.preconditioner!r}; expected 'none' or 'jacobi'")
        orderings = {"auto", "NATURAL", "MMD_ATA", "MMD_AT_PLUS_A", "COLAMD"}
        if self.superlu_ordering not in orderings:
            raise ValueError(f"unknown SuperLU ordering {self.superlu_ordering!r}; expected one of {orderings}")
        if self.matrix_free and self.method in {"dense", "scipy"}:
            raise ValueError(f"matrix_free=True needs an iterative method, not {self.method!r}; "
                             f"there is no matrix for a direct solver to factor")
        if self.backend != "b200":
            raise ValueError(f"unknown backend {self.backend!r}; this package provides 'b200'")
        if self.precision not in {"fp64", "mixed"}:
            raise ValueError(f"precision must be 'fp64' or 'mixed', got {self.precision!r}")
        if not (0 < self.inner_tol < 1):
            raise ValueError("inner_tol must lie in (0, 1)")
        if self.refinement not in {"reliable", "restart"}:
            raise ValueError(f"refinement must be 'reliable' or 'restart', got {self.refinement!r}")
        if not (0 < self.update_delta < 1):
            raise ValueError("update_delta must lie in (0, 1)")


def default_linear(problem) -> LinearOptions:
    """The reference's accelerator default for SPD linear energies (galerkin.py:255-272)."""
    return LinearOptions(method="cg", matrix_free=True, preconditioner="jacobi", tol=1e-12)


def geometry_operator(space) -> Operator:
    """Cached evaluation plan of a space (coordinates, weights, interpolation)."""
    op = space._plans.get("geometry")
    if op is None:
        op = Operator(space, "poisson", (1.0,), vec=1)
        space._plans["geometry"] = op
    return op


def qp_points(space):
    """Physical Gauss-point coordinates, cached on the host as (n_elem*n_q, dim)."""
    x = space._plans.get("qp_points")
    if x is None:
        x = geometry_operator(space).qp_coords().reshape(-1, space.dim).cpu().numpy()
        space._plans["qp_points"] = x
    return x


@dataclasses.dataclass
class Solution:
    """A solved field (post/solution.py:23-50)."""

    space: object
    u: np.ndarray
    params: object = None
    problem: object = None
    stats: dict = dataclasses.field(default_factory=dict)
    u_device: object = None

    def at(self, ps=None, basis=None):
        """Values at the interior Gauss points, ``(n_e, n_q, vec)``."""
        if ps is not None or basis is not None:
            raise NotImplementedError("the B200 backend evaluates solutions at the interior Gauss set only")
        g = geometry_operator(self.space)
        u = self.u_device if self.u_device is not None else self.u
        return g.interpolate(u).cpu().numpy()


def solve(problem, *, method: str = "galerkin", params=None, linear: LinearOptions | None = None,
          initial_guess=None, **method_opts):
    """Solve a linear problem by the Galerkin method on the GPU."""
    import torch

    if method != "galerkin":
        raise NotImplementedError(f"method={method!r}: the B200 backend implements 'galerkin' only")
    if not problem.is_linear:
        raise NotImplementedError("the B200 backend solves linear problems only")
    if problem.neumann:
        raise NotImplementedError("Neumann loads are not applied by the B200 backend")
    if problem.quadrature is not None and problem.quadrature != problem.space.degree[0] + 1:
        raise NotImplementedError("the B200 backend uses the default p+1 Gauss rule")
    if linear is None:
        linear = default_linear(problem)
    if linear.method != "cg":
        raise NotImplementedError(f"linear method {linear.method!r}: the B200 backend runs CG")
    space = problem.space
    n = space.n_dofs
    prescribed, values = problem.resolve_dirichlet(params)
    mask = np.zeros(n, dtype=bool)
    mask[prescribed] = True

    coef, field = problem.operator_coefficients(params)
    coef_qp = None
    if field is not None:
        if isinstance(field, PointField):
            coef_qp = np.asarray(field.values, dtype=float)
        else:
            x = qp_points(space)
            coef_qp = call_points(field, x, flat_params(params, x.shape[0])).reshape(-1)
    op = Operator(space, problem.op, coef, prescribed=mask, coef_qp=coef_qp,
                  want_f32=linear.precision == "mixed", plane_strain=getattr(problem, "plane", "stress") == "strain")
    try:
        F = torch.zeros(n, dtype=torch.float64, device=op.device)
        if problem.source is not None:
            x = qp_points(space)
            f = call_points(problem.source, x, flat_params(params, x.shape[0]))
            f = np.broadcast_to(f.reshape(x.shape[0], -1), (x.shape[0], space.vec))
            F = op.load(np.array(f, dtype=np.float64, copy=True))
        b = F
        g = np.zeros(n)
        g[prescribed] = values
        if np.any(values != 0):
            b = F - op.apply(g, masked=False)
        if linear.precision == "mixed" and linear.refinement == "reliable":
            xdev, st = op.mixed_pcg(b, tol=linear.tol, delta=linear.update_delta, maxiter=linear.maxiter,
                                    check_every=linear.check_every)
        elif linear.precision == "mixed":
            xdev, st = op.refine_solve(b, tol=linear.tol, inner_tol=linear.inner_tol, maxiter=linear.maxiter,
                                       check_every=linear.check_every)
        else:
            xdev, st = op.pcg(b, tol=linear.tol, maxiter=linear.maxiter, preconditioner=linear.preconditioner,
                              check_every=linear.check_every)
        if len(prescribed):
            xdev[torch.as_tensor(prescribed, device=op.device)] = torch.as_tensor(values, device=op.device)
        u = xdev.cpu().numpy()
    finally:
        op.close()
    stats = {
        "method": "galerkin",
        "linear": linear.method,
        "matrix_free": True,
        "n_free": int(n - len(prescribed)),
        "nnz": None,
        "residual": st["residual"],
        "relative_residual": st["relative_residual"],
        "converged": bool(st["converged"]),
        "finite": bool(st["finite"]),
        "iterations": int(st["iterations"]),
        "outer": int(st["outer"]),
        "seconds": st["seconds"],
        "precision": linear.precision,
        "refinement": linear.refinement if linear.precision == "mixed" else None,
    }
    if not stats["converged"]:
        warnings.warn(f"linear Galerkin solve did not converge (residual {stats['residual']:.3e}); "
                      "do not use this result for implicit sensitivities", RuntimeWarning, stacklevel=2)
    return Solution(space=space, u=u, params=params, problem=problem, stats=stats, u_device=xdev)


def _exact_at(exact, x):
    """``exact`` over points (n, dim): vectorised over rows, else point by point (norms.py:17-32)."""
    try:
        out = np.asarray(exact(x), dtype=float)
        if out.shape[0] != x.shape[0]:
            raise ValueError
    except Exception:
        out = np.stack([np.asarray(exact(xi), dtype=float) for xi in x])
    return out.reshape(x.shape[0], -1)


def errornorm(sol, exact, norm: str = "L2", exact_grad=None, quad=None, relative: bool = True) -> float:
    """Relative (default) L2 error against ``exact(x)`` (post/norms.py:59-111)."""
    if norm != "L2":
        raise NotImplementedError("the B200 backend computes the L2 error norm")
    if quad is not None:
        raise NotImplementedError("the B200 backend uses the default Gauss rule")
    space = sol.space
    g = geometry_operator(space)
    w = g.qp_weights().reshape(-1).cpu().numpy()
    uh = sol.at().reshape(-1, space.vec)
    ue = _exact_at(exact, qp_points(space)).reshape(uh.shape)
    num = np.sum(w * np.sum((uh - ue) ** 2, -1))
    if not relative:
        return float(np.sqrt(num))
    den = np.sum(w * np.sum(ue**2, -1))
    return float(np.sqrt(num / den))


def norm(sol, norm: str = "L2", quad=None) -> float:
    if norm != "L2":
        raise NotImplementedError("the B200 backend computes the L2 norm")
    g = geometry_operator(sol.space)
    w = g.qp_weights().reshape(-1).cpu().numpy()
    u = sol.at().reshape(-1, sol.space.vec)
    return float(np.sqrt(np.sum(w * np.sum(u**2, -1))))


def integrate(fn, space, quad=None) -> float:
    """Integral of ``fn(x)`` over the patch; ``x`` is (n_points, dim) (post/norms.py:36-40)."""
    if quad is not None:
        raise NotImplementedError("the B200 backend uses the default Gauss rule")
    w = geometry_operator(space).qp_weights().reshape(-1).cpu().numpy()
    x = qp_points(space)
    try:
        v = np.asarray(fn(x), dtype=float).reshape(x.shape[0], -1)
    except Exception:
        v = np.stack([np.atleast_1d(np.asarray(fn(xi[None]), dtype=float)).ravel()[0] for xi in x])[:, None]
    return float(np.sum(w[:, None] * v))
