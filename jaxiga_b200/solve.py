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

    ``restarts``: FP64 CG restarts on the true residual when CG's recursive
    residual met ``tol`` but b - K u did not (at most this many, sharing
    ``maxiter``), the correction solves of the reference's CPU CG
    (solvers/linear.py:261-321).

    ``preconditioner="multigrid"`` runs CG preconditioned by a geometric
    multigrid V-cycle over the patch with every other knot removed level by
    level (``jaxiga_b200.multigrid``; Chebyshev-Jacobi smoothing of degree
    ``mg_degree`` on the interval lmax / ``mg_range`` .. lmax, FP64).

    ``preconditioner="learned"`` runs flexible CG with the trained network of
    ``checkpoint`` (see ``jaxiga_b200.learned``), Jacobi as its fallback;
    ``learned_map`` picks how the network output n enters: ``"network"`` (n
    alone), ``"multiplicative"`` (n, then a Jacobi step on the remaining
    residual) or ``"additive"`` (n + D^-1 r). With ``precision="mixed"`` the
    flexible CG runs in FP32 with FP64 corrections.
    """

    method: str = "cg"
    # the device path is always matrix-free; the flag keeps the reference's
    # validation (a direct method cannot be matrix-free)
    matrix_free: bool = False
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
    restarts: int = 3
    mg_degree: int = 3
    mg_range: float = 20.0
    checkpoint: str | None = None
    learned_map: str = "additive"
    learned_stall: int = 50

    def __post_init__(self):
        if not np.isfinite(self.tol) or self.tol <= 0:
            raise ValueError("tol must be finite and positive")
        if self.maxiter is not None and (isinstance(self.maxiter, (bool, np.bool_))
                                         or not isinstance(self.maxiter, (int, np.integer)) or self.maxiter <= 0):
            raise ValueError("maxiter must be a positive integer or None")
        allowed = {"cg", "bicgstab", "gmres", "dense", "scipy"}
        if self.method not in allowed:
            raise ValueError(f"unknown linear method {self.method!r}; expected one of {allowed}")
        if self.preconditioner not in {"none", "jacobi", "learned", "multigrid"}:
            raise ValueError(f"unknown preconditioner {self.preconditioner!r}; expected 'none', 'jacobi', "
                             f"'learned' or 'multigrid'")
        if isinstance(self.mg_degree, (bool, np.bool_)) or not isinstance(self.mg_degree, (int, np.integer)) \
                or not 1 <= self.mg_degree <= 8:
            raise ValueError("mg_degree must be an integer in 1..8")
        if not (np.isfinite(self.mg_range) and self.mg_range > 1):
            raise ValueError("mg_range must be finite and > 1")
        if self.preconditioner == "learned" and not self.checkpoint:
            raise ValueError("preconditioner='learned' needs checkpoint=<path of a trained network (.npz)>")
        if self.learned_map not in {"network", "multiplicative", "additive"}:
            raise ValueError(f"learned_map must be 'network', 'multiplicative' or 'additive', got {self.learned_map!r}")
        if (isinstance(self.restarts, (bool, np.bool_)) or not isinstance(self.restarts, (int, np.integer))
                or not 0 <= self.restarts <= 8):
            raise ValueError("restarts must be an integer in 0..8")
        if isinstance(self.learned_stall, (bool, np.bool_)) or not isinstance(self.learned_stall, (int, np.integer)) \
                or self.learned_stall < 1:
            raise ValueError("learned_stall must be a positive integer")
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
        from .multipatch import MultiPatchGeometry, MultiPatchSpace

        from .hierarchical import HierarchicalSpace

        if isinstance(space, MultiPatchSpace):
            op = MultiPatchGeometry(space)
        elif isinstance(space, HierarchicalSpace):
            from .thb import ThbGeometry

            op = ThbGeometry(space)
        else:
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


def _points(space, ps, coef=None, val=True, grad=False, x=False, jac=False):
    """Device evaluation on a PointSet, outputs shaped (n_e, n_q, ...) on the host."""
    g = geometry_operator(space)
    elems, ref = ps.flat()
    out = g.eval_points(elems, ref, coef, val=val, grad=grad, x=x, jac=jac)
    return {k: v.cpu().numpy().reshape(ps.n_elems, ps.n_q, *v.shape[1:]) for k, v in out.items()}


@dataclasses.dataclass
class Solution:
    """A solved field (post/solution.py:23-54)."""

    space: object
    u: np.ndarray
    params: object = None
    problem: object = None
    stats: dict = dataclasses.field(default_factory=dict)
    u_device: object = None

    def _coef(self):
        return self.u_device if self.u_device is not None else self.u

    def at(self, ps=None, basis=None):
        """Values on a PointSet (default: the interior p+1 Gauss set), ``(n_e, n_q, vec)``."""
        if basis is not None:
            raise NotImplementedError("the B200 backend evaluates on PointSets (jaxiga_b200.pointset), "
                                      "not on precomputed basis data")
        if ps is None:
            return geometry_operator(self.space).interpolate(self._coef()).cpu().numpy()
        return _points(self.space, ps, self._coef())["val"]

    def __call__(self, ps):
        return self.at(ps)

    def grad(self, ps=None, basis=None):
        """Physical gradients on a PointSet, ``(n_e, n_q, vec, dim)``."""
        if basis is not None:
            raise NotImplementedError("the B200 backend evaluates on PointSets (jaxiga_b200.pointset), "
                                      "not on precomputed basis data")
        if ps is None:
            return geometry_operator(self.space).interpolate_grad(self._coef()).cpu().numpy()
        return _points(self.space, ps, self._coef(), val=False, grad=True)["grad"]


# at most this many device operators stay cached per space (each holds the
# per-point factors of one operator, up to a few GB at the largest sizes)
OPERATOR_CACHE_SIZE = 2


def _digest(a):
    """Content key of an array (or None) for the operator cache."""
    if a is None:
        return None
    import hashlib

    a = np.ascontiguousarray(a)
    return (a.shape, a.dtype.str, hashlib.blake2b(a.view(np.uint8).reshape(-1), digest_size=16).hexdigest())


def cached_operator(space, op_name, coef, prescribed_mask=None, coef_qp=None, want_f32=False, plane_strain=False):
    """The device operator of (space, operator, coefficients, Dirichlet set),
    built once and reused by later solves on the same space: the per-point
    factors, the Jacobi diagonal and the captured CG graphs persist across
    calls. Least recently used operators beyond ``OPERATOR_CACHE_SIZE`` are
    released."""
    from collections import OrderedDict

    cache = space._plans.setdefault("operators", OrderedDict())
    key = (op_name, tuple(float(c) for c in coef), _digest(coef_qp), _digest(prescribed_mask), bool(plane_strain))
    op = cache.get(key)
    if op is not None and op.handle is not None and (op.want_f32 or not want_f32):
        cache.move_to_end(key)
        return op
    if op is not None:
        cache.pop(key).close()
    from .multipatch import MultiPatchOperator, MultiPatchSpace

    from .hierarchical import HierarchicalSpace

    if isinstance(space, HierarchicalSpace):
        from .thb import ThbOperator

        cls = ThbOperator
    else:
        cls = MultiPatchOperator if isinstance(space, MultiPatchSpace) else Operator
    op = cls(space, op_name, coef, prescribed=prescribed_mask, coef_qp=coef_qp, want_f32=want_f32,
             plane_strain=plane_strain)
    cache[key] = op
    while len(cache) > OPERATOR_CACHE_SIZE:
        cache.popitem(last=False)[1].close()
    return op


def release_operators(space):
    """Free the device operators cached on ``space`` by earlier solves."""
    for op in space._plans.pop("operators", {}).values():
        op.close()


def _problem_operator(problem, params, want_f32):
    """Dirichlet partition and cached device operator of a linear problem."""
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
    op = cached_operator(space, problem.op, coef, mask, coef_qp, want_f32,
                         getattr(problem, "plane", "stress") == "strain")
    return op, prescribed, values


def _rhs(problem, params, op, prescribed, values):
    """b = F - K_fp g on the device (methods/galerkin.py:240-245), F the source
    and Neumann loads (methods/_common.py:280-318)."""
    import torch

    space = problem.space
    n = space.n_dofs
    F = torch.zeros(n, dtype=torch.float64, device=op.device)
    if problem.source is not None:
        x = qp_points(space)
        f = call_points(problem.source, x, flat_params(params, x.shape[0]))
        f = np.broadcast_to(f.reshape(x.shape[0], -1), (x.shape[0], space.vec))
        F = op.load(np.array(f, dtype=np.float64, copy=True))
    if problem.neumann:
        from .neumann import neumann_load

        F = neumann_load(op, problem, params, F)
    g = np.zeros(n)
    g[prescribed] = values
    if np.any(values != 0):
        F = F - op.apply(g, masked=False)
    return F


def _check_problem(problem, method):
    if method != "galerkin":
        raise NotImplementedError(f"method={method!r}: the B200 backend implements 'galerkin' only")
    if not problem.is_linear:
        raise NotImplementedError("the B200 backend solves linear problems and the neo-Hookean Hyperelasticity form")
    if problem.quadrature is not None and problem.quadrature != problem.space.degree[0] + 1:
        raise NotImplementedError("the B200 backend uses the default p+1 Gauss rule")


def solve(problem, *, method: str = "galerkin", params=None, linear: LinearOptions | None = None,
          initial_guess=None, features=None, **method_opts):
    """Solve a linear problem by the Galerkin method on the GPU.

    ``problem`` may also be a list of problems (with ``params`` a list of the
    same length), or ``params`` a list of parameter dicts for one problem: the
    B200 form of the reference's ``jax.vmap`` over ``solve``. The instances
    (2D Poisson, constant a0 per instance, homogeneous Dirichlet data) are then
    solved together, every CG iteration of all of them in one captured CUDA
    graph, and a list of Solutions is returned.

    ``features``: static per-control-point input channels of a learned
    preconditioner (for example a normalised log-permeability), shape
    (n_features, n_control_points); only read with ``preconditioner="learned"``.
    """
    if isinstance(problem, (list, tuple)) or isinstance(params, (list, tuple)):
        return _solve_batch(problem, params, linear, method)
    import torch

    if not problem.is_linear and method == "galerkin" and getattr(problem, "op", None) == "hyperelastic":
        # Newton on the device (methods/galerkin.py:337-354, solvers/newton.py)
        from .newton import newton_solve

        if problem.quadrature is not None and problem.quadrature != problem.space.degree[0] + 1:
            raise NotImplementedError("the B200 backend uses the default p+1 Gauss rule")
        if linear is None:
            linear = default_linear(problem)
        if linear.method != "cg" or linear.precision != "fp64" or linear.preconditioner not in ("jacobi", "none"):
            raise NotImplementedError("Newton steps run FP64 CG with the Jacobi preconditioner (or none)")
        opts = {k: method_opts[k] for k in ("tol", "max_steps", "line_search") if k in method_opts}
        unknown = set(method_opts) - set(opts)
        if unknown:
            raise TypeError(f"unknown Newton options {sorted(unknown)}")
        return newton_solve(problem, params, linear, initial_guess=initial_guess, **opts)
    _check_problem(problem, method)
    if linear is None:
        linear = default_linear(problem)
    requested = linear.method
    if linear.method in ("scipy", "dense", "gmres"):
        # Every supported operator is symmetric positive definite, so the device
        # CG reaches the same solution: the direct methods ("scipy": SuperLU,
        # "dense": LU, exact to rounding) run it to 1e-12 or the given tol if
        # tighter, GMRES to the given tol. stats["linear"] says "cg" and
        # stats["requested_method"] what was asked.
        tol = min(linear.tol, 1e-12) if linear.method in ("scipy", "dense") else linear.tol
        linear = dataclasses.replace(linear, method="cg", matrix_free=True, tol=tol)
    if linear.method == "bicgstab" and (linear.precision != "fp64" or linear.preconditioner not in ("jacobi", "none")):
        raise NotImplementedError("BiCGSTAB runs in FP64 with the Jacobi preconditioner (or none)")
    space = problem.space
    n = space.n_dofs
    # The Kirchhoff plate's FP32 operator cannot resolve the biharmonic system:
    # its condition number (~h^-4) times FP32 rounding exceeds 1, so FP32
    # iterations diverge. Its mixed form keeps the FP64 operator and FP64
    # Krylov loop and runs in FP32 only what the preconditioner computes (the
    # learned network; the Jacobi scaling otherwise).
    fp32_operator = linear.precision == "mixed" and problem.op != "plate"
    from .multipatch import MultiPatchSpace

    if isinstance(space, MultiPatchSpace):
        if linear.precision != "fp64" or linear.preconditioner not in ("jacobi", "none") or linear.method != "cg":
            raise NotImplementedError("multipatch spaces solve with FP64 Jacobi-PCG")
    from .hierarchical import HierarchicalSpace

    if isinstance(space, HierarchicalSpace):
        if linear.precision != "fp64" or linear.preconditioner not in ("jacobi", "none") or linear.method != "cg":
            raise NotImplementedError("hierarchical spaces solve with FP64 Jacobi-PCG")

    op, prescribed, values = _problem_operator(problem, params, fp32_operator)
    b = _rhs(problem, params, op, prescribed, values)
    from .adjoint import SOLVE_COUNTER

    SOLVE_COUNTER["forward"] += 1
    if linear.preconditioner == "learned":
        from .learned import LearnedPreconditioner

        lp = LearnedPreconditioner.from_checkpoint(op, linear.checkpoint, features=features)
        try:
            two = {"network": False, "multiplicative": "multiplicative", "additive": "additive"}[linear.learned_map]
            reliable = linear.refinement == "reliable"
            xdev, st = lp.solve(b, tol=linear.tol, maxiter=linear.maxiter, stall=linear.learned_stall,
                                mixed=fp32_operator, two_level=two, refinement=linear.refinement,
                                inner_tol=linear.update_delta if reliable else linear.inner_tol,
                                check_every=linear.check_every)
        finally:
            lp.close()
        st["outer"] = st["learned_iterations"]
    elif linear.method == "bicgstab":
        xdev, st = op.bicgstab(b, tol=linear.tol, maxiter=linear.maxiter, preconditioner=linear.preconditioner,
                               check_every=linear.check_every)
        st["outer"] = 0
    elif linear.preconditioner == "multigrid":
        mg = getattr(op, "_multigrid", None)
        if mg is None or mg.handle is None or (mg.degree, mg.smooth_range) != (linear.mg_degree, linear.mg_range):
            from .multigrid import Multigrid

            if mg is not None:
                mg.close()
            mg = Multigrid(problem, params, degree=linear.mg_degree, smooth_range=linear.mg_range, fine_op=op)
            op._multigrid = mg
        xdev, st = mg.solve(b, tol=linear.tol, maxiter=linear.maxiter, check_every=min(linear.check_every, 8))
    elif fp32_operator and linear.refinement == "reliable":
        xdev, st = op.mixed_pcg(b, tol=linear.tol, delta=linear.update_delta, maxiter=linear.maxiter,
                                check_every=linear.check_every)
    elif fp32_operator:
        xdev, st = op.refine_solve(b, tol=linear.tol, inner_tol=linear.inner_tol, maxiter=linear.maxiter,
                                   check_every=linear.check_every)
    else:
        xdev, st = op.pcg(b, tol=linear.tol, maxiter=linear.maxiter, preconditioner=linear.preconditioner,
                          check_every=linear.check_every, restarts=linear.restarts)
    if len(prescribed):
        xdev[torch.as_tensor(prescribed, device=op.device)] = torch.as_tensor(values, device=op.device)
    u = xdev.cpu().numpy()
    stats = {
        "method": "galerkin",
        "linear": linear.method,
        "requested_method": requested,
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
        "fp32_operator": fp32_operator,
        "preconditioner": linear.preconditioner,
        "refinement": linear.refinement if fp32_operator else None,
    }
    if not stats["converged"]:
        warnings.warn(f"linear Galerkin solve did not converge (residual {stats['residual']:.3e}); "
                      "do not use this result for implicit sensitivities", RuntimeWarning, stacklevel=2)
    return Solution(space=space, u=u, params=params, problem=problem, stats=stats, u_device=xdev)


def _solve_batch(problems, params, linear, method):
    """Many independent instances in one device batch (``BatchSolver``)."""
    from .batch import BatchSolver

    if isinstance(problems, (list, tuple)):
        problems = list(problems)
        params = list(params) if isinstance(params, (list, tuple)) else [params] * len(problems)
    else:
        params = list(params)
        problems = [problems] * len(params)
    if len(problems) != len(params):
        raise ValueError(f"{len(problems)} problems but {len(params)} parameter sets")
    if not problems:
        return []
    for pr in problems:
        _check_problem(pr, method)
    linear = linear or default_linear(problems[0])
    if linear.method != "cg" or linear.preconditioner != "jacobi" or linear.precision != "fp64":
        raise NotImplementedError("batched solves run FP64 Jacobi-PCG")
    bs = BatchSolver(problems, params)
    try:
        xs, sts, secs = bs.solve(tol=linear.tol, maxiter=linear.maxiter, check_every=linear.check_every)
        out = []
        for pr, pa, x, st in zip(problems, params, xs, sts):
            u = x.cpu().numpy().copy()
            stats = {"method": "galerkin", "linear": "cg", "matrix_free": True,
                     "n_free": int(pr.space.n_dofs - len(pr.resolve_dirichlet(pa)[0])), "nnz": None,
                     "residual": st["residual"], "relative_residual": st["relative_residual"],
                     "converged": bool(st["converged"]), "finite": bool(st["finite"]),
                     "iterations": int(st["iterations"]), "outer": 0, "seconds": secs, "batched": len(problems),
                     "precision": "fp64", "preconditioner": "jacobi", "refinement": None}
            out.append(Solution(space=pr.space, u=u, params=pa, problem=pr, stats=stats, u_device=x.clone()))
    finally:
        bs.close()
    bad = [i for i, so in enumerate(out) if not so.stats["converged"]]
    if bad:
        warnings.warn(f"{len(bad)} of {len(out)} batched solves did not converge (first: instance {bad[0]})",
                      RuntimeWarning, stacklevel=3)
    return out


def _exact_at(exact, x):
    """``exact`` over points (n, dim): vectorised over rows, else point by point (norms.py:17-32)."""
    try:
        out = np.asarray(exact(x), dtype=float)
        if out.shape[0] != x.shape[0]:
            raise ValueError
    except Exception:
        out = np.stack([np.asarray(exact(xi), dtype=float) for xi in x])
    return out.reshape(x.shape[0], -1)


def _quadrature(space, quad, coef=None, grad=False):
    """Weights, points, and (optionally) values and gradients of a field on the
    Gauss set with ``quad`` points per direction (default p + 1), flattened over
    (element, point)."""
    from .pointset import gauss

    g = geometry_operator(space)
    if quad is None or all(int(quad) == p + 1 for p in space.degree):
        out = {"w": g.qp_weights().reshape(-1).cpu().numpy(), "x": qp_points(space)}
        if coef is not None:
            out["val"] = g.interpolate(coef).cpu().numpy().reshape(len(out["w"]), -1)
            if grad:
                out["grad"] = g.interpolate_grad(coef).cpu().numpy().reshape(len(out["w"]), -1, space.dim)
        return out
    ps = gauss(space, quad)
    r = _points(space, ps, coef, val=coef is not None, grad=grad and coef is not None, x=True, jac=True)
    out = {"w": (ps.flat_weights() * r["jac"].reshape(-1)), "x": r["x"].reshape(-1, space.dim)}
    if coef is not None:
        out["val"] = r["val"].reshape(ps.n_pts, -1)
        if grad:
            out["grad"] = r["grad"].reshape(ps.n_pts, -1, space.dim)
    return out


def _strain_voigt(g):
    """Engineering Voigt strain of displacement gradients (n, dim, dim) (materials.py:91-112)."""
    if g.shape[-1] == 2:
        return np.stack([g[:, 0, 0], g[:, 1, 1], g[:, 0, 1] + g[:, 1, 0]], axis=1)
    return np.stack([g[:, 0, 0], g[:, 1, 1], g[:, 2, 2], g[:, 1, 2] + g[:, 2, 1], g[:, 0, 2] + g[:, 2, 0],
                     g[:, 0, 1] + g[:, 1, 0]], axis=1)


def errornorm(sol, exact, norm: str = "L2", exact_grad=None, quad=None, relative: bool = True) -> float:
    """Error against an exact solution, relative by default (post/norms.py:59-140).

    ``norm`` is ``"L2"``, ``"H1"`` (the gradient seminorm, needs ``exact_grad``
    returning (vec, dim) per point) or ``"energy"`` (needs a problem with a
    constitutive matrix and ``exact_grad`` returning the exact Voigt stress).
    ``quad`` is the Gauss points per direction (default p + 1).
    """
    if norm not in ("L2", "H1", "energy"):
        raise ValueError(f"unknown norm {norm!r}")
    if norm in ("H1", "energy") and exact_grad is None:
        raise ValueError(f"the {norm!r} norm needs exact_grad")
    space = sol.space
    Q = _quadrature(space, quad, sol._coef(), grad=norm != "L2")
    w, x = Q["w"], Q["x"]
    if norm == "L2":
        uh = Q["val"]
        ue = _exact_at(exact, x).reshape(uh.shape)
        num = np.sum(w * np.sum((uh - ue) ** 2, -1))
        den = np.sum(w * np.sum(ue**2, -1))
    elif norm == "H1":
        gh = Q["grad"]
        ge = _exact_at(exact_grad, x).reshape(gh.shape)
        num = np.sum(w * np.sum((gh - ge) ** 2, axis=(-1, -2)))
        den = np.sum(w * np.sum(ge**2, axis=(-1, -2)))
    else:
        problem = sol.problem
        if problem is None or not hasattr(problem, "C"):
            raise ValueError(f"the energy norm needs a problem with a constitutive matrix; "
                             f"{type(problem).__name__} has none")
        C = problem.C(sol.params)
        Cinv = np.linalg.inv(C)
        stress_h = _strain_voigt(Q["grad"]) @ C.T
        stress_e = _exact_at(exact_grad, x).reshape(stress_h.shape)
        d = stress_h - stress_e
        num = np.sum(w * np.einsum("ni,ij,nj->n", d, Cinv, d))
        den = np.sum(w * np.einsum("ni,ij,nj->n", stress_e, Cinv, stress_e))
    if not relative:
        return float(np.sqrt(num))
    return float(np.sqrt(num / den))


def norm(sol, norm: str = "L2", quad=None) -> float:
    """L2 or H1 norm of the solution field (post/norms.py:43-56)."""
    if norm not in ("L2", "H1"):
        raise ValueError(f"unknown norm {norm!r}")
    Q = _quadrature(sol.space, quad, sol._coef(), grad=norm == "H1")
    s = np.sum(Q["w"] * np.sum(Q["val"] ** 2, -1))
    if norm == "H1":
        s += np.sum(Q["w"] * np.sum(Q["grad"] ** 2, axis=(-1, -2)))
    return float(np.sqrt(s))


def integrate(fn, space, quad=None) -> float:
    """Integral of ``fn(x)`` over the patch; ``x`` is (n_points, dim) (post/norms.py:36-40)."""
    Q = _quadrature(space, quad)
    w, x = Q["w"], Q["x"]
    try:
        v = np.asarray(fn(x), dtype=float).reshape(x.shape[0], -1)
    except Exception:
        v = np.stack([np.atleast_1d(np.asarray(fn(xi[None]), dtype=float)).ravel()[0] for xi in x])[:, None]
    return float(np.sum(w[:, None] * v))
