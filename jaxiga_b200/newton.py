"""Newton's method for the nonlinear Galerkin path on the GPU.

The drop-in for the reference's ``newton`` (src/jaxiga/solvers/newton.py:27-135)
driven by ``solve_galerkin`` for a nonlinear problem
(src/jaxiga/methods/galerkin.py:337-354), here for the compressible neo-Hookean
``Hyperelasticity`` form. Each step:

* sets the device state to the iterate u (``Operator.state``: F, F^-T, ln J and
  the Piola flux at every Gauss point, one kernel),
* forms the residual R(u) = int P(F) : grad v - f_ext on the free DOFs
  (``Operator.residual``, the backward half of the brick apply),
* solves K(u) du = -R with the matrix-free tangent at u (Jacobi-PCG on the
  device, the reference's ``matvec_fn`` path, galerkin.py:207-237), and
* backtracks by halving (at most 20 times) until the residual norm decreases,
  as the reference's line search does (newton.py:66-90).

The loop's stopping rule, history and flags (``converged``, ``finite``,
``iteration_limit``, ``stalled``) follow newton.py:92-135. The reference's
implicit-function-theorem correction changes derivatives, not values, so the
returned state is the same.
"""

from __future__ import annotations

import math
import time
import warnings

import numpy as np

MAX_BACKTRACKS = 20


def history_list(stats):
    """The residual history as a plain list, NaN padding removed (newton.py:193-196)."""
    h = np.asarray(stats["history"], dtype=float)
    return [float(v) for v in h[~np.isnan(h)]]


def _external_loads(problem, params, op):
    """Source and Neumann loads f_ext (methods/_common.py:280-318) on the device."""
    import torch

    from .forms import call_points, flat_params
    from .solve import qp_points

    space = problem.space
    F = torch.zeros(space.n_dofs, dtype=torch.float64, device=op.device)
    if problem.source is not None:
        x = qp_points(space)
        f = call_points(problem.source, x, flat_params(params, x.shape[0]))
        f = np.broadcast_to(f.reshape(x.shape[0], -1), (x.shape[0], space.vec))
        F = op.load(np.array(f, dtype=np.float64, copy=True))
    if problem.neumann:
        from .neumann import neumann_load

        F = neumann_load(op, problem, params, F)
    return F


def newton_solve(problem, params, linear, initial_guess=None, tol: float = 1e-8, max_steps: int = 25,
                 line_search: bool = True):
    """Solve R(u) = 0 for a nonlinear problem; returns a ``Solution`` whose stats
    carry the reference's Newton diagnostics plus the linear iterations."""
    import torch

    from .solve import Solution, cached_operator

    space = problem.space
    n = space.n_dofs
    prescribed, values = problem.resolve_dirichlet(params)
    mask = np.zeros(n, dtype=bool)
    mask[prescribed] = True
    coef, _ = problem.operator_coefficients(params)
    op = cached_operator(space, problem.op, coef, mask)
    dev = op.device
    f_ext = _external_loads(problem, params, op)
    pres = torch.as_tensor(np.asarray(prescribed, dtype=np.int64), device=dev)
    u = torch.zeros(n, dtype=torch.float64, device=dev)
    if initial_guess is not None:
        g = torch.as_tensor(np.asarray(initial_guess, dtype=np.float64), device=dev)
        if g.numel() == n:
            u.copy_(g)
        elif g.numel() == n - len(prescribed):
            u[torch.as_tensor(~mask, device=dev)] = g
        else:
            raise ValueError(f"initial_guess has {g.numel()} entries; expected {n} or {n - len(prescribed)}")
    if len(prescribed):
        u[pres] = torch.as_tensor(np.asarray(values, dtype=np.float64), device=dev)

    def residual(uu):
        op.state(uu)
        r = op.residual() - f_ext
        if len(prescribed):
            r[pres] = 0.0
        return r

    def norm_of(uu):
        return float(torch.linalg.norm(residual(uu)))

    def backtrack(uu, du, r_norm):
        alpha = 1.0
        trial = norm_of(uu + alpha * du)
        k = 0
        while (not math.isfinite(trial) or trial >= r_norm) and k < MAX_BACKTRACKS:
            alpha *= 0.5
            trial = norm_of(uu + alpha * du)
            k += 1
        accepted = math.isfinite(trial) and trial < r_norm
        return (alpha if accepted else 0.0), trial

    t0 = time.perf_counter()
    r_norm = norm_of(u)
    history = np.full(int(max_steps) + 1, np.nan)
    history[0] = r_norm
    step, alpha, lin_its = 0, 1.0, 0
    while math.isfinite(r_norm) and r_norm > tol and step < max_steps and alpha > 0.0:
        r = residual(u)  # the state is u for the tangent solve
        du, st = op.pcg(-r, tol=linear.tol, maxiter=linear.maxiter, preconditioner=linear.preconditioner,
                        check_every=linear.check_every, restarts=linear.restarts)
        lin_its += int(st["iterations"])
        if line_search:
            alpha, trial = backtrack(u, du, r_norm)
        else:
            alpha, trial = 1.0, norm_of(u + du)
        if alpha > 0.0:
            u = u + alpha * du
            r_norm = trial
        step += 1
        history[step] = r_norm
    converged = r_norm <= tol
    stalled = alpha <= 0.0 and not converged
    r_final = norm_of(u)  # leaves the device state at the returned u
    finite = math.isfinite(r_final) and bool(torch.isfinite(u).all())
    converged = finite and r_final <= tol
    stats = {
        "method": "galerkin",
        "nonlinear": "newton",
        "iterations": step,
        "residual": r_final,
        "converged": converged,
        "finite": finite,
        "iteration_limit": step >= max_steps and not converged,
        "stalled": stalled,
        "history": history,
        "linear_iterations": lin_its,
        "matrix_free": True,
        "seconds": time.perf_counter() - t0,
    }
    if not converged:
        if not math.isfinite(r_final):
            reason = "a non-finite state was encountered"
        elif stalled:
            reason = "the line search found no finite decreasing step"
        elif step >= max_steps:
            reason = f"the {max_steps}-step limit was reached"
        else:
            reason = "the final correction did not satisfy the tolerance"
        warnings.warn(f"Newton did not reach tol={tol:g}: {reason} after {step} steps, final residual "
                      f"{r_final:.3e}", RuntimeWarning, stacklevel=3)
    return Solution(space=space, u=u.cpu().numpy(), params=params, problem=problem, stats=stats, u_device=u)
