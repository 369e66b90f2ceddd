"""Gradients through the device solve: one forward and one adjoint solve.

The reference differentiates ``solve`` with ``jax.grad``; its linear solves go
through ``jax.lax.custom_linear_solve`` / a custom VJP so that a gradient
costs exactly one forward and one adjoint (transposed) solve, never a
differentiation through the Krylov iterations
(src/jaxiga/solvers/linear.py:360-389, 414-442; pinned by
tests/test_galerkin.py:264-274 through ``SOLVE_COUNTER``).

Without JAX the same contract is offered explicitly. For an objective J(u)
of the lifted solution u (the caller supplies J and dJ/du),

    K_ff u_f = b_f = F_f - K_fp g,        r(u_f, theta) = (K u)_f - F_f,
    dJ/dtheta = -lambda^T (dK/dtheta u)_f,   K_ff lambda = (dJ/du)_f,

with one more ``jxb_pcg`` on the same cached device operator for lambda (the
Galerkin operator is symmetric, so the adjoint operator is K itself). The
parameter terms are formed on the device from the operator, or from the
gradients of lambda and u at the Gauss points:

* Poisson ``a0`` scalar:   dK/da0 u = K u / a0
* Poisson ``a0`` per point (a PointField, one value per Gauss point):
  dJ/da0_q = -w_q grad(lambda)(x_q) . grad(u)(x_q)
* elasticity ``E``:        dK/dE u = K u / E
* elasticity ``nu``:       dJ/dnu = -sum_q w_q eps(lambda)_q^T dC/dnu eps(u)_q,
  dC/dnu by a complex step of the constitutive matrix (exact to rounding)
* plate ``E`` / ``t``:     K scales with E t^3, so dK/dE u = K u / E, dK/dt u = 3 K u / t

Parameters that also enter the source or the Dirichlet data are not covered:
the objective's explicit dependence on them is the caller's.
"""

from __future__ import annotations

import numpy as np

SOLVE_COUNTER = {"forward": 0, "adjoint": 0}


def reset_solve_counter():
    """Zero the solve counters (src/jaxiga/solvers/linear.py:70-73)."""
    SOLVE_COUNTER["forward"] = 0
    SOLVE_COUNTER["adjoint"] = 0


def adjoint_solve(sol, dJ_du, linear=None):
    """lambda with K_ff lambda = (dJ/du)_f on the free DOFs (0 on prescribed DOFs),
    from the operator cached by the forward solve; returns (lambda, stats)."""
    import torch

    from .solve import _problem_operator, default_linear

    problem = sol.problem
    linear = linear or default_linear(problem)
    op, prescribed, _ = _problem_operator(problem, sol.params, False)
    g = torch.as_tensor(np.asarray(dJ_du, dtype=np.float64).reshape(-1), device=op.device).contiguous()
    if g.numel() != op.n_dofs:
        raise ValueError(f"dJ/du has {g.numel()} entries, expected {op.n_dofs}")
    SOLVE_COUNTER["adjoint"] += 1
    lam, st = op.pcg(g, tol=linear.tol, maxiter=linear.maxiter, preconditioner=linear.preconditioner,
                     check_every=linear.check_every, restarts=linear.restarts)
    return lam, st


def _scalar_param(params, name):
    v = params.get(name) if isinstance(params, dict) else None
    return v


def parameter_gradients(sol, lam, wrt):
    """-lambda^T (dK/dtheta u)_f for each name in ``wrt`` (see the module doc)."""
    import torch

    from .forms import PointField
    from .solve import _problem_operator, geometry_operator

    problem, params = sol.problem, sol.params
    op, prescribed, _ = _problem_operator(problem, params, False)
    u = torch.as_tensor(sol.u, dtype=torch.float64, device=op.device)
    lam = lam.to(op.device)
    out = {}
    Ku = None

    def k_u():
        nonlocal Ku
        if Ku is None:
            Ku = op.apply(u, masked=False)
        return Ku

    def free_dot(v):
        w = lam.clone()
        if len(prescribed):
            w[torch.as_tensor(prescribed, device=op.device)] = 0.0
        return float(torch.dot(w, v))

    for name in wrt:
        val = _scalar_param(params, name)
        if problem.op == "poisson" and name == "a0":
            if callable(val) and not isinstance(val, PointField):
                raise NotImplementedError("a0 given as a function of x: pass it as a PointField to differentiate")
            if isinstance(val, PointField):
                geo = geometry_operator(problem.space)
                w = geo.qp_weights().reshape(-1)
                gl = geo.interpolate_grad(lam).reshape(w.numel(), -1)
                gu = geo.interpolate_grad(u).reshape(w.numel(), -1)
                out[name] = (-(w[:, None] * gl * gu).sum(-1)).reshape(problem.space.n_elems, -1).cpu().numpy()
            else:
                a0 = float(1.0 if val is None else val)
                out[name] = -free_dot(k_u()) / a0
        elif problem.op == "elasticity" and name == "E":
            out[name] = -free_dot(k_u()) / float(params["E"])
        elif problem.op == "elasticity" and name == "nu":
            from .forms import constitutive
            from .solve import _strain_voigt

            E, nu, h = float(params["E"]), float(params["nu"]), 1e-30
            dC = np.imag(constitutive(E, complex(nu, h), problem.space.dim, problem.plane)) / h
            geo = geometry_operator(problem.space)
            w = geo.qp_weights().reshape(-1).cpu().numpy()
            d = problem.space.dim
            el = _strain_voigt(geo.interpolate_grad(lam).reshape(-1, d, d).cpu().numpy())
            eu = _strain_voigt(geo.interpolate_grad(u).reshape(-1, d, d).cpu().numpy())
            out[name] = float(-np.sum(w * np.einsum("ni,ij,nj->n", el, dC, eu)))
        elif problem.op == "plate" and name in ("E", "t"):
            scale = 1.0 if name == "E" else 3.0
            out[name] = -scale * free_dot(k_u()) / float(params[name])
        else:
            raise NotImplementedError(f"no device gradient with respect to {name!r} for the {problem.op} operator")
    return out


def value_and_grad(problem, params, objective, wrt, linear=None, **solve_opts):
    """J(u(theta)) and dJ/dtheta for the named parameters, at the cost of one
    forward and one adjoint device solve.

    ``objective(u)`` takes the lifted solution (host array, length n_dofs) and
    returns ``(J, dJ/du)``. Returns ``(J, grads, solution)``; ``grads`` maps each
    name of ``wrt`` to a float, or, for a per-point coefficient, an
    (n_elem, n_q) array.
    """
    from .solve import solve

    sol = solve(problem, params=params, linear=linear, **solve_opts)
    J, dJ = objective(sol.u)
    lam, _ = adjoint_solve(sol, dJ, linear)
    return float(J), parameter_gradients(sol, lam, tuple(wrt)), sol
