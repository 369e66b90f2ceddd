"""A posteriori error estimation and the adaptive refinement driver
(src/jaxiga/post/estimators.py).

The explicit residual indicator of the reference,

    eta_e^2 = h_e^2 sum_q w_q |r(u_h)(x_q)|^2,   h_e = |e|^(1/dim),

takes the volume term only, on a Gauss rule of p + 2 points per direction
(estimators.py:33-88). The reference differentiates the energy density to get
the strong residual r; here r is written out for the linear forms it applies
to: r = -a0 lap u - f for Poisson with a constant a0 (library.py:40-65) and
r = -div(C eps(u)) - f for linear elasticity with the problem's constitutive
matrix C (library.py:146-203).

The evaluation runs on the host from the same element data the device plans
take -- per element its DOFs, the extraction operator from its Bernstein
polynomials and the NURBS weights -- so tensor and THB spaces share it: the
rational numerator and W and their first and second reference derivatives at
the points, the second-order quotient rule, and the push-forward of second
derivatives through the geometry's own first and second derivatives
(evaluation.py:95-172).
"""

from __future__ import annotations

import numpy as np

from .forms import LinearElasticity, Poisson, call_points, flat_params
from .space import gauss_1d


def _element_data(space):
    """(elem_dofs, extraction (n_e, n_loc, nb)) of a tensor, multipatch or THB space (THB rows padded)."""
    from .hierarchical import HierarchicalSpace
    from .multipatch import MultiPatchSpace
    from .space import FunctionSpace

    if isinstance(space, HierarchicalSpace):
        return space.elem_dofs, space.extraction
    if isinstance(space, MultiPatchSpace):  # elements patch by patch, global (conforming) DOFs
        return space.elem_dofs, np.concatenate([s.extraction() for s in space.spaces])
    if isinstance(space, FunctionSpace):
        return space.elem_dofs, space.extraction()
    raise NotImplementedError("residual indicators run on tensor, multipatch and THB spaces")


def second_derivatives(space, u, n=None, chunk=2048):
    """Values, physical gradients and Hessians of the field with control
    coefficients ``u`` ((n_scalar, vec) or flat, interleaved) at the n^dim
    Gauss points of every element (default n = p + 2): x (e, q, dim),
    w (e, q), val (e, q, vec), grad (e, q, vec, dim), hess (e, q, vec, dim, dim)."""
    from .thb import tables_at

    dim, p = space.dim, space.degree[0]
    if space.dim_phys != dim:
        raise NotImplementedError("residual indicators need the physical and parametric dimensions equal")
    n = p + 2 if n is None else int(n)
    g1, w1 = gauss_1d(n)
    pts = np.stack([g.ravel(order="F") for g in np.meshgrid(*([g1] * dim), indexing="ij")], -1)
    wq = np.prod(np.stack([gw.ravel(order="F") for gw in np.meshgrid(*([w1] * dim), indexing="ij")], -1), -1)
    T = tables_at(pts, p, order=2)                          # (1 + dim + npairs, nq, nb)
    pairs = [(a, b) for a in range(dim) for b in range(a, dim)]
    elem_dofs, ext = _element_data(space)
    ns = space.n_scalar_basis
    U = np.asarray(u, dtype=float).reshape(ns, -1)
    vec = U.shape[1]
    hom = np.concatenate([space.cpts * space.wgts[:, None], space.wgts[:, None]], 1)
    hom = np.concatenate([hom, np.zeros((1, dim + 1))])
    Uw = np.concatenate([U * space.wgts[:, None], np.zeros((1, vec))])
    ne, nq = len(elem_dofs), len(wq)
    X, Wt = np.zeros((ne, nq, dim)), np.zeros((ne, nq))
    val, grad = np.zeros((ne, nq, vec)), np.zeros((ne, nq, vec, dim))
    hess = np.zeros((ne, nq, vec, dim, dim))
    for lo in range(0, ne, chunk):
        sl = slice(lo, min(lo + chunk, ne))
        C = ext[sl]
        d = elem_dofs[sl]
        geo = np.einsum("cqa,eia,eik->eqck", T, C, hom[d])   # channels of (w x, w)
        num = np.einsum("cqa,eia,eik->eqck", T, C, Uw[d])    # channels of the field's numerator
        W = geo[:, :, 0, dim]
        Wa = geo[:, :, 1:1 + dim, dim]
        x = geo[:, :, 0, :dim] / W[..., None]
        xa = (geo[:, :, 1:1 + dim, :dim] - Wa[..., None] * x[:, :, None]) / W[..., None, None]  # [a][i]

        def quotient(ch):  # reference derivatives of ch / W from the channels ch (e, q, NC, m)
            f = ch[:, :, 0] / W[..., None]
            fa = (ch[:, :, 1:1 + dim] - Wa[..., None] * f[:, :, None]) / W[..., None, None]
            fab = np.stack([(ch[:, :, 1 + dim + k] - fa[:, :, a] * Wa[..., b, None] - fa[:, :, b] * Wa[..., a, None]
                             - f * geo[:, :, 1 + dim + k, dim, None]) / W[..., None]
                            for k, (a, b) in enumerate(pairs)], 2)
            return f, fa, fab

        _, _, xab = quotient(geo[..., :dim])
        f, fa, fab = quotient(num)
        J = xa                                                # [a][i] = d x_i / d xi_a
        gx = np.linalg.solve(J, fa)                           # (e, q, dim, vec): physical gradient
        Tm = np.zeros(J.shape[:2] + (len(pairs), len(pairs)))
        for r, (a, b) in enumerate(pairs):
            for c, (i, j) in enumerate(pairs):
                Tm[..., r, c] = J[..., a, i] * J[..., b, j] + (J[..., a, j] * J[..., b, i] if i != j else 0.0)
        hx = np.linalg.solve(Tm, fab - np.einsum("eqki,eqic->eqkc", xab, gx))  # (e, q, pair, vec)
        X[sl], Wt[sl], val[sl] = x, wq[None, :] * np.abs(np.linalg.det(J)), f
        grad[sl] = np.moveaxis(gx, 2, 3)
        for k, (a, b) in enumerate(pairs):
            hess[sl, :, :, a, b] = hx[:, :, k]
            hess[sl, :, :, b, a] = hx[:, :, k]
    return X, Wt, val, grad, hess


def _voigt(dim):
    return [(0, 0), (1, 1), (0, 1)] if dim == 2 else [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]


def strong_residual(problem, params, x, grad, hess):
    """r (n, vec) of the problem's strong form at points x from the physical
    gradients (n, vec, dim) and Hessians (n, vec, dim, dim) of u_h."""
    n, vec, dim = grad.shape
    f = np.zeros((n, vec))
    if problem.source is not None:
        f = np.broadcast_to(call_points(problem.source, x, flat_params(params, n)).reshape(n, -1), (n, vec))
    if isinstance(problem, Poisson):
        (a0,), field = problem.operator_coefficients(params)
        if field is not None:
            raise NotImplementedError("residual indicators take a constant a0")
        return -a0 * np.trace(hess, axis1=-2, axis2=-1) - f
    if isinstance(problem, LinearElasticity):
        C = np.asarray(problem.C(params), dtype=float)
        V = _voigt(dim)
        # d eps / d x_k in engineering Voigt order, then d sigma / d x_k = C d eps / d x_k
        deps = np.stack([np.stack([hess[:, i, i, k] if i == j else hess[:, i, j, k] + hess[:, j, i, k]
                                   for i, j in V], 1) for k in range(dim)], 2)  # (n, nv, dim)
        dsig = np.einsum("st,ntk->nsk", C, deps)
        div = np.zeros((n, dim))
        for s, (i, j) in enumerate(V):
            div[:, i] += dsig[:, s, j]
            if i != j:
                div[:, j] += dsig[:, s, i]
        return -div - f
    raise NotImplementedError(f"residual indicators cover Poisson and linear elasticity, not {type(problem).__name__}")


def residual_indicator(sol, params=None, quad: int | None = None) -> np.ndarray:
    """Per-element explicit residual indicators eta_e (estimators.py:33-88):
    volume term only, on p + 2 Gauss points per direction unless ``quad``."""
    problem = sol.problem
    if problem is None:
        raise ValueError("residual_indicator needs a Solution that carries its problem")
    params = sol.params if params is None else params
    space = problem.space
    x, w, _, grad, hess = second_derivatives(space, sol.u, quad)
    ne, nq = w.shape
    r = strong_residual(problem, params, x.reshape(ne * nq, -1), grad.reshape((ne * nq,) + grad.shape[2:]),
                        hess.reshape((ne * nq,) + hess.shape[2:])).reshape(ne, nq, -1)
    h = np.sum(w, axis=1) ** (1.0 / space.dim)
    eta2 = h**2 * np.sum(w * np.sum(r**2, axis=-1), axis=1)
    return np.sqrt(np.maximum(eta2, 0.0))


def adapt(make_problem, params=None, *, space=None, n_cycles: int = 5, frac: float = 0.3, exact=None,
          exact_grad=None, solve_kwargs=None, verbose: bool = False):
    """Solve-estimate-mark-refine (estimators.py:91-183): ``make_problem`` maps
    a space to a problem; returns the last solution, its space and a history of
    per-cycle dicts (cycle, n_dofs, n_elems, eta and, with an exact solution,
    L2 and H1)."""
    from .hierarchical import dorfler_mark, refine_elements
    from .solve import errornorm, solve

    if not callable(make_problem):
        raise TypeError("adapt() takes a factory FunctionSpace -> Problem, not a Problem: a problem is bound "
                        "to one space at construction")
    if space is None:
        space = getattr(make_problem, "space", None)
    if space is None:
        raise TypeError("adapt() needs a starting space: pass space=V, or set make_problem.space = V")
    history, sol = [], None
    for cycle in range(n_cycles):
        sol = solve(make_problem(space), params=params, **(solve_kwargs or {}))
        eta = residual_indicator(sol, params)
        entry = {"cycle": cycle, "n_dofs": space.n_dofs, "n_elems": space.n_elems,
                 "eta": float(np.sqrt(np.sum(eta**2)))}
        if exact is not None:
            entry["L2"] = errornorm(sol, exact, "L2")
            if exact_grad is not None:
                entry["H1"] = errornorm(sol, exact, "H1", exact_grad=exact_grad)
        history.append(entry)
        if verbose:
            extra = "".join(f"  {k}={entry[k]:.4e}" for k in ("L2", "H1") if k in entry)
            print(f"  cycle {cycle}: {entry['n_dofs']:6d} dofs, {entry['n_elems']:6d} elems, "
                  f"eta={entry['eta']:.4e}{extra}")
        if cycle + 1 < n_cycles:
            space = refine_elements(space, dorfler_mark(eta, frac))
    return sol, space, history
