"""Geometric multigrid over nested spline spaces: the V-cycle preconditioner.

Levels. The finest level is the problem's own patch; each coarser one is the
same patch with every other distinct interior knot removed (per parametric
direction), so every coarse space is contained in the next finer one and the
prolongation is exact knot insertion. Its 1D matrices come from inserting the
removed knots into the identity (``insert_knots_1d``), and the coarse control
points and weights are fitted through them in homogeneous coordinates (exact
whenever the geometry lives on the coarse knots, as for every workload here).
Coarsening stops when a level has at most ``max_coarse`` DOFs or a direction
has a single span left.

Operators. Every level gets a libjxb plan of the same operator rediscretised on
its space, with the problem's Dirichlet conditions applied there (homogeneous:
the V-cycle acts on residuals). A per-point coefficient (a PointField a0) is
carried to a coarse Gauss point as the mean of the fine element containing it.
The coarsest operator is formed column by column with its plan and inverted
on the host (dense Cholesky of the free block).

Solve. ``jxb_mg_pcg`` runs CG with the V-cycle (Chebyshev-Jacobi smoothing of
degree ``degree`` before and after each coarse correction) as the
preconditioner, in FP64, graph-captured; see csrc/mg.cu.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .geometry import Patch, insert_knots_1d
from .operator import Operator
from .space import FunctionSpace


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def coarse_knots(kv):
    """The knot vector without every other distinct interior knot (all copies),
    and the removed knots (with multiplicity), which insertion puts back."""
    kv = np.asarray(kv, dtype=float)
    uniq = np.unique(kv)
    interior = uniq[1:-1]
    removed = set(interior[0::2].tolist())
    keep = np.array([k for k in kv if k not in removed])
    back = np.array([k for k in kv if k in removed])
    return keep, back


def prolongation_1d(kc, p, back):
    """(n_fine, n_coarse) matrix taking coarse B-spline coefficients to fine ones."""
    nc = len(kc) - p - 1
    _, P = insert_knots_1d(p, kc, np.eye(nc), back)
    P[np.abs(P) < 1e-15] = 0.0
    return P


def coarsen(space):
    """(coarse FunctionSpace, [P_d], exact) for a single-patch space, or None
    when some direction has no interior knot to remove."""
    patch = space.patch
    p = space.degree
    kcs, backs, Ps = [], [], []
    for d in range(space.dim):
        kc, back = coarse_knots(space.knots[d])
        if back.size == 0:
            return None
        kcs.append(kc)
        backs.append(back)
        Ps.append(prolongation_1d(kc, p[d], back))
    # fit the coarse homogeneous control points through the tensor prolongation
    h = patch.homogeneous()
    nf = list(space.n_cp)
    grid = h.reshape(*reversed(nf), h.shape[1])
    for d in range(space.dim):
        ax = space.dim - 1 - d
        sol = np.linalg.lstsq(Ps[d], np.moveaxis(grid, ax, 0).reshape(nf[d], -1), rcond=None)[0]
        grid = np.moveaxis(sol.reshape(Ps[d].shape[1], *np.moveaxis(grid, ax, 0).shape[1:]), 0, ax)
    hc = grid.reshape(-1, h.shape[1])
    # exactness: prolong back and compare
    back_grid = hc.reshape(*reversed([P.shape[1] for P in Ps]), h.shape[1])
    for d in range(space.dim):
        ax = space.dim - 1 - d
        back_grid = np.moveaxis(np.tensordot(Ps[d], np.moveaxis(back_grid, ax, 0), axes=(1, 0)), 0, ax)
    exact = bool(np.abs(back_grid.reshape(-1, h.shape[1]) - h).max() <= 1e-10 * max(1.0, np.abs(h).max()))
    w = hc[:, -1]
    cp = hc[:, :-1] / w[:, None]
    if np.all(patch.weights == 1.0):
        # a polynomial patch stays polynomial: the fit reproduces unit weights only
        # to rounding, and exact ones keep the coarse plans on the polynomial kernels
        w = np.ones_like(w)
    coarse = Patch.create(kcs, p, cp, w, labels=patch.labels)
    return FunctionSpace(coarse, vec=space.vec), Ps, exact


def coarse_coefficients(fine, coarse, coef_qp):
    """Per-point coefficient on the coarse Gauss points: the mean over the fine
    element that contains each coarse point."""
    if coef_qp is None:
        return None
    nq = coarse.degree[0] + 1
    nodes = np.polynomial.legendre.leggauss(nq)[0]
    fine_means = np.asarray(coef_qp, dtype=float).reshape(fine.n_elems, -1).mean(1)
    idx = []
    for d in range(coarse.dim):
        lo, hi = np.asarray(coarse.span_lo[d]), np.asarray(coarse.span_hi[d])
        u = lo[:, None] + (nodes[None, :] + 1.0) * 0.5 * (hi - lo)[:, None]  # (span, q)
        f = np.clip(np.searchsorted(np.asarray(fine.span_lo[d]), u, side="right") - 1, 0, fine.n_span[d] - 1)
        idx.append(f)
    dim = coarse.dim
    # fine element of every (coarse element, coarse point), both first direction fastest
    shp = [coarse.n_span[d] for d in range(dim)]
    out = np.zeros((coarse.n_elems, nq**dim))
    ec = np.indices(shp[::-1]).reshape(dim, -1)[::-1]  # per-direction coarse span per element
    qq = np.indices([nq] * dim).reshape(dim, -1)[::-1]  # per-direction point per element point
    fe = np.zeros((coarse.n_elems, nq**dim), dtype=np.int64)
    stride = 1
    for d in range(dim):
        fe += idx[d][ec[d][:, None], qq[d][None, :]] * stride
        stride *= fine.n_span[d]
    out[:] = fine_means[fe]
    return out


def _coarse_problem(problem, space):
    kw = {"dirichlet": problem.dirichlet}
    if problem.op == "elasticity":
        kw["plane"] = problem.plane
    return type(problem)(space, **kw)


def dense_inverse(op, mask):
    """Inverse of the operator's free block, embedded in an (n, n) array."""
    import torch

    n = op.n_dofs
    free = np.nonzero(~mask)[0]
    K = np.zeros((len(free), len(free)))
    e = torch.zeros(n, dtype=torch.float64, device=op.device)
    freet = torch.as_tensor(free, device=op.device)
    for k, j in enumerate(free):
        e.zero_()
        e[int(j)] = 1.0
        K[:, k] = op.apply(e)[freet].cpu().numpy()
    K = 0.5 * (K + K.T)
    L = np.linalg.cholesky(K)
    Li = np.linalg.solve(L, np.eye(len(free)))
    Kinv = Li.T @ Li
    out = np.zeros((n, n))
    out[np.ix_(free, free)] = Kinv
    return out


class Multigrid:
    """V-cycle preconditioner and MG-preconditioned CG for one linear problem.

    Parameters
    ----------
    problem, params : the problem (its space is the finest level) and parameters
    degree : Chebyshev smoother degree (1..8); each costs degree - 1 operator
        applications per smoothing, two smoothings per level and V-cycle
    smooth_range : lmax / lmin of the damped interval of D^-1 K
    max_coarse : stop coarsening at or below this many DOFs
    fine_op : an existing finest-level Operator to reuse (its mask must be the
        problem's), else one is built
    """

    def __init__(self, problem, params=None, degree=3, smooth_range=20.0, max_coarse=1500, fine_op=None,
                 max_levels=12):
        self.lib = _lib.load()
        self.problem = problem
        coef, field = problem.operator_coefficients(params)
        self._owned = []
        pres, _ = problem.resolve_dirichlet(params)
        m = np.zeros(problem.space.n_dofs, bool)
        m[pres] = True
        if fine_op is None:  # an operator of its own, released with this object
            fq = None if field is None else np.asarray(getattr(field, "values", field), dtype=float)
            fine_op = Operator(problem.space, problem.op, coef, prescribed=m, coef_qp=fq,
                               plane_strain=getattr(problem, "plane", "stress") == "strain")
            self._owned.append(fine_op)
        self.ops, self.spaces, self.masks, self.transfers, self.exact = [fine_op], [problem.space], [m], [], []
        coef_qp = None
        if field is not None:
            if getattr(field, "values", None) is None:
                raise NotImplementedError("multigrid takes a coefficient given as a PointField or a constant")
            coef_qp = np.asarray(field.values, dtype=float)
        self.coefs = [coef_qp]
        space = problem.space
        while space.n_dofs > max_coarse and len(self.ops) < max_levels:
            c = coarsen(space)
            if c is None:
                break
            cs, Ps, exact = c
            cpr = _coarse_problem(problem, cs)
            cpres, _ = cpr.resolve_dirichlet(params)
            cm = np.zeros(cs.n_dofs, bool)
            cm[cpres] = True
            coef_qp = coarse_coefficients(space, cs, coef_qp)
            op = Operator(cs, problem.op, coef, prescribed=cm, coef_qp=coef_qp,
                          plane_strain=getattr(problem, "plane", "stress") == "strain")
            self._owned.append(op)
            self.ops.append(op)
            self.spaces.append(cs)
            self.masks.append(cm)
            self.transfers.append(Ps)
            self.exact.append(exact)
            self.coefs.append(coef_qp)
            space = cs
        if len(self.ops) < 2:
            raise ValueError("the space is too small to coarsen: use Jacobi-PCG")
        self.coarse_inverse = dense_inverse(self.ops[-1], self.masks[-1])
        keep = []
        T = (_lib.Transfer1d * (3 * (len(self.ops) - 1)))()
        for l, Ps in enumerate(self.transfers):
            for d, P in enumerate(Ps):
                rows, cols = P.shape
                nz = [np.nonzero(P[i])[0] for i in range(rows)]
                ptr = np.zeros(rows + 1, np.int32)
                ptr[1:] = np.cumsum([len(z) for z in nz])
                idx = np.concatenate(nz).astype(np.int32)
                val = np.concatenate([P[i, z] for i, z in enumerate(nz)]).astype(np.float64)
                keep += [ptr, idx, val]
                t = T[3 * l + d]
                t.rows, t.cols = rows, cols
                t.ptr = ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
                t.idx = idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
                t.val = val.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        plans = (ctypes.c_void_p * len(self.ops))(*[op.handle.value for op in self.ops])
        ci = np.ascontiguousarray(self.coarse_inverse)
        h = ctypes.c_void_p()
        _lib.check(self.lib.jxb_mg_create(plans, len(self.ops), T, ci.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          int(degree), float(smooth_range), ctypes.byref(h)))
        self.handle = h
        self.degree, self.smooth_range = int(degree), float(smooth_range)
        lm = (ctypes.c_double * len(self.ops))()
        _lib.check(self.lib.jxb_mg_info(h, lm))
        self.lmax = list(lm)

    @property
    def levels(self):
        return len(self.ops)

    def vcycle(self, r):
        op = self.ops[0]
        r = op._vec(r)
        z = op._empty(op.n_dofs)
        _lib.check(self.lib.jxb_mg_vcycle(self.handle, _stream(), _dptr(r), _dptr(z)))
        return z

    def solve(self, b, tol=1e-8, atol=0.0, maxiter=None, check_every=8):
        """CG preconditioned by the V-cycle from x = 0 (jax CG semantics); returns (x, stats)."""
        op = self.ops[0]
        b = op._vec(b)
        x = op._empty(op.n_dofs)
        st = _lib.Stats()
        o = op._opts(tol, atol, maxiter, "jacobi", check_every, 0.0, 0)
        rc = self.lib.jxb_mg_pcg(self.handle, _stream(), _dptr(b), _dptr(x), ctypes.byref(o), ctypes.byref(st))
        _lib.check_solve(rc)
        out = {k: getattr(st, k) for k, _ in _lib.Stats._fields_}
        out["levels"] = self.levels
        return x, out

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.jxb_mg_destroy(self.handle)
            self.handle = None
        for op in self._owned:
            op.close()
        self._owned = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _workload(name, span):
    """(problem, params, load) of a benchmark workload for the multigrid timing."""
    import torch

    from . import workloads
    from .forms import PointField
    from .solve import _problem_operator, _rhs, geometry_operator

    if name == "plate":
        V, problem, params = workloads.config5(n=span)
    elif name == "darcy":
        V, problem, params = workloads.config4(n=span)
        a = torch.exp(geometry_operator(V).interpolate(params["loga"])[..., 0]).cpu().numpy()
        params = {"a0": PointField(a)}
    else:
        V, problem, params = workloads.config2(n=span)
        fq = geometry_operator(V).interpolate(params["eta"]).cpu().numpy()
        fq[..., 2] -= 1.0
        params = dict(params, f=PointField(fq))
    op, prescribed, values = _problem_operator(problem, params, False)
    return problem, params, op, _rhs(problem, params, op, prescribed, values)


if __name__ == "__main__":
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser(description="multigrid-preconditioned CG against Jacobi-PCG on a workload")
    ap.add_argument("--workload", choices=["plate", "elasticity", "darcy"], default="plate")
    ap.add_argument("--span", type=int, default=256)
    ap.add_argument("--degree", type=int, default=3)
    ap.add_argument("--range", type=float, default=20.0)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--once", action="store_true", help="one multigrid solve only (for a profiler launch list)")
    a = ap.parse_args()
    problem, params, op, b = _workload(a.workload, a.span)
    t0 = time.perf_counter()
    mg = Multigrid(problem, params, degree=a.degree, smooth_range=a.range, fine_op=op)
    setup = time.perf_counter() - t0
    mg.solve(b, tol=a.tol)  # captures the graph
    if a.once:
        mg.close()
        raise SystemExit(0)
    _, st = mg.solve(b, tol=a.tol)
    op.pcg(b, tol=a.tol, restarts=3, maxiter=80000, check_every=32)
    _, sj = op.pcg(b, tol=a.tol, restarts=3, maxiter=80000, check_every=32)
    print(json.dumps({"workload": a.workload, "span": a.span, "levels": mg.levels, "degree": a.degree,
                      "range": a.range, "setup_seconds": setup, "lmax": mg.lmax,
                      "multigrid_pcg": {k: st[k] for k in ("iterations", "seconds", "relative_residual", "converged")},
                      "jacobi_pcg": {k: sj[k] for k in ("iterations", "seconds", "relative_residual", "converged")},
                      "speedup": sj["seconds"] / st["seconds"] if st["converged"] and sj["converged"] else None}))
    mg.close()
