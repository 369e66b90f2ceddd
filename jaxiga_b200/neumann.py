"""Neumann loads: tractions or fluxes t(x, n, params) on boundary sides.

The reference adds the work of each Neumann condition to the energy
(``neumann_work``, src/jaxiga/methods/_common.py:312-318): on the boundary
Gauss set of the condition's sides (src/jaxiga/space/pointset.py:148-200),
sum_q w_q t(x_q, n_q) . u(x_q), whose negative gradient is the load
F_i,c = sum_q w_q t_c R_i. Here the points, outward normals and surface
weights come from ``jxb_boundary_points``, the user's ``t`` is evaluated on
the host at those points (it is a Python callable), and ``jxb_boundary_load``
integrates and scatters the face-local loads into F in a fixed order.

A condition's sides are a labelled boundary, or the boundary (element, side)
pairs whose physical side centre satisfies a predicate
(src/jaxiga/forms/problem.py:305-381).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .pointset import boundary_gauss
from .space import BoundarySet


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def side_centres(space, elems, sides):
    """Physical centre of the side each boundary element presents (problem.py:364-381)."""
    from .hierarchical import HierarchicalSpace
    from .solve import geometry_operator

    if isinstance(space, HierarchicalSpace):
        from .thb import side_centres as thb_side_centres

        return thb_side_centres(space, elems, sides)

    ref = np.zeros((len(elems), space.dim))
    for i, code in enumerate(sides):
        direction, end = divmod(int(code), 2)
        ref[i, direction] = -1.0 if end == 0 else 1.0
    return geometry_operator(space).eval_points(elems, ref, None, val=False, x=True)["x"].cpu().numpy()


def resolve_set(space, where):
    """BoundarySet of a Neumann condition: a label, or a predicate over side centres."""
    if isinstance(where, str):
        return space.boundary(where)
    elems, sides = [], []
    for b in space.boundaries.values():
        elems.append(np.asarray(b.elems))
        sides.append(np.asarray(b.sides))
    elems, sides = np.concatenate(elems), np.concatenate(sides)
    _, unique = np.unique(np.stack([elems, sides], axis=1), axis=0, return_index=True)
    keep = np.sort(unique)
    elems, sides = elems[keep], sides[keep]
    mask = np.asarray(where(side_centres(space, elems, sides)), dtype=bool).ravel()
    if mask.shape != elems.shape:
        raise ValueError(f"Neumann predicate returned shape {mask.shape}, expected {elems.shape} "
                         "(one bool per boundary element side centre)")
    if not mask.any():
        raise ValueError("Neumann predicate selected no boundary elements; it is evaluated at the physical "
                         "centre of each boundary element side")
    ke, ks = elems[mask], sides[mask]
    from .hierarchical import HierarchicalSpace

    if isinstance(space, HierarchicalSpace):  # padded element rows
        ed = space.elem_dofs[ke]
        return BoundarySet(ke, ks, np.unique(ed[ed < space.n_scalar_basis]))
    return BoundarySet(ke, ks, np.unique(space.element_dofs(ke)))


def _call_traction(fn, x, n, params, vec):
    """t(x, n, params) over points: vectorised over rows, else point by point."""
    m = x.shape[0]
    try:
        out = np.asarray(fn(x, n, params), dtype=float)
        if out.ndim == 0 or out.shape[0] != m:
            raise ValueError
        out = out.reshape(m, -1)
    except Exception:
        out = np.stack([np.atleast_1d(np.asarray(fn(x[i], n[i], params), dtype=float)) for i in range(m)])
    if out.shape[1] == 1 and vec > 1:
        out = np.repeat(out, vec, axis=1)
    if out.shape[1] != vec:
        raise ValueError(f"Neumann value returned {out.shape[1]} components, expected {vec}")
    return out


def boundary_points(op, ps):
    """(x, normal, w) at the points of a boundary PointSet, device tensors."""
    import torch

    dim, nf, nq = op.space.dim, ps.n_elems, ps.n_q
    dev = op.device
    e = torch.as_tensor(ps.elems, dtype=torch.int64, device=dev)
    sides = torch.as_tensor(ps.sides, dtype=torch.int32, device=dev)
    ref = torch.as_tensor(ps.ref.reshape(-1, dim), dtype=torch.float64, device=dev).contiguous()
    wref = torch.as_tensor(ps.weights.reshape(-1), dtype=torch.float64, device=dev).contiguous()
    x = torch.empty(max(nf * nq * dim, 1), dtype=torch.float64, device=dev)
    nrm = torch.empty_like(x)
    w = torch.empty(max(nf * nq, 1), dtype=torch.float64, device=dev)
    _lib.check(op.lib.jxb_boundary_points(op.handle, _stream(), nf, nq, _dptr(e), _dptr(sides), _dptr(ref),
                                          _dptr(wref), _dptr(x), _dptr(nrm), _dptr(w)))
    n = nf * nq
    return x[: n * dim].view(n, dim), nrm[: n * dim].view(n, dim), w[:n], (e, ref)


def neumann_load(op, problem, params, F=None):
    """F (device, full length) plus the loads of every Neumann condition of ``problem``."""
    import torch

    space = problem.space
    vec = space.vec
    F = torch.zeros(space.n_dofs, dtype=torch.float64, device=op.device) if F is None else F
    if hasattr(op, "patch_ops"):  # multipatch: patch by patch through the numbering
        from .multipatch import neumann_load_multipatch

        return neumann_load_multipatch(op, problem, params, F)
    from .hierarchical import HierarchicalSpace

    if isinstance(space, HierarchicalSpace):
        from .thb import neumann_load as thb_neumann_load

        return thb_neumann_load(op, problem, params, F)
    for bc in problem.neumann:
        bset = resolve_set(space, bc.where)
        ps = boundary_gauss(space, bset, problem.quadrature)
        if ps.n_elems == 0:
            continue
        x, nrm, w, (e, ref) = boundary_points(op, ps)
        t = _call_traction(bc.value, x.cpu().numpy(), nrm.cpu().numpy(), params, vec)
        t = torch.as_tensor(np.ascontiguousarray(t), device=op.device)
        # deterministic scatter: per scalar DOF its (face, local function) entries in order
        ed = space.element_dofs(ps.elems).reshape(-1)
        order = np.argsort(ed, kind="stable")
        dofs, starts = np.unique(ed[order], return_index=True)
        ptr = np.append(starts, len(order)).astype(np.int64)
        dev = op.device
        d_dofs = torch.as_tensor(dofs.astype(np.int64), device=dev)
        d_ptr = torch.as_tensor(ptr, device=dev)
        d_contrib = torch.as_tensor(order.astype(np.int64), device=dev)
        local = torch.empty(ps.n_elems * space.n_local * vec, dtype=torch.float64, device=dev)
        _lib.check(op.lib.jxb_boundary_load(op.handle, _stream(), ps.n_elems, ps.n_q, _dptr(e), _dptr(ref), _dptr(w),
                                            _dptr(t), len(dofs), _dptr(d_dofs), _dptr(d_ptr), _dptr(d_contrib),
                                            _dptr(local), _dptr(F)))
    return F
