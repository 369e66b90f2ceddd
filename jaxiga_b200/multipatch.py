"""Conforming multipatch spaces: interface detection, global numbering, boundaries.

Host setup (NumPy), the counterpart of src/jaxiga/geometry/multipatch.py:441-580
(``compute_topology``) and src/jaxiga/space/function_space.py:372-535
(``build_function_space`` for several patches). Patches are glued only along
*verified* interfaces (multipatch.py module docstring):

1. the two sides carry the same number of control points;
2. the points coincide as sets within ``tol``;
3. the matching is a legal reorientation of the side grid (flips of its
   tangential directions, in 3D possibly a transpose), not a shuffle;
4. the tangential knot vectors agree under that reorientation;
5. the NURBS weights agree at matched points;
6. the outward normals are antiparallel (the patches lie on opposite sides).

Control points that coincide only at corners (2D) or along edges (3D) of the
patches are merged as contacts; any other coincidence raises
``NonConformingError``. The device side keeps one libjxb plan per patch and
a composite plan that gathers each patch's DOFs from the global vector and
sums the patches' contributions back in a fixed order (``jxb_mp_create``).
"""

from __future__ import annotations

import dataclasses
from functools import cached_property

import numpy as np

from .geometry import TOL, Patch, side_name

try:  # SciPy's KD-tree for coincident points (the reference uses the same)
    from scipy.spatial import cKDTree
except Exception:  # pragma: no cover
    cKDTree = None


class NonConformingError(Exception):
    """Two patches meet along an interface whose discretizations do not match."""


class OrientationError(Exception):
    """Two patches meet with inconsistent orientation."""


@dataclasses.dataclass(frozen=True)
class Interface:
    patch_a: int
    side_a: str
    patch_b: int
    side_b: str
    reversed: bool = False


@dataclasses.dataclass(frozen=True)
class Topology:
    local_to_global: tuple  # one (n_cp_patch,) int array per patch
    n_global_dofs: int = 0
    interfaces: tuple = ()

    def patch_dofs(self, i):
        return self.local_to_global[i]


def _side_grid(patch, side):
    """Local control-point indices of a side as a grid over its tangential
    directions (first tangential direction fastest)."""
    n = patch.n_cp_per_dir
    d = "uvw".index(side[0])
    fixed = 0 if side[1] == "0" else n[d] - 1
    grid = np.arange(patch.n_cp).reshape(n[::-1])  # [.., v, u] (u fastest)
    axis = patch.dim - 1 - d
    face = np.take(grid, fixed, axis=axis)  # tangential axes in reversed order
    return face.T  # [t0, t1] with t0 the lower tangential direction


def _tangential_dirs(dim, d):
    return [k for k in range(dim) if k != d]


def _outward_normal(patch, side):
    """Outward direction of a side at its centre: from the second control-point
    layer towards the side (exact for the sign test of step 6)."""
    d = "uvw".index(side[0])
    end = int(side[1])
    n = patch.n_cp_per_dir
    grid = np.arange(patch.n_cp).reshape(n[::-1])
    axis = patch.dim - 1 - d
    on = np.take(grid, 0 if end == 0 else n[d] - 1, axis=axis).ravel()
    inner = np.take(grid, 1 if end == 0 else n[d] - 2, axis=axis).ravel()
    v = patch.ctrl_pts[on].mean(axis=0) - patch.ctrl_pts[inner].mean(axis=0)
    nv = np.linalg.norm(v)
    return v / nv if nv > 0 else v


def _corners(patch, g):
    """Corner control points of a side grid."""
    idx = [g[0], g[-1]] if g.ndim == 1 else [g[0, 0], g[0, -1], g[-1, 0], g[-1, -1]]
    return patch.ctrl_pts[np.asarray(idx)]


def _reorientations(gb):
    """Legal reorientations of a side grid: (transposed, flips per axis, grid)."""
    if gb.ndim == 1:
        yield False, (0,), gb
        yield False, (1,), gb[::-1]
        return
    for tr in (False, True):
        g = gb.T if tr else gb
        for f0 in (0, 1):
            for f1 in (0, 1):
                h = g[::-1, :] if f0 else g
                h = h[:, ::-1] if f1 else h
                yield tr, (f0, f1), h


def _verify(patches, pa, sa, pb, sb, tol):
    """The checks of the module docstring for side sa of patch pa against side sb
    of patch pb; returns (Interface, b's local indices matched to a's side
    points in order) or None when the sides do not touch as a whole."""
    A, B = patches[pa], patches[pb]
    ga, gb = _side_grid(A, sa), _side_grid(B, sb)
    xa, xb = A.ctrl_pts[ga.ravel()], B.ctrl_pts[gb.ravel()]
    scale = max(1.0, float(np.abs(np.concatenate([xa, xb])).max()))
    atol = tol * scale
    if ga.size != gb.size or not np.allclose(np.sort(xa, axis=0), np.sort(xb, axis=0), atol=atol, rtol=0):
        # no whole-side match; but two sides with the same corners cover the same
        # face, discretized differently (refinement, degree)
        ca, cb = _corners(A, ga), _corners(B, gb)
        if len(ca) == len(cb) and all(np.linalg.norm(cb - c, axis=1).min() <= atol for c in ca):
            raise NonConformingError(f"patches {pa} and {pb} meet along {sa}/{sb}, but their control nets on it "
                                     "differ (different refinement or degree)")
        return None
    ta = _tangential_dirs(A.dim, "uvw".index(sa[0]))
    tb = _tangential_dirs(B.dim, "uvw".index(sb[0]))
    for tr, flips, h in _reorientations(gb):
        if h.shape != ga.shape or not np.allclose(xa, B.ctrl_pts[h.ravel()], atol=atol, rtol=0):
            continue
        for axa in range(len(ta)):  # step 4: tangential knots and degrees under the reorientation
            axb = 1 - axa if tr else axa
            ka = np.asarray(A.knots[ta[axa]], dtype=float)
            kb = np.asarray(B.knots[tb[axb]], dtype=float)
            if flips[axa]:
                kb = kb[0] + kb[-1] - kb[::-1]
            ka = (ka - ka[0]) / (ka[-1] - ka[0])
            kb = (kb - kb[0]) / (kb[-1] - kb[0])
            if A.degree[ta[axa]] != B.degree[tb[axb]] or len(ka) != len(kb) or not np.allclose(ka, kb, atol=1e-10):
                raise NonConformingError(f"patches {pa} and {pb} meet along {sa}/{sb} with different knot "
                                         "vectors or degrees")
        if not np.allclose(A.weights[ga.ravel()], B.weights[h.ravel()], atol=max(tol, 1e-12), rtol=0):
            raise NonConformingError(f"patches {pa} and {pb} assign different NURBS weights on {sa}/{sb}")
        if float(_outward_normal(A, sa) @ _outward_normal(B, sb)) >= 0:
            raise NonConformingError(f"patches {pa} and {pb} overlap along {sa}/{sb}: their outward normals agree")
        return Interface(pa, sa, pb, sb, reversed=bool(tr or any(flips))), h.ravel()
    raise OrientationError(f"patches {pa} and {pb} share the points of {sa}/{sb} in an order that no "
                           "reorientation of the side explains")


def _on_feature(patch):
    """Local control points on at least two sides (corners, edges in 3D)."""
    n = patch.n_cp_per_dir
    idx = np.indices(n[::-1]).reshape(patch.dim, -1)[::-1]
    count = np.zeros(patch.n_cp, dtype=int)
    for d in range(patch.dim):
        count += (idx[d] == 0) | (idx[d] == n[d] - 1)
    return count >= 2


def compute_topology(patches, tol: float = TOL) -> Topology:
    """Conforming global numbering of a patch collection (multipatch.py:441-580)."""
    patches = list(patches)
    n_cp = [p.n_cp for p in patches]
    offsets = np.concatenate([[0], np.cumsum(n_cp)]).astype(np.int64)
    all_pts = np.concatenate([np.asarray(p.ctrl_pts, dtype=float) for p in patches])
    all_w = np.concatenate([np.asarray(p.weights, dtype=float) for p in patches])
    patch_of = np.concatenate([np.full(n, i) for i, n in enumerate(n_cp)])
    parent = np.arange(len(all_pts))

    def find(i):
        while parent[i] != i:
            parent[i] = parent[parent[i]]
            i = parent[i]
        return i

    def union(i, j):
        ri, rj = find(i), find(j)
        if ri != rj:
            parent[max(ri, rj)] = min(ri, rj)

    sides = [(i, side_name(d, e)) for i, p in enumerate(patches) for d in range(p.dim) for e in (0, 1)]
    boxes = []
    for i, s in sides:
        pts = patches[i].ctrl_pts[_side_grid(patches[i], s).ravel()]
        boxes.append((pts.min(axis=0), pts.max(axis=0)))
    span = float(np.ptp(all_pts, axis=0).max()) if len(all_pts) else 1.0
    cut = max(tol, 1e-12) * 10 + 1e-9 * max(span, 1.0)
    interfaces, explained = [], set()
    for a in range(len(sides)):
        for b in range(a + 1, len(sides)):
            (pa, sa), (pb, sb) = sides[a], sides[b]
            if pa == pb:
                continue
            if np.any(boxes[a][0] > boxes[b][1] + cut) or np.any(boxes[b][0] > boxes[a][1] + cut):
                continue
            v = _verify(patches, pa, sa, pb, sb, tol)
            if v is None:
                continue
            iface, matched = v
            interfaces.append(iface)
            for la, lb in zip(_side_grid(patches[pa], sa).ravel(), matched):
                gi, gj = int(offsets[pa] + la), int(offsets[pb] + lb)
                union(gi, gj)
                explained.add((min(gi, gj), max(gi, gj)))
    feature = np.concatenate([_on_feature(p) for p in patches])
    if len(patches) > 1:
        if cKDTree is not None:
            pairs = cKDTree(all_pts).query_pairs(r=max(tol, 1e-12))
        else:  # pragma: no cover
            pairs = {(i, j) for i in range(len(all_pts)) for j in range(i + 1, len(all_pts))
                     if np.linalg.norm(all_pts[i] - all_pts[j]) <= max(tol, 1e-12)}
        for i, j in sorted(pairs):
            if patch_of[i] == patch_of[j] or (min(i, j), max(i, j)) in explained or find(i) == find(j):
                continue
            if feature[i] and feature[j]:
                if abs(all_w[i] - all_w[j]) > max(tol, 1e-12):
                    raise NonConformingError(f"patches {patch_of[i]} and {patch_of[j]} touch at {all_pts[i]} "
                                             "with different NURBS weights")
                union(i, j)
                continue
            raise NonConformingError(f"patches {patch_of[i]} and {patch_of[j]} share the control point "
                                     f"{all_pts[i]} inside a face without a verified interface (overlapping or "
                                     "partly abutting patches)")
    roots = np.array([find(i) for i in range(len(all_pts))])
    _, gidx = np.unique(roots, return_inverse=True)
    n_global = int(gidx.max()) + 1 if len(gidx) else 0
    l2g = tuple(gidx[offsets[i]:offsets[i + 1]].astype(np.int64) for i in range(len(patches)))
    return Topology(local_to_global=l2g, n_global_dofs=n_global, interfaces=tuple(interfaces))


class BoundarySet:
    def __init__(self, elems, sides, dofs):
        self.elems = np.asarray(elems, dtype=np.int64)
        self.sides = np.asarray(sides, dtype=np.int64)
        self.dofs = np.asarray(dofs, dtype=np.int64)

    def __len__(self):
        return len(self.elems)


class MultiPatchSpace:
    """A function space over several conforming patches (function_space.py:372-535).

    Global scalar basis numbered by ``topology``; DOF of component c of basis i
    at vec*i + c; elements numbered patch by patch, each patch's first
    direction fastest. ``spaces[i]`` is patch i's single-patch space.
    """

    def __init__(self, patches, vec: int = 1, tol: float = TOL):
        from .space import FunctionSpace

        patches = list(patches)
        if not patches or not all(isinstance(p, Patch) for p in patches):
            raise TypeError("MultiPatchSpace expects a list of Patch")
        degree = patches[0].degree
        for i, p in enumerate(patches):
            if p.degree != degree or p.dim != patches[0].dim:
                raise ValueError(f"all patches must share a degree and dimension: patch 0 has {degree}, "
                                 f"patch {i} has {p.degree}. Elevate them to a common degree.")
        self.patches = patches
        self.topology = compute_topology(patches, tol)
        self.vec = int(vec)
        self.dim = patches[0].dim
        self.degree = tuple(degree)
        self.spaces = [FunctionSpace(p, vec=vec) for p in patches]
        self.n_scalar_basis = self.topology.n_global_dofs
        self.n_elems = int(sum(s.n_elems for s in self.spaces))
        self.elem_offsets = np.concatenate([[0], np.cumsum([s.n_elems for s in self.spaces])]).astype(np.int64)
        self.n_local = self.spaces[0].n_local
        self.cell_type = "tensor"
        cpts = np.full((self.n_scalar_basis, patches[0].dim_phys), np.nan)
        wgts = np.full(self.n_scalar_basis, np.nan)
        for i, p in enumerate(patches):
            g = self.topology.local_to_global[i]
            seen = ~np.isnan(wgts[g])
            if np.any(seen):
                dev = max(np.abs(cpts[g][seen] - p.ctrl_pts[seen]).max(initial=0.0),
                          np.abs(wgts[g][seen] - p.weights[seen]).max(initial=0.0))
                if dev > TOL:
                    raise ValueError(f"patch {i} disagrees with an earlier patch about shared control data by {dev:.3e}")
            cpts[g] = p.ctrl_pts
            wgts[g] = p.weights
        self.cpts, self.wgts = cpts, wgts
        self._plans = {}

    @property
    def n_dofs(self) -> int:
        return self.n_scalar_basis * self.vec

    @property
    def dim_phys(self) -> int:
        return self.cpts.shape[1]

    @cached_property
    def elem_dofs(self) -> np.ndarray:
        return np.concatenate([self.topology.local_to_global[i][s.elem_dofs] for i, s in enumerate(self.spaces)])

    def element_dofs(self, elems) -> np.ndarray:
        """Global scalar DOFs of the given (global) elements, (len(elems), (p+1)^dim)."""
        elems = np.asarray(elems, dtype=np.int64).reshape(-1)
        patch = np.searchsorted(self.elem_offsets, elems, side="right") - 1
        out = np.zeros((len(elems), self.n_local), dtype=np.int64)
        for i, s in enumerate(self.spaces):
            sel = patch == i
            if sel.any():
                out[sel] = self.topology.local_to_global[i][s.element_dofs(elems[sel] - self.elem_offsets[i])]
        return out

    def elem_dofs_vec(self):
        from .space import expand_dofs

        return expand_dofs(self.elem_dofs, self.vec)

    @cached_property
    def boundaries(self) -> dict:
        """label -> BoundarySet over the sides not glued to another patch;
        unlabelled sides get ``patch{i}/<side>`` (function_space.py:490-535)."""
        inner = {(f.patch_a, f.side_a) for f in self.topology.interfaces}
        inner |= {(f.patch_b, f.side_b) for f in self.topology.interfaces}
        out = {}
        for i, (p, s) in enumerate(zip(self.patches, self.spaces)):
            labels = p.label_map
            for d in range(self.dim):
                for e in (0, 1):
                    side = side_name(d, e)
                    if (i, side) in inner:
                        continue
                    label = labels.get(side, f"patch{i}/{side}")
                    entry = out.setdefault(label, ([], [], []))
                    entry[0].append(s._side_elements(d, e) + self.elem_offsets[i])
                    entry[1].append(np.full(len(s._side_elements(d, e)), 2 * d + e))
                    entry[2].append(self.topology.local_to_global[i][s.side_indices(side)])
        return {k: BoundarySet(np.concatenate(v[0]), np.concatenate(v[1]), np.unique(np.concatenate(v[2])))
                for k, v in out.items()}

    def boundary(self, label: str) -> BoundarySet:
        if label not in self.boundaries:
            raise KeyError(f"unknown boundary label {label!r}; available: {sorted(self.boundaries)}")
        return self.boundaries[label]

    def sides_of_label(self, label: str):
        return []

    def summary(self) -> str:
        return (f"MultiPatchSpace(patches={len(self.patches)}, dim={self.dim}, vec={self.vec}, degree={self.degree}, "
                f"n_elems={self.n_elems}, n_scalar_basis={self.n_scalar_basis}, "
                f"interfaces={len(self.topology.interfaces)})")


class MultiPatchOperator:
    """The composite device operator of a multipatch problem: one libjxb plan per
    patch (no Dirichlet mask) and a composite plan (``jxb_mp_create``) gluing
    them; it offers the single-patch ``Operator``'s apply, diagonal, load, dot
    and Jacobi-PCG on the global DOF vector."""

    def __init__(self, space, op="poisson", coef=(1.0,), prescribed=None, coef_qp=None, want_f32=False,
                 plane_strain=False):
        import ctypes

        import torch

        from . import _lib
        from .operator import Operator

        if want_f32:
            raise NotImplementedError("multipatch operators run in FP64")
        if not torch.cuda.is_available():
            raise RuntimeError("the B200 solver needs a CUDA device; none is visible")
        self.lib = _lib.load()
        self.space, self.op, self.vec = space, op, space.vec
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.want_f32, self.tile = False, None
        nqe = int(np.prod([p + 1 for p in space.degree]))
        self.nqe = nqe
        cq = None if coef_qp is None else np.asarray(coef_qp, dtype=float).reshape(space.n_elems, nqe)
        self.patch_ops = []
        for i, s in enumerate(space.spaces):
            part = None if cq is None else cq[space.elem_offsets[i]:space.elem_offsets[i + 1]]
            self.patch_ops.append(Operator(s, op, coef, coef_qp=part, plane_strain=plane_strain))
        self._maps = [np.ascontiguousarray(m, dtype=np.int64) for m in space.topology.local_to_global]
        ptrs = (ctypes.c_void_p * len(self._maps))(*[m.ctypes.data for m in self._maps])
        plans = (ctypes.c_void_p * len(self.patch_ops))(*[o.handle.value for o in self.patch_ops])
        pm = None
        if prescribed is not None:
            pm = np.ascontiguousarray(np.asarray(prescribed).astype(np.uint8))
            if pm.size != space.n_dofs:
                raise ValueError("prescribed mask must have n_dofs entries")
        self.prescribed_mask = (np.zeros(space.n_dofs, bool) if prescribed is None
                                else np.asarray(prescribed).astype(bool).copy())
        h = ctypes.c_void_p()
        _lib.check(self.lib.jxb_mp_create(plans, len(self.patch_ops), ptrs, int(space.n_scalar_basis),
                                          None if pm is None else pm.ctypes.data, ctypes.byref(h)))
        self.handle = h
        info = _lib.Info()
        _lib.check(self.lib.jxb_plan_info(h, ctypes.byref(info)))
        self.info = {k: getattr(info, k) for k, _ in _lib.Info._fields_}
        self.n_dofs = info.n_dofs
        self.n_qp = info.n_qp

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.jxb_plan_destroy(self.handle)
            self.handle = None
        for o in getattr(self, "patch_ops", []):
            o.close()
        self.patch_ops = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _bind_operator_methods():
    """The single-patch Operator's device methods that work on a composite plan."""
    from .operator import Operator

    for name in ("_vec", "_empty", "apply", "diag", "load", "dot", "_opts", "pcg", "bicgstab"):
        setattr(MultiPatchOperator, name, getattr(Operator, name))


_bind_operator_methods()


class MultiPatchGeometry:
    """Gauss-point coordinates, weights and interpolation of global fields on a
    multipatch space, patch by patch (elements in patch order)."""

    def __init__(self, space):
        import torch

        from .solve import geometry_operator

        self.space = space
        self.ops = [geometry_operator(s) for s in space.spaces]
        self._idx = [torch.as_tensor(m, dtype=torch.int64, device=self.ops[0].device)
                     for m in space.topology.local_to_global]

    def qp_coords(self):
        import torch

        return torch.cat([o.qp_coords() for o in self.ops])

    def qp_weights(self):
        import torch

        return torch.cat([o.qp_weights() for o in self.ops])

    def _local(self, coef, i):
        import torch

        c = torch.as_tensor(coef, dtype=torch.float64, device=self.ops[0].device).contiguous()
        ncomp = c.numel() // self.space.n_scalar_basis
        if ncomp * self.space.n_scalar_basis != c.numel():
            raise ValueError("coefficient field must have n_scalar_basis * ncomp entries")
        return c.view(-1, ncomp)[self._idx[i]].reshape(-1)

    def interpolate(self, coef):
        import torch

        return torch.cat([o.interpolate(self._local(coef, i)) for i, o in enumerate(self.ops)])

    def interpolate_grad(self, coef):
        import torch

        return torch.cat([o.interpolate_grad(self._local(coef, i)) for i, o in enumerate(self.ops)])

    def eval_points(self, elems, ref, coef=None, val=True, grad=False, x=False, jac=False):
        """Evaluation at (global element, reference point) pairs, patch by patch,
        outputs in the order of the pairs."""
        import torch

        elems = np.asarray(elems, dtype=np.int64).reshape(-1)
        ref = np.asarray(ref, dtype=float).reshape(len(elems), -1)
        off = self.space.elem_offsets
        patch = np.searchsorted(off, elems, side="right") - 1
        out = {}
        for i, o in enumerate(self.ops):
            sel = np.flatnonzero(patch == i)
            if len(sel) == 0:
                continue
            c = None if coef is None else self._local(coef, i)
            r = o.eval_points(elems[sel] - off[i], ref[sel], c, val=val, grad=grad, x=x, jac=jac)
            idx = torch.as_tensor(sel, device=o.device)
            for k, v in r.items():
                if k not in out:
                    out[k] = torch.empty((len(elems),) + tuple(v.shape[1:]), dtype=v.dtype, device=v.device)
                out[k][idx] = v
        return out


def neumann_load_multipatch(op, problem, params, F):
    """Neumann loads on a multipatch space: each condition's boundary faces split
    by patch, integrated with the patch's plan (``jxb_boundary_load``), and the
    patch vectors added into the global one through the numbering on the host,
    patch after patch (a fixed order)."""
    import torch

    from .neumann import _call_traction, boundary_points, resolve_set
    from .pointset import boundary_gauss

    space = problem.space
    vec = space.vec
    off = space.elem_offsets
    total = np.zeros(space.n_dofs)
    for bc in problem.neumann:
        bset = resolve_set(space, bc.where)
        patch = np.searchsorted(off, bset.elems, side="right") - 1
        for i, (sub, pop) in enumerate(zip(space.spaces, op.patch_ops)):
            sel = patch == i
            if not sel.any():
                continue
            e = bset.elems[sel] - off[i]
            local = BoundarySet(e, bset.sides[sel], np.unique(sub.element_dofs(e)))
            ps = boundary_gauss(sub, local, problem.quadrature)
            if ps.n_elems == 0:
                continue
            x, nrm, w, (de, ref) = boundary_points(pop, ps)
            t = _call_traction(bc.value, x.cpu().numpy(), nrm.cpu().numpy(), params, vec)
            Fi = _patch_boundary_load(pop, sub, ps, de, ref, w, t)
            g = space.topology.local_to_global[i]
            gd = (g[:, None] * vec + np.arange(vec)[None, :]).reshape(-1)
            total[gd] += Fi.cpu().numpy()
    return F + torch.as_tensor(total, device=F.device)


def _patch_boundary_load(pop, sub, ps, de, ref, w, t):
    """The load of given traction values t at a patch's boundary Gauss points."""
    import torch

    from . import _lib
    from .neumann import _dptr, _stream

    vec = sub.vec
    dev = pop.device
    ed = sub.element_dofs(ps.elems).reshape(-1)
    order = np.argsort(ed, kind="stable")
    dofs, starts = np.unique(ed[order], return_index=True)
    ptr = np.append(starts, len(order)).astype(np.int64)
    d_dofs = torch.as_tensor(dofs.astype(np.int64), device=dev)
    d_ptr = torch.as_tensor(ptr, device=dev)
    d_contrib = torch.as_tensor(order.astype(np.int64), device=dev)
    tt = torch.as_tensor(np.ascontiguousarray(t), device=dev)
    local = torch.empty(ps.n_elems * sub.n_local * vec, dtype=torch.float64, device=dev)
    Fi = torch.zeros(sub.n_dofs, dtype=torch.float64, device=dev)
    _lib.check(pop.lib.jxb_boundary_load(pop.handle, _stream(), ps.n_elems, ps.n_q, _dptr(de), _dptr(ref), _dptr(w),
                                         _dptr(tt), len(dofs), _dptr(d_dofs), _dptr(d_ptr), _dptr(d_contrib),
                                         _dptr(local), _dptr(Fi)))
    return Fi
