"""Single-patch function spaces (host setup stage).

Mirrors ``src/jaxiga/space/function_space.py`` for one tensor-product NURBS
patch, plus the univariate pieces of ``src/jaxiga/space/bernstein.py`` and the
Gauss rule of ``src/jaxiga/space/pointset.py``.

Unlike the reference, no dense ``(n_elem, (p+1)^d, (p+1)^d)`` Kronecker
extraction or ``(n_elem, n_local)`` connectivity is materialised up front: the
device kernels need only the per-direction operators and first-basis indices.
``extraction`` and ``elem_dofs`` are still available, computed on demand with
the reference's numbering (first direction fastest, ``kron(C_w, C_v, C_u)``).
"""

from __future__ import annotations

from functools import cached_property

import numpy as np


def bezier_extraction(knot, deg):
    """Bezier extraction operators of a univariate B-spline, one per non-empty span.

    Borden, Scott, Evans & Hughes, "Isogeometric finite element data
    structures based on Bezier extraction" (IJNME 2011), Algorithm 1 -- the
    algorithm of src/jaxiga/space/bernstein.py:16-76, computed with the same
    floating-point operations so the operators agree bit for bit. Operator
    ``C_e`` maps the span's Bernstein polynomials to its B-splines, N = C_e B.
    """
    U = np.asarray(knot, dtype=float)
    m = len(U) - deg - 1          # number of basis functions
    ops = [np.eye(deg + 1)]
    a, b = deg + 1, deg + 2       # 1-based knot positions bracketing the current span
    while b <= m:
        ops.append(np.eye(deg + 1))
        cur = ops[-2]
        start = b
        while b <= m and U[b] == U[b - 1]:
            b += 1
        mult = b - start + 1
        if mult < deg:
            r = deg - mult
            numer = U[b - 1] - U[a - 1]
            alphas = [0.0] * r
            for j in range(deg, mult, -1):
                alphas[j - mult - 1] = numer / (U[a + j - 1] - U[a - 1])
            for j in range(1, r + 1):
                s = mult + j
                for k in range(deg, s - 1, -1):      # columns deg .. s (0-based k)
                    alpha = alphas[k - s]
                    cur[:, k] = alpha * cur[:, k] + (1 - alpha) * cur[:, k - 1]
                if b <= m:
                    save = r - j                      # 0-based column of the next operator
                    ops[-1][save: save + j + 1, save] = cur[deg - j: deg + 1, deg]
            if b <= m:
                a, b = b, b + 1
        elif mult == deg:
            if b <= m:
                a, b = b, b + 1
        else:
            ops.pop()
            break
    if len(ops) > len(element_spans(U, deg)[0]):
        ops = ops[: len(element_spans(U, deg)[0])]
    return ops


def element_spans(knot, deg):
    """Non-empty spans ``(lo, hi)`` and first supported basis index ``i - deg``.

    src/jaxiga/space/bernstein.py:261-284 (``i`` indexes the full knot vector).
    """
    U = np.asarray(knot, dtype=float)
    i = np.flatnonzero(U[1:] > U[:-1])
    return U[i], U[i + 1], (i - deg).astype(np.int64)


def bernstein_basis(uhat, deg):
    """Bernstein polynomials on [-1, 1] (bernstein.py:79-97)."""
    uhat = np.atleast_1d(np.asarray(uhat, dtype=float))
    B = np.zeros((len(uhat), deg + 1))
    B[:, 0] = 1.0
    for j in range(1, deg + 1):
        saved = np.zeros(len(uhat))
        for k in range(j):
            temp = B[:, k].copy()
            B[:, k] = saved + (1 - uhat) * temp
            saved = (1 + uhat) * temp
        B[:, j] = saved
    return B / 2.0**deg


def gauss_1d(n: int):
    """Gauss-Legendre nodes and weights on [-1, 1] (pointset.py:98-101)."""
    return np.polynomial.legendre.leggauss(int(n))


def expand_dofs(scalar_dofs, vec: int) -> np.ndarray:
    """Component c of scalar basis i is DOF ``vec*i + c`` (function_space.py:300-312)."""
    scalar_dofs = np.asarray(scalar_dofs)
    if vec == 1:
        return scalar_dofs
    out = vec * scalar_dofs[..., :, None] + np.arange(vec)
    return out.reshape(*scalar_dofs.shape[:-1], -1)


class BoundarySet:
    """Elements, sides and scalar DOFs of one labelled side (function_space.py:147-156)."""

    def __init__(self, elems, sides, dofs):
        self.elems = np.asarray(elems, dtype=np.int64)
        self.sides = np.asarray(sides, dtype=np.int64)
        self.dofs = np.asarray(dofs, dtype=np.int64)

    def __len__(self):
        return len(self.elems)


class FunctionSpace:
    """Global NURBS basis over one patch (function_space.py:182-274, 372-454).

    ``FunctionSpace(patch, vec=1)``; a one-element list of patches is also
    accepted; a list of several conforming patches gives a ``MultiPatchSpace``.
    """

    def __new__(cls, patches=None, vec: int = 1):
        # several patches: a conforming multipatch space (multipatch.py)
        if isinstance(patches, (list, tuple)) and len(patches) > 1:
            from .multipatch import MultiPatchSpace

            return MultiPatchSpace(patches, vec=vec)
        return super().__new__(cls)

    def __init__(self, patches, vec: int = 1):
        from .geometry import Patch

        if isinstance(patches, (list, tuple)):
            if len(patches) != 1:
                raise ValueError("internal error: a multipatch list reached the single-patch space")
            patches = patches[0]
        if not isinstance(patches, Patch):
            raise TypeError("FunctionSpace expects a Patch")
        degs = set(patches.degree)
        if len(degs) != 1:
            raise NotImplementedError(
                f"the B200 backend needs equal degrees in every direction, got {patches.degree}; "
                "elevate the patch first")
        self.patch = patches
        self.vec = int(vec)
        self.dim = patches.dim
        self.degree = tuple(patches.degree)
        self.knots = patches.knot_arrays()
        self.cpts = np.asarray(patches.ctrl_pts, dtype=float)
        self.wgts = np.asarray(patches.weights, dtype=float)
        self.n_cp = list(patches.n_cp_per_dir)
        self.n_scalar_basis = int(np.prod(self.n_cp))
        spans = [element_spans(self.knots[d], self.degree[d]) for d in range(self.dim)]
        self.span_lo = [s[0] for s in spans]
        self.span_hi = [s[1] for s in spans]
        self.first = [s[2] for s in spans]
        self.n_span = [len(s[0]) for s in spans]
        self.ext1d = [np.stack(bezier_extraction(self.knots[d], self.degree[d])) for d in range(self.dim)]
        for d in range(self.dim):
            if self.ext1d[d].shape[0] != self.n_span[d]:
                raise ValueError("internal error: extraction operators do not match the spans")
        self.n_elems = int(np.prod(self.n_span))
        self.n_local = int(np.prod([p + 1 for p in self.degree]))
        self.cell_type = "tensor"
        self._plans = {}

    # -- sizes -------------------------------------------------------------
    @property
    def n_dofs(self) -> int:
        return self.n_scalar_basis * self.vec

    @property
    def dim_phys(self) -> int:
        return self.cpts.shape[1]

    # -- connectivity, on demand ---------------------------------------------
    @cached_property
    def elem_index(self):
        """(dim, n_elem) per-direction span index, first direction fastest."""
        return np.indices(self.n_span[::-1]).reshape(self.dim, -1)[::-1].copy()

    @cached_property
    def elem_dofs(self) -> np.ndarray:
        """(n_elem, (p+1)^dim) scalar DOFs per element (function_space.py:326-369)."""
        idx = self.elem_index
        strides = np.array([1, *np.cumprod(self.n_cp[:-1])], dtype=np.int64)
        local = np.indices([p + 1 for p in self.degree[::-1]]).reshape(self.dim, -1)[::-1]
        ien = np.zeros((self.n_elems, self.n_local), dtype=np.int64)
        for d in range(self.dim):
            ien += (self.first[d][idx[d]][:, None] + local[d][None, :]) * strides[d]
        return ien

    def element_dofs(self, elems) -> np.ndarray:
        """Scalar DOFs of the given elements only, (len(elems), (p+1)^dim) (function_space.py:326-369)."""
        elems = np.asarray(elems, dtype=np.int64).reshape(-1)
        strides = np.array([1, *np.cumprod(self.n_cp[:-1])], dtype=np.int64)
        local = np.indices([p + 1 for p in self.degree[::-1]]).reshape(self.dim, -1)[::-1]
        out = np.zeros((len(elems), self.n_local), dtype=np.int64)
        rest = elems.copy()
        for d in range(self.dim):
            idx = rest % self.n_span[d]
            rest //= self.n_span[d]
            out += (np.asarray(self.first[d])[idx][:, None] + local[d][None, :]) * strides[d]
        return out

    @cached_property
    def elem_vertex(self) -> np.ndarray:
        idx = self.elem_index
        boxes = np.zeros((self.n_elems, 2 * self.dim))
        for d in range(self.dim):
            boxes[:, d] = self.span_lo[d][idx[d]]
            boxes[:, self.dim + d] = self.span_hi[d][idx[d]]
        return boxes

    def extraction(self, elems=None) -> np.ndarray:
        """Dense Kronecker extraction operators for ``elems`` (all when None)."""
        elems = np.arange(self.n_elems) if elems is None else np.atleast_1d(elems)
        idx = self.elem_index
        out = np.empty((len(elems), self.n_local, self.n_local))
        for j, e in enumerate(elems):
            C = self.ext1d[-1][idx[-1][e]]
            for d in range(self.dim - 2, -1, -1):
                C = np.kron(C, self.ext1d[d][idx[d][e]])
            out[j] = C
        return out

    def elem_dofs_vec(self) -> np.ndarray:
        return expand_dofs(self.elem_dofs, self.vec)

    # -- boundaries ------------------------------------------------------------
    def side_indices(self, side: str, offset: int = 0) -> np.ndarray:
        """Control points on a side, ``offset`` layers inward (multipatch.py:99-131)."""
        direction = "uvw".index(side[0])
        end = int(side[1:])
        n = self.n_cp
        if not 0 <= offset < n[direction]:
            raise ValueError(f"offset {offset} is outside the {n[direction]} control points along direction {direction}")
        fixed = offset if end == 0 else n[direction] - 1 - offset
        strides = np.array([1, *np.cumprod(n[:-1])], dtype=np.int64)
        ranges = [np.arange(k) for k in n]
        ranges[direction] = np.array([fixed])
        mesh = np.meshgrid(*ranges, indexing="ij")
        return sum(m.ravel(order="F") * strides[d] for d, m in enumerate(mesh)).astype(np.int64)

    def _side_elements(self, direction, end):
        strides = np.array([1, *np.cumprod(self.n_span[:-1])], dtype=np.int64)
        ranges = [np.arange(k) for k in self.n_span]
        ranges[direction] = np.array([0 if end == 0 else self.n_span[direction] - 1])
        mesh = np.meshgrid(*ranges, indexing="ij")
        return sum(m.ravel(order="F") * strides[d] for d, m in enumerate(mesh)).astype(np.int64)

    @cached_property
    def boundaries(self) -> dict:
        """label -> BoundarySet; unlabelled sides get ``patch0/<side>`` (function_space.py:490-535)."""
        labels = self.patch.label_map
        out = {}
        for d in range(self.dim):
            for end in (0, 1):
                side = f"{'uvw'[d]}{end}"
                label = labels.get(side, f"patch0/{side}")
                elems = self._side_elements(d, end)
                entry = out.setdefault(label, ([], [], []))
                entry[0].append(elems)
                entry[1].append(np.full(len(elems), 2 * d + end))
                entry[2].append(self.side_indices(side))
        return {k: BoundarySet(np.concatenate(v[0]), np.concatenate(v[1]), np.unique(np.concatenate(v[2])))
                for k, v in out.items()}

    def boundary(self, label: str) -> BoundarySet:
        if label not in self.boundaries:
            raise KeyError(f"unknown boundary label {label!r}; available: {sorted(self.boundaries)}")
        return self.boundaries[label]

    def sides_of_label(self, label: str):
        labels = self.patch.label_map
        return [f"{'uvw'[d]}{e}" for d in range(self.dim) for e in (0, 1)
                if labels.get(f"{'uvw'[d]}{e}", f"patch0/{'uvw'[d]}{e}") == label]

    def summary(self) -> str:
        return (f"FunctionSpace(dim={self.dim}, vec={self.vec}, degree={self.degree}, "
                f"n_elems={self.n_elems}, n_scalar_basis={self.n_scalar_basis}, "
                f"n_dofs={self.n_dofs}, boundaries={sorted(self.boundaries)})")
