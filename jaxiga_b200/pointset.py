"""Point sets: elements plus reference points in [-1, 1]^dim
(src/jaxiga/space/pointset.py:27-136).

A :class:`PointSet` names elements of a single-patch space (reference order,
first direction fastest) and, for each, points in the reference cube -- one
rule shared by every element (``ref`` of shape (n_q, dim)) or one per element
((n_e, n_q, dim)). ``weights`` are reference-cube quadrature weights without
the element Jacobian, which the evaluation applies. ``Solution.at``,
``Solution.grad``, ``errornorm``, ``norm`` and ``integrate`` take one; the
device evaluates the basis at its points (``jxb_eval_points``).
"""

from __future__ import annotations

import dataclasses

import numpy as np

from .space import gauss_1d


@dataclasses.dataclass(frozen=True)
class PointSet:
    """Evaluation points attached to elements of a function space. ``sides``
    (boundary sets only) holds each element's side code 2 * direction + end."""

    elems: np.ndarray
    ref: np.ndarray
    weights: np.ndarray | None = None
    sides: np.ndarray | None = None
    tag: str = "interior"

    def __post_init__(self):
        elems = np.asarray(self.elems, dtype=np.int64).reshape(-1)
        ref = np.asarray(self.ref, dtype=np.float64)
        if ref.ndim not in (2, 3) or (ref.ndim == 3 and ref.shape[0] != len(elems)):
            raise ValueError("ref must be (n_q, dim) or (n_elems, n_q, dim)")
        object.__setattr__(self, "elems", elems)
        object.__setattr__(self, "ref", ref)
        if self.weights is not None:
            object.__setattr__(self, "weights", np.asarray(self.weights, dtype=np.float64))

    @property
    def n_elems(self) -> int:
        return len(self.elems)

    @property
    def n_q(self) -> int:
        return self.ref.shape[-2]

    @property
    def dim(self) -> int:
        return self.ref.shape[-1]

    @property
    def shared_ref(self) -> bool:
        return self.ref.ndim == 2

    @property
    def n_pts(self) -> int:
        return self.n_elems * self.n_q

    def flat(self):
        """(elements, reference points) per point, (n_pts,) and (n_pts, dim)."""
        ref = np.broadcast_to(self.ref, (self.n_elems, self.n_q, self.dim)) if self.shared_ref else self.ref
        return np.repeat(self.elems, self.n_q), np.ascontiguousarray(ref.reshape(-1, self.dim))

    def flat_weights(self):
        """Reference weights per point, (n_pts,), or None."""
        if self.weights is None:
            return None
        w = np.broadcast_to(self.weights, (self.n_elems, self.n_q)) if self.weights.ndim == 1 else self.weights
        return np.ascontiguousarray(w.reshape(-1))


def tensor_rule(n_per_dir):
    """Tensor-product Gauss rule, first direction fastest (pointset.py:104-112)."""
    per_dir = [gauss_1d(n) for n in n_per_dir]
    grids = np.meshgrid(*[p[0] for p in per_dir], indexing="ij")
    wgrids = np.meshgrid(*[p[1] for p in per_dir], indexing="ij")
    pts = np.stack([g.ravel(order="F") for g in grids], axis=1)
    wts = np.prod([w.ravel(order="F") for w in wgrids], axis=0)
    return pts, wts


def gauss(space, n: int | None = None) -> PointSet:
    """Gauss quadrature on every element, ``n`` points per direction (default
    p + 1) (pointset.py:115-136)."""
    pts, wts = tensor_rule([(p + 1) if n is None else int(n) for p in space.degree])
    return PointSet(elems=np.arange(space.n_elems), ref=pts, weights=wts, tag="interior")


def boundary_gauss(space, bset, n: int | None = None, label: str = "set") -> PointSet:
    """Gauss rule of dimension dim - 1 on the sides of a boundary set, per
    element (pointset.py:148-200): the tangential directions carry ``n``
    (default p + 1) points, the pinned one sits at -1 or +1."""
    dim = space.dim
    n_per_dir = [(p + 1) if n is None else int(n) for p in space.degree]
    sides = np.asarray(bset.sides, dtype=np.int64)
    rules = {}
    for code in np.unique(sides):
        direction, end = divmod(int(code), 2)
        tangential = [d for d in range(dim) if d != direction]
        fp, fw = tensor_rule([n_per_dir[d] for d in tangential])
        pts = np.zeros((len(fp), dim))
        for k, d in enumerate(tangential):
            pts[:, d] = fp[:, k]
        pts[:, direction] = -1.0 if end == 0 else 1.0
        rules[int(code)] = (pts, fw)
    n_q = len(next(iter(rules.values()))[0]) if rules else 0
    ref = np.zeros((len(sides), n_q, dim))
    wts = np.zeros((len(sides), n_q))
    for i, code in enumerate(sides):
        ref[i], wts[i] = rules[int(code)]
    return PointSet(elems=np.asarray(bset.elems), ref=ref, weights=wts, sides=sides, tag=f"boundary:{label}")
