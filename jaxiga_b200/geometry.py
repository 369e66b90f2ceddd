"""NURBS patches and their refinement (host setup stage).

Mirrors the public surface of ``src/jaxiga/geometry/nurbs.py`` (``Patch``,
``create``, ``elevate``, ``insert_knots``, ``refine``) and the constructors of
``src/jaxiga/geometry/primitives.py`` that the solver workloads use.

Conventions follow the reference (nurbs.py:1-20): control points form a
tensor grid flattened with the first parametric direction fastest, are stored
unweighted with separate weights, knot vectors are normalised to [0, 1], and
sides are ``u0/u1/v0/v1/w0/w1``.

Refinement works on homogeneous coordinates along one direction at a time:

* knot insertion is Boehm's algorithm, one knot at a time;
* degree elevation goes through Bezier form: the extraction operators of the
  current knot vector give each span's Bezier control points, those are
  raised with the binomial degree-elevation formula, and the control points
  of the elevated spline (interior multiplicities raised by the same amount)
  are recovered span by span through the inverse transposed extraction
  operators of the new knot vector.
"""

from __future__ import annotations

import dataclasses
from math import comb

import numpy as np

from .space import bezier_extraction, element_spans

DIR_NAMES = ("u", "v", "w")
LEGACY_SIDES = {"left": "u0", "right": "u1", "down": "v0", "up": "v1"}
TOL = 1e-10


def side_name(direction: int, end: int) -> str:
    return f"{DIR_NAMES[direction]}{end}"


def canonical_side(name: str) -> str:
    return LEGACY_SIDES.get(name, name)


def _normalize_knots(kv) -> tuple:
    kv = np.asarray(kv, dtype=float)
    lo, hi = kv[0], kv[-1]
    if hi - lo <= 0:
        raise ValueError(f"degenerate knot vector with span [{lo}, {hi}]")
    return tuple(((kv - lo) / (hi - lo)).tolist())


def _labels_to_tuple(labels) -> tuple:
    if labels is None:
        return ()
    items = labels.items() if isinstance(labels, dict) else labels
    return tuple(sorted((canonical_side(k), v) for k, v in items))


# --------------------------------------------------------------------------
# univariate operators on (n_cp, ncomp) homogeneous coefficients
# --------------------------------------------------------------------------


def _insert_one(deg, knots, coefs, u):
    """Boehm insertion of a single knot ``u`` into a degree-``deg`` curve."""
    knots = np.asarray(knots, dtype=float)
    n = coefs.shape[0]
    k = int(np.searchsorted(knots, u, side="right") - 1)
    k = min(k, n - 1)
    out = np.empty((n + 1, coefs.shape[1]))
    out[: k - deg + 1] = coefs[: k - deg + 1]
    for i in range(k - deg + 1, k + 1):
        alpha = (u - knots[i]) / (knots[i + deg] - knots[i])
        out[i] = alpha * coefs[i] + (1.0 - alpha) * coefs[i - 1]
    out[k + 1:] = coefs[k:]
    return np.insert(knots, k + 1, u), out


def insert_knots_1d(deg, knots, coefs, new):
    knots = np.asarray(knots, dtype=float)
    for u in np.sort(np.asarray(new, dtype=float)):
        knots, coefs = _insert_one(deg, knots, coefs, float(u))
    return knots, coefs


def _bezier_elevation_matrix(p, t):
    """(p+t+1, p+1) map from degree-p to degree-(p+t) Bezier control points."""
    q = p + t
    E = np.zeros((q + 1, p + 1))
    for i in range(q + 1):
        for j in range(max(0, i - t), min(p, i) + 1):
            E[i, j] = comb(p, j) * comb(t, i - j) / comb(q, i)
    return E


def elevate_1d(deg, knots, coefs, t):
    """Raise the degree of a curve by ``t`` through its Bezier segments."""
    knots = np.asarray(knots, dtype=float)
    if t == 0:
        return knots, coefs
    C_old = bezier_extraction(knots, deg)
    _, _, first = element_spans(knots, deg)
    E = _bezier_elevation_matrix(deg, t)
    # Bezier control points of every span, elevated: N = C B  =>  bezier = C^T c
    bez = [E @ (C_old[e].T @ coefs[first[e]: first[e] + deg + 1]) for e in range(len(C_old))]
    # new knot vector: every distinct knot gains t in multiplicity
    uniq, mult = np.unique(knots, return_counts=True)
    new_knots = np.repeat(uniq, mult + t)
    q = deg + t
    C_new = bezier_extraction(new_knots, q)
    _, _, first_new = element_spans(new_knots, q)
    n_new = len(new_knots) - q - 1
    out = np.full((n_new, coefs.shape[1]), np.nan)
    for e in range(len(C_new)):
        local = np.linalg.solve(C_new[e].T, bez[e])
        sl = slice(first_new[e], first_new[e] + q + 1)
        todo = np.isnan(out[sl, 0])
        out[sl][todo] = local[todo]
    return new_knots, out


def _apply_along_dir(coefs, n_per_dir, d, fn):
    """Apply a univariate operator along direction ``d`` of a tensor grid."""
    dim = len(n_per_dir)
    ncomp = coefs.shape[1]
    grid = np.asarray(coefs, dtype=float).reshape(*reversed(n_per_dir), ncomp)
    grid = np.moveaxis(grid, dim - 1 - d, 0)  # (n_d, ..., comp)
    rest = grid.shape[1:]
    # every curve along direction d at once: columns of an (n_d, n_curves * comp) matrix
    kv, out = fn(grid.reshape(grid.shape[0], -1))
    out = np.moveaxis(out.reshape(out.shape[0], *rest), 0, dim - 1 - d)
    return out.reshape(-1, ncomp), kv


# --------------------------------------------------------------------------
# Patch
# --------------------------------------------------------------------------


@dataclasses.dataclass(frozen=True)
class Patch:
    """A single NURBS patch (src/jaxiga/geometry/nurbs.py:279-496)."""

    ctrl_pts: np.ndarray
    weights: np.ndarray
    knots: tuple
    degree: tuple
    labels: tuple = ()

    @classmethod
    def create(cls, knots, degree, ctrl_pts, weights=None, labels=None) -> "Patch":
        degree = tuple(int(p) for p in degree)
        knots = tuple(_normalize_knots(kv) for kv in knots)
        if len(knots) != len(degree):
            raise ValueError(f"{len(knots)} knot vectors but {len(degree)} degrees")
        ctrl_pts = np.asarray(ctrl_pts, dtype=float)
        if ctrl_pts.ndim != 2:
            raise ValueError(f"ctrl_pts must be (n_cp, dim_phys), got shape {ctrl_pts.shape}")
        expected = [len(kv) - p - 1 for kv, p in zip(knots, degree)]
        if int(np.prod(expected)) != ctrl_pts.shape[0]:
            raise ValueError(f"knots/degree imply {expected} control points but {ctrl_pts.shape[0]} were given")
        weights = np.ones(ctrl_pts.shape[0]) if weights is None else np.asarray(weights, dtype=float)
        if weights.shape != (ctrl_pts.shape[0],):
            raise ValueError(f"weights must be ({ctrl_pts.shape[0]},), got {weights.shape}")
        return cls(ctrl_pts, weights, knots, degree, _labels_to_tuple(labels))

    @property
    def dim(self) -> int:
        return len(self.degree)

    @property
    def dim_phys(self) -> int:
        return self.ctrl_pts.shape[1]

    @property
    def n_cp_per_dir(self) -> tuple:
        return tuple(len(kv) - p - 1 for kv, p in zip(self.knots, self.degree))

    @property
    def n_cp(self) -> int:
        return int(np.prod(self.n_cp_per_dir))

    @property
    def label_map(self) -> dict:
        return dict(self.labels)

    def knot_arrays(self) -> list:
        return [np.asarray(kv, dtype=float) for kv in self.knots]

    def homogeneous(self) -> np.ndarray:
        return np.concatenate([self.ctrl_pts * self.weights[:, None], self.weights[:, None]], 1)

    def side_names(self) -> tuple:
        return tuple(side_name(d, e) for d in range(self.dim) for e in (0, 1))

    def with_labels(self, **side_labels) -> "Patch":
        merged = self.label_map
        for side, label in side_labels.items():
            side = canonical_side(side)
            if side not in self.side_names():
                raise ValueError(f"unknown side {side!r}; expected one of {self.side_names()}")
            merged[side] = label
        return dataclasses.replace(self, labels=_labels_to_tuple(merged))

    def _rebuild(self, coefs, knots, degree) -> "Patch":
        w = coefs[:, -1]
        return Patch.create(knots, degree, coefs[:, :-1] / w[:, None], w, self.labels)

    def elevate(self, target_degree) -> "Patch":
        """Raise the degree *to* ``target_degree`` (a scalar applies to every direction)."""
        target = (int(target_degree),) * self.dim if np.isscalar(target_degree) else tuple(int(p) for p in target_degree)
        if len(target) != self.dim:
            raise ValueError(f"expected {self.dim} target degrees, got {len(target)}")
        times = [t - p for t, p in zip(target, self.degree)]
        if any(t < 0 for t in times):
            raise ValueError(f"cannot lower degree: patch has degree {self.degree}, target {target}")
        if all(t == 0 for t in times):
            return self
        coefs = self.homogeneous()
        knots = self.knot_arrays()
        n = list(self.n_cp_per_dir)
        degree = list(self.degree)
        for d in range(self.dim):
            if times[d] == 0:
                continue
            coefs, kv = _apply_along_dir(coefs, n, d, lambda c: elevate_1d(degree[d], knots[d], c, times[d]))
            knots[d] = kv
            degree[d] = target[d]
            n[d] = len(kv) - degree[d] - 1
        return self._rebuild(coefs, knots, degree)

    def insert_knots(self, *knots_per_dir) -> "Patch":
        if len(knots_per_dir) != self.dim:
            raise ValueError(f"expected {self.dim} knot sequences, got {len(knots_per_dir)}")
        coefs = self.homogeneous()
        knots = self.knot_arrays()
        n = list(self.n_cp_per_dir)
        for d in range(self.dim):
            new = np.asarray(knots_per_dir[d], dtype=float)
            if new.size == 0:
                continue
            if new.min() <= 0.0 or new.max() >= 1.0:
                raise ValueError(f"interior knots must lie in (0, 1); got {new}")
            coefs, kv = _apply_along_dir(coefs, n, d, lambda c: insert_knots_1d(self.degree[d], knots[d], c, new))
            knots[d] = kv
            n[d] = len(kv) - self.degree[d] - 1
        return self._rebuild(coefs, knots, self.degree)

    def refine(self, n: int = 1) -> "Patch":
        """``n`` rounds of uniform bisection of every non-empty span."""
        patch = self
        for _ in range(int(n)):
            new = []
            for kv in patch.knot_arrays():
                uniq = np.unique(kv)
                new.append((uniq[:-1] + uniq[1:]) / 2)
            patch = patch.insert_knots(*new)
        return patch

    def summary(self) -> str:
        return f"Patch(dim={self.dim}, degree={self.degree}, n_cp={self.n_cp} {self.n_cp_per_dir}, labels={self.label_map})"


# --------------------------------------------------------------------------
# primitives (src/jaxiga/geometry/primitives.py)
# --------------------------------------------------------------------------


class primitives:  # noqa: N801 -- namespace mirroring ``jaxiga.primitives``
    @staticmethod
    def quadrilateral(corners) -> Patch:
        """Bilinear quadrilateral through four counter-clockwise corners (primitives.py:41-69)."""
        corners = np.asarray(corners, dtype=float)
        if corners.shape != (4, 2):
            raise ValueError(f"expected 4 corners of dimension 2, got shape {corners.shape}")
        a, b, c, d = corners
        return Patch.create([[0, 0, 1, 1], [0, 0, 1, 1]], (1, 1), np.array([a, b, d, c]), np.ones(4),
                            {"u0": "left", "u1": "right", "v0": "bottom", "v1": "top"})

    @staticmethod
    def rectangle(x0, y0, x1, y1) -> Patch:
        return primitives.quadrilateral([[x0, y0], [x1, y0], [x1, y1], [x0, y1]])

    @staticmethod
    def quarter_annulus(radius_int, radius_ext) -> Patch:
        """Quarter annulus in the first quadrant (primitives.py:107-133).

        u runs radially (u0 inner, u1 outer), v circumferentially from the x
        axis (v0) to the y axis (v1); the middle circumferential row carries
        weight sqrt(2)/2.
        """
        ri, re = float(radius_int), float(radius_ext)
        s = 1.0 / np.sqrt(2.0)
        cpts = np.array([[ri, 0.0], [re, 0.0], [ri, ri], [re, re], [0.0, ri], [0.0, re]])
        w = np.array([1.0, 1.0, s, s, 1.0, 1.0])
        return Patch.create([[0, 0, 1, 1], [0, 0, 0, 1, 1, 1]], (1, 2), cpts, w,
                            {"u0": "inner", "u1": "outer", "v0": "sym_y", "v1": "sym_x"})

    @staticmethod
    def cuboid(lower, upper) -> Patch:
        """Trilinear axis-aligned box (primitives.py:285-309)."""
        lo = np.asarray(lower, dtype=float)
        hi = np.asarray(upper, dtype=float)
        if lo.shape != (3,) or hi.shape != (3,):
            raise ValueError("lower and upper must each have 3 components")
        corners = np.array([[lo[0] if i == 0 else hi[0], lo[1] if j == 0 else hi[1], lo[2] if k == 0 else hi[2]]
                            for k in (0, 1) for j in (0, 1) for i in (0, 1)])
        return Patch.create([[0, 0, 1, 1]] * 3, (1, 1, 1), corners, np.ones(8),
                            {"u0": "left", "u1": "right", "v0": "bottom", "v1": "top", "w0": "back", "w1": "front"})
