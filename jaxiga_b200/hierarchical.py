"""Truncated hierarchical B-spline (THB) spaces on one patch.

The reference builds adaptive spaces in src/jaxiga/space/hierarchical.py: the
level-0 patch's knot vectors are bisected once per level, a ``Hierarchy``
records which elements of each level were replaced by their 2^dim children,
and the basis is the set of "active" B-splines of every level, truncated
against the finer active functions. Elements then carry different numbers of
basis functions, so connectivity and extraction are padded to the largest
count (the padded-element contract, src/jaxiga/space/function_space.py:23-38):
padding DOFs use the index ``n_scalar_basis`` and their extraction rows are
zero.

This module restates that construction for a single patch:

* levels (``_Levels``): bisected knot vectors, spans and Bezier extraction per
  level (hierarchical.py:225-288);
* the refinement state and its closure (``_State``, ``_close``): domains and
  leaves per level, marking with ancestors, and the class-2 admissibility of
  Buffa and Giannelli through level-(l-1) support extensions
  (hierarchical.py:301-585);
* relevant and active functions, the restricted two-scale operators from
  per-direction Oslo rows (Lyche and Morken, knot insertion), and the
  truncated coefficient matrices (hierarchical.py:588-708);
* per leaf element the supported hierarchical functions and the extraction
  operator V^T C_bez that maps its Bernstein polynomials to them, the control
  net pushed through the two-scale operators (so the geometry is the level-0
  patch's), and the boundary sets (hierarchical.py:746-1040);
* ``refine_elements`` and ``dorfler_mark`` (hierarchical.py:1042-1156).

Multipatch hierarchies (interface mirroring and gluing) are not restated.
The device operator on these spaces is ``ThbOperator`` (thb.py).
"""

from __future__ import annotations

import dataclasses

import numpy as np
import scipy.sparse as sp

from .space import BoundarySet, bezier_extraction, element_spans, expand_dofs

COEFF_TOL = 1e-13        # two-scale and truncated coefficients below this are dropped
MAX_LOCAL_GROWTH = 3.0   # functions per element at most this times a tensor element's


class HierarchyError(Exception):
    """A hierarchy that cannot be represented (bad marking, too many local functions)."""


@dataclasses.dataclass(frozen=True)
class Hierarchy:
    """Refined elements per level: ``refined[l]`` is the sorted tuple of level-l
    element indices (first direction fastest) replaced by their children."""

    refined: tuple = ()
    truncate: bool = True
    admissible: bool = True

    @property
    def n_levels(self) -> int:
        return 1 + len(self.refined)


def _ravel(idx, dims):
    return np.ravel_multi_index(tuple(np.asarray(i, dtype=np.int64) for i in idx), tuple(dims), order="F")


def _unravel(flat, dims):
    return np.unravel_index(np.asarray(flat, dtype=np.int64), tuple(dims), order="F")


def _tensor(ranges, dims):
    """Flat indices of the tensor product of per-direction ranges, first direction fastest."""
    strides = np.concatenate([[1], np.cumprod(np.asarray(dims[:-1], dtype=np.int64))])
    flat = np.asarray(ranges[0], dtype=np.int64) * strides[0]
    for d in range(1, len(ranges)):
        flat = (flat[:, None] + np.asarray(ranges[d], dtype=np.int64)[None, :] * strides[d]).ravel(order="F")
    return flat


def _bisect(kv):
    """Every non-empty span of a knot vector cut in half."""
    u = np.unique(kv)
    return np.sort(np.concatenate([kv, 0.5 * (u[:-1] + u[1:])]))


def oslo_row(tau, deg, t, i):
    """Row i of the two-scale operator from knots ``tau`` to the finer ``t``:
    (offset, w) with fine coefficient d_i = w . c[offset : offset + deg + 1].

    The discrete B-splines of Lyche and Morken: for tau_mu <= t_i < tau_mu+1,
    the row is R_1(t_{i+1}) R_2(t_{i+2}) ... R_deg(t_{i+deg}), R_k(x) the k x
    (k+1) matrix with the entries (tau_{j+k} - x, x - tau_j) / (tau_{j+k} -
    tau_j) for j = mu-k+1 .. mu, taken here left to right (a row vector times
    each R_k in turn). A zero denominator (repeated knots) passes the entry on.
    """
    mu = int(np.searchsorted(tau, t[i], side="right") - 1)
    mu = min(max(mu, deg), len(tau) - deg - 2)
    row = np.ones(1)
    for k in range(1, deg + 1):
        x = t[i + k]
        new = np.zeros(k + 1)
        for r in range(k):
            hi, lo = tau[mu + 1 + r], tau[mu + 1 + r - k]
            den = hi - lo
            if den <= 0.0:
                new[r + 1] += row[r]
            else:
                new[r] += row[r] * (hi - x) / den
                new[r + 1] += row[r] * (x - lo) / den
        row = new
    return mu - deg, row


class _Levels:
    """Per-direction data of every level of the patch (never a tensor array)."""

    def __init__(self, patch, n_levels):
        self.patch = patch
        self.dim = patch.dim
        self.degree = tuple(patch.degree)
        self.knots = [patch.knot_arrays()]
        self.spans, self.ext, self.n_elem, self.n_func = [], [], [], []
        self.extend(n_levels)

    def extend(self, n):
        while len(self.knots) < n:
            self.knots.append([_bisect(kv) for kv in self.knots[-1]])
        while len(self.n_elem) < n:
            kv = self.knots[len(self.n_elem)]
            spans = [element_spans(kv[d], self.degree[d]) for d in range(self.dim)]
            self.spans.append(spans)
            self.ext.append([bezier_extraction(kv[d], self.degree[d]) for d in range(self.dim)])
            self.n_elem.append(tuple(len(s[0]) for s in spans))
            self.n_func.append(tuple(len(kv[d]) - self.degree[d] - 1 for d in range(self.dim)))

    def funcs_of_elem(self, l, d, e):
        f = self.spans[l][d][2][e]
        return np.arange(f, f + self.degree[d] + 1)

    def elems_of_func(self, l, d, j):
        first = self.spans[l][d][2]
        return np.arange(np.searchsorted(first, j - self.degree[d], side="left"),
                         np.searchsorted(first, j, side="right"))

    def parent(self, l, e):
        """Level-(l-1) element containing level-l element e."""
        idx = np.array(_unravel([e], self.n_elem[l]))[:, 0]
        return int(_ravel(idx // 2, self.n_elem[l - 1]))

    def children(self, l, elems):
        """The 2^dim level-(l+1) elements of each level-l element."""
        elems = np.asarray(sorted(elems), dtype=np.int64)
        if elems.size == 0:
            return np.zeros(0, dtype=np.int64)
        idx = np.array(_unravel(elems, self.n_elem[l]))
        out = [_ravel(2 * idx + np.array([(c >> d) & 1 for d in range(self.dim)])[:, None], self.n_elem[l + 1])
               for c in range(2 ** self.dim)]
        return np.concatenate(out)


class _State:
    """Refinement state: ``refined[l]`` sets, with domains and leaves derived."""

    def __init__(self, patch, refined):
        self.refined = [set(int(e) for e in lv) for lv in refined]
        self.levels = _Levels(patch, self.n_levels)
        self._dom = None

    @property
    def n_levels(self):
        deepest = max((l for l, s in enumerate(self.refined) if s), default=-1)
        return deepest + 2

    def _sync(self):
        self.levels.extend(self.n_levels)
        while len(self.refined) < self.n_levels:
            self.refined.append(set())
        self._dom = None

    def domains(self):
        """(dom, leaf): per level, the live elements and those not refined further."""
        if self._dom is None:
            self._sync()
            L = self.levels
            dom = [set(range(int(np.prod(L.n_elem[0]))))]
            for l in range(self.n_levels - 1):
                bad = self.refined[l] - dom[l]
                if bad:
                    raise HierarchyError(f"{len(bad)} elements marked at level {l} lie outside the level-{l} domain")
                dom.append(set(int(k) for k in L.children(l, self.refined[l])))
            leaf = [dom[l] - (self.refined[l] if l < len(self.refined) else set()) for l in range(self.n_levels)]
            self._dom = (dom, leaf)
        return self._dom

    def mark(self, l, e):
        """Refine level-l element e (its ancestors first); True when that changed anything."""
        self._sync()
        if l >= self.n_levels:
            raise HierarchyError(f"level {l} does not exist yet")
        e = int(e)
        if l > 0:
            p = self.levels.parent(l, e)
            if p not in self.refined[l - 1]:
                self.mark(l - 1, p)
        while len(self.refined) <= l:
            self.refined.append(set())
        if e in self.refined[l]:
            return False
        self.refined[l].add(e)
        self._sync()
        return True

    def ensure_live(self, l, e):
        """Make level-l element e part of the level-l domain (refining its parent)."""
        dom, _ = self.domains()
        if l == 0 or int(e) in dom[l]:
            return False
        return self.mark(l - 1, self.levels.parent(l, int(e)))

    def support_extension(self, l, elems):
        """Level-(l-1) elements met by a level-(l-1) function whose support
        meets the parent of any of ``elems`` (level-l elements): per direction
        the elements whose first function lies within deg of the parent's."""
        L = self.levels
        elems = np.asarray(elems, dtype=np.int64)
        if elems.size == 0:
            return np.zeros(0, dtype=np.int64)
        par = np.array(_unravel(elems, L.n_elem[l])) // 2
        lo, wd = [], []
        for d in range(L.dim):
            first = L.spans[l - 1][d][2]
            anchor = first[par[d]]
            a = np.searchsorted(first, anchor - L.degree[d], side="left")
            b = np.searchsorted(first, anchor + L.degree[d], side="right")
            lo.append(a)
            wd.append(b - a)
        dims = L.n_elem[l - 1]
        strides = np.concatenate([[1], np.cumprod(np.asarray(dims[:-1], dtype=np.int64))])
        out = []
        for off in np.ndindex(*[int(w.max()) for w in wd]):
            ok = np.ones(len(elems), bool)
            flat = np.zeros(len(elems), dtype=np.int64)
            for d in range(L.dim):
                ok &= off[d] < wd[d]
                flat += (lo[d] + off[d]) * strides[d]
            out.append(flat[ok])
        return np.unique(np.concatenate(out))

    def close(self, admissible):
        """Class-2 admissibility: every level-l element's level-(l-1) support
        extension lies in the level-(l-1) domain; swept to a fixpoint."""
        if not admissible:
            return
        for _ in range(256):
            changed = False
            for l in range(self.n_levels - 1, 0, -1):
                dom, _ = self.domains()
                if l >= len(dom):
                    continue
                req = self.support_extension(l, np.fromiter(dom[l], dtype=np.int64, count=len(dom[l])))
                coarse = dom[l - 1]
                for c in req:
                    if int(c) not in coarse:
                        changed |= self.ensure_live(l - 1, int(c))
            if not changed:
                return
        raise HierarchyError("refinement closure did not converge in 256 sweeps")

    def hierarchy(self, truncate, admissible):
        lv = [tuple(sorted(s)) for s in self.refined]
        while lv and not lv[-1]:
            lv.pop()
        return Hierarchy(refined=tuple(lv), truncate=truncate, admissible=admissible)


# --------------------------------------------------------------------------
# the basis: relevant and active functions, two-scale and truncation
# --------------------------------------------------------------------------
def _relevant(L, l, elems):
    """Level-l functions supported on at least one of ``elems`` (sorted)."""
    if not elems:
        return np.zeros(0, dtype=np.int64)
    return np.unique(_elem_funcs(L, l, np.fromiter(elems, dtype=np.int64, count=len(elems))))


def _elem_funcs(L, l, elems):
    """(n, (p+1)^dim) level-l tensor functions of each element, first direction fastest."""
    dim, n1 = L.dim, L.degree[0] + 1
    idx = np.array(_unravel(elems, L.n_elem[l]))
    strides = np.concatenate([[1], np.cumprod(np.asarray(L.n_func[l][:-1], dtype=np.int64))])
    t = np.arange(n1 ** dim)
    out = np.zeros((len(elems), n1 ** dim), dtype=np.int64)
    for d in range(dim):
        out += (L.spans[l][d][2][idx[d]][:, None] + (t // n1 ** d) % n1) * strides[d]
    return out


def _box_counts(L, l, marked, lo, hi):
    """Per box [lo, hi) of level-l element indices (dim, n), how many of its
    elements are in ``marked`` (a set of flat indices): summed-area table."""
    shape = tuple(L.n_elem[l])
    flag = np.zeros(int(np.prod(shape)), dtype=np.int64)
    if marked:
        flag[np.fromiter(marked, dtype=np.int64, count=len(marked))] = 1
    P = np.zeros(tuple(s + 1 for s in shape), dtype=np.int64)
    A = flag.reshape(shape, order="F")
    for d in range(len(shape)):
        A = np.cumsum(A, axis=d)
    P[tuple(slice(1, None) for _ in shape)] = A
    total = np.zeros(lo.shape[1], dtype=np.int64)
    for corner in np.ndindex(*([2] * len(shape))):
        sign = (-1) ** (len(shape) - sum(corner))
        total += sign * P[tuple(hi[d] if c else lo[d] for d, c in enumerate(corner))]
    return total


def _active(L, l, cand, dom, leaf):
    """Candidates whose support lies in the level-l domain and meets a leaf."""
    cand = np.asarray(cand, dtype=np.int64)
    if not len(cand):
        return cand
    jd = np.array(_unravel(cand, L.n_func[l]))
    lo = np.stack([np.searchsorted(L.spans[l][d][2], jd[d] - L.degree[d], side="left") for d in range(L.dim)])
    hi = np.stack([np.searchsorted(L.spans[l][d][2], jd[d], side="right") for d in range(L.dim)])
    size = np.prod(hi - lo, axis=0)
    keep = (_box_counts(L, l, dom, lo, hi) == size) & (_box_counts(L, l, leaf, lo, hi) > 0)
    return cand[keep]


def _two_scale(L, l, coarse, fine):
    """Two-scale operator restricted to level-(l+1) rows ``fine`` and level-l
    columns ``coarse``: the tensor product of per-direction Oslo rows."""
    dim = L.dim
    fidx = np.array(_unravel(fine, L.n_func[l + 1]))
    shapes = [L.degree[d] + 1 for d in range(dim)]
    local = np.array(_unravel(np.arange(int(np.prod(shapes))), shapes))  # (dim, n_loc), first direction fastest
    strides = np.concatenate([[1], np.cumprod(np.asarray(L.n_func[l][:-1], dtype=np.int64))])
    flat = np.zeros((len(fine), local.shape[1]), dtype=np.int64)
    coef = np.ones((len(fine), local.shape[1]))
    for d in range(dim):
        uniq, inv = np.unique(fidx[d], return_inverse=True)
        rows = [oslo_row(L.knots[l][d], L.degree[d], L.knots[l + 1][d], int(i)) for i in uniq]
        off = np.array([r[0] for r in rows], dtype=np.int64)[inv]
        w = np.array([r[1] for r in rows])[inv]
        flat += (off[:, None] + local[d][None, :]) * strides[d]
        coef *= w[:, local[d]]
    order = np.argsort(coarse)
    sc = np.asarray(coarse)[order]
    pos = np.searchsorted(sc, flat).clip(0, max(len(sc) - 1, 0))
    live = (len(sc) > 0) & (sc[pos] == flat) & (np.abs(coef) > COEFF_TOL)
    rows = np.repeat(np.arange(len(fine)), local.shape[1]).reshape(flat.shape)[live]
    return sp.csr_matrix((coef[live], (rows, order[pos][live])), shape=(len(fine), len(coarse)))


def _thb_coefficients(relevant, active, S, truncate):
    """Per level l the (relevant[l] x n_basis) matrix of the hierarchical
    functions' coefficients in the level-l B-splines; the columns are the
    active functions, level by level, ascending within a level."""
    columns = [(l, int(j)) for l, a in enumerate(active) for j in a]
    col = {c: k for k, c in enumerate(columns)}
    Q = []
    cur = sp.csr_matrix((len(relevant[0]), len(columns)))
    for l in range(len(relevant)):
        row = {int(j): r for r, j in enumerate(relevant[l])}
        if l > 0:
            cur = (S[l - 1] @ cur).tocsr()
            if truncate and len(active[l]):
                keep = np.ones(len(relevant[l]))
                keep[[row[int(j)] for j in active[l]]] = 0.0
                cur = (sp.diags(keep) @ cur).tocsr()
            cur.data[np.abs(cur.data) < COEFF_TOL] = 0.0
            cur.eliminate_zeros()
        if len(active[l]):
            r = [row[int(j)] for j in active[l]]
            c = [col[(l, int(j))] for j in active[l]]
            cur = (cur + sp.csr_matrix((np.ones(len(r)), (r, c)), shape=cur.shape)).tocsr()
        blk = cur.tocsr()
        blk.sum_duplicates()
        Q.append(blk)
    return Q, columns


def _level_elements(L, l, elems, Q, relevant):
    """Connectivity and extraction of the leaf elements ``elems`` (sorted) of
    level l, all at once: per element the active functions that its level-l
    tensor functions touch through the THB rows Q (ascending), the values V of
    those rows, and the extraction V^T kron(C_{dim-1}, ..., C_0) from the
    element's Bernstein polynomials to them (function_space.py:315-323).
    Returns (columns per element as a padded (n, m) array with counts, the
    extraction (n, m, nb), the parametric boxes (n, 2 dim))."""
    dim, p = L.dim, L.degree[0]
    n1 = p + 1
    nb = n1 ** dim
    E = np.asarray(elems, dtype=np.int64)
    n = len(E)
    idx = np.array(_unravel(E, L.n_elem[l]))                      # (dim, n)
    loc = _elem_funcs(L, l, E)                                     # level-l tensor functions
    rows = np.searchsorted(relevant, loc)                          # rows of Q (relevant is sorted)
    ip, ind, dat = Q.indptr, Q.indices, Q.data
    r = rows.ravel()
    cnt = ip[r + 1] - ip[r]
    src = np.repeat(ip[r], cnt) + (np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt))
    ent = np.repeat(np.arange(n * nb), cnt)
    col, val = ind[src].astype(np.int64), dat[src]
    nz = val != 0.0
    ent, col, val = ent[nz], col[nz], val[nz]
    el, lrow = ent // nb, ent % nb
    key = el * Q.shape[1] + col
    uk, inv = np.unique(key, return_inverse=True)                  # per element, its columns ascending
    ue, uc = uk // Q.shape[1], uk % Q.shape[1]
    count = np.bincount(ue, minlength=n)
    lcol = np.arange(len(uk)) - (np.cumsum(count) - count)[ue]
    m = int(count.max()) if n else 0
    cols = np.zeros((n, m), dtype=np.int64)
    cols[ue, lcol] = uc
    V = np.zeros((n, nb, m))
    V[el, lrow, lcol[inv]] = val
    C = np.asarray(L.ext[l][dim - 1])[idx[dim - 1]]
    for d in range(dim - 2, -1, -1):                               # kron, the last direction outermost
        Ed = np.asarray(L.ext[l][d])[idx[d]]
        C = np.einsum("eij,ekl->eikjl", C, Ed).reshape(n, C.shape[1] * Ed.shape[1], C.shape[2] * Ed.shape[2])
    ops = np.matmul(V.transpose(0, 2, 1), C)
    boxes = np.concatenate([np.stack([L.spans[l][d][0][idx[d]] for d in range(dim)], 1),
                            np.stack([L.spans[l][d][1][idx[d]] for d in range(dim)], 1)], 1)
    return cols, count, ops, boxes


# --------------------------------------------------------------------------
# the space
# --------------------------------------------------------------------------
class HierarchicalSpace:
    """A THB space on one patch, in the padded-element form of the reference
    (build_hierarchical_space, hierarchical.py:891-980).

    elem_dofs (n_elems, n_local_max): scalar DOFs per leaf element, padding =
    n_scalar_basis; extraction (n_elems, n_local_max, (p+1)^dim): maps the
    element's Bernstein polynomials on [-1, 1]^dim to its functions, zero rows
    for the padding; elem_vertex (n_elems, 2 dim): parametric box (minima,
    maxima); elem_key (n_elems, 3): (patch, level, element of that level);
    cpts / wgts: the hierarchical control net (it reproduces the level-0
    geometry). Leaf elements come level by level, ascending within a level.
    """

    cell_type = "thb"

    def __init__(self, patch, hierarchy: Hierarchy, vec: int = 1):
        degs = set(patch.degree)
        if len(degs) != 1:
            raise NotImplementedError(f"equal degrees in every direction are needed, got {patch.degree}")
        self.patch, self.hierarchy, self.vec = patch, hierarchy, int(vec)
        self.dim, self.degree = patch.dim, tuple(patch.degree)
        state = _State(patch, hierarchy.refined)
        dom, leaf = state.domains()
        L = state.levels
        self._levels = L
        nl = len(dom)
        relevant = [_relevant(L, l, dom[l]) for l in range(nl)]
        active = [_active(L, l, relevant[l], dom[l], leaf[l]) for l in range(nl)]
        S = [_two_scale(L, l, relevant[l], relevant[l + 1]) for l in range(nl - 1)]
        Q, columns = _thb_coefficients(relevant, active, S, hierarchy.truncate)
        # control net: the level-0 homogeneous net pushed through the two-scale operators
        hom = [np.asarray(patch.homogeneous())[relevant[0]]]
        for l in range(nl - 1):
            hom.append(np.asarray(S[l] @ hom[l]))
        rowof = [{int(j): r for r, j in enumerate(relevant[l])} for l in range(nl)]
        control = np.array([hom[l][rowof[l][j]] for l, j in columns]).reshape(len(columns), -1)
        self.columns = columns
        self.n_scalar_basis = len(columns)
        self.wgts = control[:, -1].copy()
        self.cpts = control[:, :-1] / control[:, -1:]
        nb = int(np.prod([p + 1 for p in self.degree]))
        parts = []  # per level with leaves: (level, elements, columns, counts, extraction, boxes)
        for l in range(nl):
            if leaf[l]:
                E = np.array(sorted(leaf[l]), dtype=np.int64)
                parts.append((l, E) + _level_elements(L, l, E, Q[l], relevant[l]))
        n_loc = max([nb] + [int(c.max()) for *_, c, _, _ in parts if len(c)])
        if n_loc > MAX_LOCAL_GROWTH * nb:
            raise HierarchyError(f"an element gathers {n_loc} functions where a tensor-product element of this "
                                 f"degree gathers {nb}; refine with admissible=True, or mark fewer elements")
        self.n_elems = sum(len(E) for _, E, *_ in parts)
        self.n_local_max = n_loc
        self.n_local = nb
        self.elem_dofs = np.full((self.n_elems, n_loc), self.n_scalar_basis, dtype=np.int64)
        self.extraction = np.zeros((self.n_elems, n_loc, nb))
        self.elem_vertex = np.zeros((self.n_elems, 2 * self.dim))
        self.elem_key = np.zeros((self.n_elems, 3), dtype=np.int64)
        k = 0
        for l, E, cols, count, ops, boxes in parts:
            sl = slice(k, k + len(E))
            m = cols.shape[1]
            pad = np.arange(m)[None, :] >= count[:, None]
            self.elem_dofs[sl, :m] = np.where(pad, self.n_scalar_basis, cols)
            self.extraction[sl, :m] = np.where(pad[..., None], 0.0, ops)
            self.elem_vertex[sl] = boxes
            self.elem_key[sl, 1], self.elem_key[sl, 2] = l, E
            k += len(E)
        self._boundaries = self._classify()
        self._plans = {}  # device operators and evaluation data cached by solve()

    # -- sizes -------------------------------------------------------------
    @property
    def n_dofs(self) -> int:
        return self.n_scalar_basis * self.vec

    @property
    def dim_phys(self) -> int:
        return self.cpts.shape[1]

    def elem_dofs_vec(self):
        return expand_dofs(self.elem_dofs, self.vec)

    # -- boundaries --------------------------------------------------------
    def _classify(self):
        """label -> BoundarySet: the leaf elements on a patch side and the
        active functions whose tensor index sits on it (hierarchical.py:982-1039)."""
        L, labels = self._levels, self.patch.label_map
        nd = self.dim
        lev = np.array([l for l, _ in self.columns], dtype=np.int64)
        fnum = np.array([j for _, j in self.columns], dtype=np.int64)
        # per function and per element: its tensor index at its level and that level's extent
        fidx, fext = np.zeros((nd, len(fnum)), dtype=np.int64), np.zeros((nd, len(fnum)), dtype=np.int64)
        eidx, eext = np.zeros((nd, self.n_elems), dtype=np.int64), np.zeros((nd, self.n_elems), dtype=np.int64)
        for l in np.unique(np.concatenate([lev, self.elem_key[:, 1]])):
            f, e = lev == l, self.elem_key[:, 1] == l
            fidx[:, f] = np.array(_unravel(fnum[f], L.n_func[l])).reshape(nd, -1)
            fext[:, f] = np.asarray(L.n_func[l])[:, None]
            eidx[:, e] = np.array(_unravel(self.elem_key[e, 2], L.n_elem[l])).reshape(nd, -1)
            eext[:, e] = np.asarray(L.n_elem[l])[:, None]
        out = {}
        for d in range(self.dim):
            for end in (0, 1):
                side = f"{'uvw'[d]}{end}"
                label = labels.get(side, f"patch0/{side}")
                elems = np.flatnonzero(eidx[d] == (0 if end == 0 else eext[d] - 1))
                dofs = np.flatnonzero(fidx[d] == (0 if end == 0 else fext[d] - 1))
                entry = out.setdefault(label, ([], [], []))
                entry[0].append(np.asarray(elems, dtype=np.int64))
                entry[1].append(np.full(len(elems), 2 * d + end, dtype=np.int64))
                entry[2].append(np.asarray(dofs, dtype=np.int64))
        return {k: BoundarySet(np.concatenate(v[0]), np.concatenate(v[1]), np.unique(np.concatenate(v[2])))
                for k, v in out.items()}

    @property
    def boundaries(self) -> dict:
        return self._boundaries

    def boundary(self, label: str) -> BoundarySet:
        if label not in self._boundaries:
            raise KeyError(f"unknown boundary label {label!r}; available: {sorted(self._boundaries)}")
        return self._boundaries[label]

    def sides_of_label(self, label: str):
        labels = self.patch.label_map
        return [f"{'uvw'[d]}{e}" for d in range(self.dim) for e in (0, 1)
                if labels.get(f"{'uvw'[d]}{e}", f"patch0/{'uvw'[d]}{e}") == label]

    def side_indices(self, side: str, offset: int = 0):
        if offset:
            raise NotImplementedError("clamped conditions (a second control-point layer) on hierarchical spaces")
        d, end = "uvw".index(side[0]), int(side[1:])
        L = self._levels
        return np.array([c for c, (l, j) in enumerate(self.columns)
                         if np.array(_unravel([j], L.n_func[l]))[d, 0] == (0 if end == 0 else L.n_func[l][d] - 1)],
                        dtype=np.int64)

    def summary(self) -> str:
        return (f"HierarchicalSpace(dim={self.dim}, vec={self.vec}, degree={self.degree}, levels="
                f"{self.hierarchy.n_levels}, n_elems={self.n_elems}, n_scalar_basis={self.n_scalar_basis}, "
                f"n_local_max={self.n_local_max})")


def _initial_keys(space):
    """(patch, level, element) of a tensor space's elements: all level 0."""
    keys = np.zeros((space.n_elems, 3), dtype=np.int64)
    keys[:, 2] = np.arange(space.n_elems)
    return keys


def refine_elements(space, marked, *, truncate: bool = True, admissible: bool = True) -> HierarchicalSpace:
    """Refine the marked elements of ``space`` (a single-patch tensor space or
    a hierarchical one; indices of this space's elements) and return the new
    THB space (hierarchical.py:1042-1110)."""
    if isinstance(space, HierarchicalSpace):
        patch, base, keys = space.patch, space.hierarchy.refined, space.elem_key
    else:
        if getattr(space, "cell_type", None) != "tensor" or not hasattr(space, "patch"):
            raise NotImplementedError("hierarchical refinement needs a single-patch tensor or THB space")
        patch, base, keys = space.patch, (), _initial_keys(space)
    marked = np.unique(np.asarray(marked, dtype=np.int64).reshape(-1))
    if marked.size and (marked.min() < 0 or marked.max() >= space.n_elems):
        raise IndexError(f"marked element index out of range for a space with {space.n_elems} elements")
    state = _State(patch, base)
    for e in marked:
        _, l, local = (int(v) for v in keys[e])
        state.mark(l, local)
    state.close(admissible)
    return HierarchicalSpace(patch, state.hierarchy(truncate, admissible), vec=space.vec)


def dorfler_mark(eta, frac: float = 0.3) -> np.ndarray:
    """Bulk marking: the fewest elements whose squared indicators reach
    ``frac`` of the total (hierarchical.py:1137-1156)."""
    eta = np.asarray(eta, dtype=float).reshape(-1)
    if not 0.0 < frac <= 1.0:
        raise ValueError(f"frac must lie in (0, 1], got {frac}")
    order = np.argsort(eta ** 2)[::-1]
    cum = np.cumsum(eta[order] ** 2)
    total = cum[-1] if cum.size else 0.0
    if total <= 0.0:
        return np.zeros(0, dtype=np.int64)
    return np.sort(order[: int(np.searchsorted(cum, frac * total) + 1)])
