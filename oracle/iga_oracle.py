"""CPU oracle for the Galerkin linear-solve path (NumPy / SciPy, FP64).

TEST INFRASTRUCTURE ONLY. This module is the checker: the tests, the smoke
check and the CPU-baseline leg of the benchmark call it to produce the answer
that the CUDA path must reproduce. Nothing in the product package imports it.

It restates, in vectorised NumPy, the reference algorithm of JAXIGA for
single-patch tensor-product NURBS spaces. Each function names the reference
function it follows (paths relative to the reference's ``src/jaxiga``):

* Bernstein bases and Bezier extraction        space/bernstein.py:16-284
* Gauss rule                                    space/pointset.py:98-136
* connectivity / element boxes / dense ops      space/function_space.py:300-369
* side control-point layers, Dirichlet sets     geometry/multipatch.py:99-131,
                                                forms/problem.py:179-302
* basis evaluation (rational, push-forward)     space/evaluation.py:95-172, 305-467
* element tangents                              forms/library.py:17-65, 108-181,
                                                forms/materials.py:53-112
* CSR pattern and scatter                       methods/_common.py:203-264,
                                                methods/galerkin.py:122-142
* load vector (source work of element_energy)   methods/_common.py:280-309
* SciPy SuperLU and Jacobi-CG host solves       solvers/linear.py:221-321
* true-residual diagnostics                     solvers/diagnostics.py:8-19
* relative L2 error                             post/norms.py:59-111

The matrix-free GPU default of the reference runs
``jax.scipy.sparse.linalg.cg`` (jax 0.11.1, pinned in the reference's
requirements-lock.txt; not vendored under the reference tree). Its published
algorithm -- preconditioned CG from x0 = 0, stopping when the *unpreconditioned*
residual satisfies r.r <= max(tol^2 b.b, atol^2) or after maxiter = 10 n
iterations -- is restated in :func:`jax_cg`.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


# --------------------------------------------------------------------------
# Bernstein bases and Bezier extraction (space/bernstein.py)
# --------------------------------------------------------------------------


def bernstein_basis(uhat, deg):
    """space/bernstein.py:79-97 -- de Casteljau-style recurrence, then /2^p."""
    uhat = np.atleast_1d(np.asarray(uhat, dtype=float))
    B = np.zeros((len(uhat), deg + 1))
    B[:, 0] = 1.0
    u1, u2 = 1 - uhat, 1 + uhat
    for j in range(1, deg + 1):
        saved = 0.0
        for k in range(j):
            temp = B[:, k].copy()
            B[:, k] = saved + u1 * temp
            saved = u2 * temp
        B[:, j] = saved
    return B / np.power(2.0, deg)


def _lower(uhat, deg, drop):
    """Degree ``deg - drop`` Bernstein rows scaled by 1/2^deg (bernstein.py:100-156)."""
    n = deg + 1 - drop
    u1, u2 = 1 - uhat, 1 + uhat
    B = np.zeros((len(uhat), n))
    B[:, 0] = 1.0
    for j in range(1, n):
        saved = 0.0
        for k in range(j):
            temp = B[:, k].copy()
            B[:, k] = saved + u1 * temp
            saved = u2 * temp
        B[:, j] = saved
    return B / np.power(2.0, deg)


def _difference(B, factor):
    zero = np.zeros((B.shape[0], 1))
    B = np.concatenate((zero, B, zero), axis=1)
    return (B[:, 0:-1] - B[:, 1:]) * factor


def bernstein_basis_deriv(uhat, deg):
    """space/bernstein.py:100-126."""
    uhat = np.atleast_1d(np.asarray(uhat, dtype=float))
    if deg == 0:
        return np.zeros((len(uhat), 1))
    return _difference(_lower(uhat, deg, 1), deg)


def bernstein_basis_2nd_deriv(uhat, deg):
    """space/bernstein.py:129-156."""
    uhat = np.atleast_1d(np.asarray(uhat, dtype=float))
    if deg < 2:
        return np.zeros((len(uhat), deg + 1))
    return _difference(_difference(_lower(uhat, deg, 2), deg - 1), deg)


def bezier_extraction(knot, deg):
    """Borden et al. Algorithm 1, as in space/bernstein.py:16-76.

    Returns the list of (deg+1, deg+1) operators, one per non-empty span.
    """
    knot = np.asarray(knot, dtype=float)
    m = len(knot) - deg - 1
    a, b = deg + 1, deg + 2
    C = [np.eye(deg + 1)]
    nb = 1
    while b <= m:
        C.append(np.eye(deg + 1))
        i = b
        while b <= m and knot[b] == knot[b - 1]:
            b += 1
        mult = b - i + 1
        if mult < deg:
            alphas = np.zeros(deg - mult)
            numer = knot[b - 1] - knot[a - 1]
            for j in range(deg, mult, -1):
                alphas[j - mult - 1] = numer / (knot[a + j - 1] - knot[a - 1])
            r = deg - mult
            for j in range(1, r + 1):
                save = r - j + 1
                s = mult + j
                for k in range(deg + 1, s, -1):
                    alpha = alphas[k - s - 1]
                    C[nb - 1][:, k - 1] = alpha * C[nb - 1][:, k - 1] + (1 - alpha) * C[nb - 1][:, k - 2]
                if b <= m:
                    C[nb][save - 1: save + j, save - 1] = C[nb - 1][deg - j: deg + 1, deg]
            nb += 1
            if b <= m:
                a, b = b, b + 1
        elif mult == deg:
            if b <= m:
                nb += 1
                a, b = b, b + 1
    return C[:nb]


def element_spans(knot, deg):
    """space/bernstein.py:261-284: non-empty spans and first basis index i-deg."""
    knot = np.asarray(knot, dtype=float)
    idx = np.flatnonzero(knot[1:] > knot[:-1])
    return knot[idx], knot[idx + 1], (idx - deg).astype(int)


def tensor(factors):
    """space/bernstein.py:159-171: per-point tensor product, first direction fastest."""
    out = factors[-1]
    for d in range(len(factors) - 2, -1, -1):
        out = np.einsum("q...,qb->q...b", out, factors[d])
    return out.reshape(out.shape[0], -1)


def voigt_pairs(dim):
    return [(i, j) for i in range(dim) for j in range(i, dim)]


def bernstein_tensor(pts, deg, order=1):
    """space/bernstein.py:174-232."""
    pts = np.atleast_2d(np.asarray(pts, dtype=float))
    dim = pts.shape[1]
    vals = [bernstein_basis(pts[:, d], deg[d]) for d in range(dim)]
    ders = [bernstein_basis_deriv(pts[:, d], deg[d]) for d in range(dim)]
    ders2 = [bernstein_basis_2nd_deriv(pts[:, d], deg[d]) for d in range(dim)]
    B = tensor(vals)
    dB = np.stack([tensor([ders[k] if k == d else vals[k] for k in range(dim)]) for d in range(dim)], axis=1)
    d2B = None
    if order >= 2:
        cols = []
        for i, j in voigt_pairs(dim):
            if i == j:
                f = [ders2[k] if k == i else vals[k] for k in range(dim)]
            else:
                f = [ders[k] if k in (i, j) else vals[k] for k in range(dim)]
            cols.append(tensor(f))
        d2B = np.stack(cols, axis=1)
    return B, dB, d2B


def gauss_rule(n_per_dir):
    """space/pointset.py:98-112: Gauss-Legendre tensor rule, first direction fastest."""
    per = [np.polynomial.legendre.leggauss(n) for n in n_per_dir]
    grids = np.meshgrid(*[p[0] for p in per], indexing="ij")
    wgrids = np.meshgrid(*[p[1] for p in per], indexing="ij")
    pts = np.stack([g.ravel(order="F") for g in grids], axis=1)
    wts = np.prod([w.ravel(order="F") for w in wgrids], axis=0)
    return pts, wts


# --------------------------------------------------------------------------
# Space (space/function_space.py)
# --------------------------------------------------------------------------


class Space:
    """Single-patch tensor-product space: what ``build_function_space`` yields."""

    def __init__(self, knots, degree, cpts, wgts, vec=1):
        self.knots = [np.asarray(k, dtype=float) for k in knots]
        self.degree = tuple(int(p) for p in degree)
        self.dim = len(self.degree)
        self.cpts = np.asarray(cpts, dtype=float)
        self.wgts = np.asarray(wgts, dtype=float)
        self.vec = int(vec)
        self.n_cp = [len(k) - p - 1 for k, p in zip(self.knots, self.degree)]
        self.n_scalar = int(np.prod(self.n_cp))
        self.n_dofs = self.n_scalar * self.vec
        self.spans = [element_spans(self.knots[d], self.degree[d]) for d in range(self.dim)]
        self.ext1d = [np.stack(bezier_extraction(self.knots[d], self.degree[d])) for d in range(self.dim)]
        self.n_span = [len(s[0]) for s in self.spans]
        self.n_elems = int(np.prod(self.n_span))
        self.n_local = int(np.prod([p + 1 for p in self.degree]))
        self._connectivity()

    def _connectivity(self):
        """function_space.py:326-369, vectorised over elements."""
        dim = self.dim
        idx = np.indices(self.n_span[::-1]).reshape(dim, -1)[::-1]  # first direction fastest
        strides = np.array([1, *np.cumprod(self.n_cp[:-1])], dtype=np.int64)
        boxes = np.zeros((self.n_elems, 2 * dim))
        local = np.indices([p + 1 for p in self.degree[::-1]]).reshape(dim, -1)[::-1]
        ien = np.zeros((self.n_elems, self.n_local), dtype=np.int64)
        for d in range(dim):
            lo, hi, first = self.spans[d]
            boxes[:, d] = lo[idx[d]]
            boxes[:, dim + d] = hi[idx[d]]
            ien += (first[idx[d]][:, None] + local[d][None, :]) * strides[d]
        self.elem_idx = idx  # (dim, n_e) per-direction span index
        self.elem_dofs = ien
        self.elem_vertex = boxes

    def extraction(self, elems):
        """Dense kron(kron(C_w, C_v), C_u) for the given elements (function_space.py:315-323)."""
        out = []
        for e in np.atleast_1d(elems):
            C = self.ext1d[-1][self.elem_idx[-1][e]]
            for d in range(self.dim - 2, -1, -1):
                C = np.kron(C, self.ext1d[d][self.elem_idx[d][e]])
            out.append(C)
        return np.stack(out)

    def expand(self, scalar_dofs):
        """function_space.py:300-312: interleaved vector DOFs vec*i + c."""
        scalar_dofs = np.asarray(scalar_dofs)
        if self.vec == 1:
            return scalar_dofs
        out = self.vec * scalar_dofs[..., :, None] + np.arange(self.vec)
        return out.reshape(*scalar_dofs.shape[:-1], -1)

    def side_indices(self, side, offset=0):
        """geometry/multipatch.py:99-131."""
        direction = "uvw".index(side[0])
        end = int(side[1:])
        fixed = offset if end == 0 else self.n_cp[direction] - 1 - offset
        strides = np.array([1, *np.cumprod(self.n_cp[:-1])], dtype=int)
        ranges = [np.arange(n) for n in self.n_cp]
        ranges[direction] = np.array([fixed])
        mesh = np.meshgrid(*ranges, indexing="ij")
        return sum(m.ravel(order="F") * strides[d] for d, m in enumerate(mesh)).astype(int)

    def boundary_dofs(self):
        sides = [f"{'uvw'[d]}{e}" for d in range(self.dim) for e in (0, 1)]
        return np.unique(np.concatenate([self.side_indices(s) for s in sides]))


def dirichlet(space, specs):
    """Prescribed DOFs and values (forms/problem.py:179-302).

    ``specs`` is a list of ``(kind, where, value, component)`` with kind
    ``"dirichlet"`` or ``"clamped"``; ``where`` is a list of side names or a
    predicate over boundary control points; ``value`` a constant, a
    per-component sequence, or a callable ``g(x)``.
    """
    entries = {}
    for kind, where, value, comp in specs:
        if kind == "clamped":
            sd = set()
            for s in where:
                sd.update(space.side_indices(s).tolist())
                sd.update(space.side_indices(s, offset=1).tolist())
            scalar = np.array(sorted(sd), dtype=int)
        elif callable(where):
            allb = space.boundary_dofs()
            mask = np.asarray(where(space.cpts[allb]), dtype=bool)
            scalar = allb[mask]
        else:
            scalar = np.unique(np.concatenate([space.side_indices(s) for s in where]))
        comps = range(space.vec) if comp is None else [comp]
        for s_ in scalar:
            val = np.atleast_1d(np.asarray(value(space.cpts[s_]) if callable(value) else value, dtype=float))
            for c in comps:
                entries[int(space.vec * s_ + c)] = val[c] if val.shape[0] == space.vec else val[0]
    dofs = np.array(sorted(entries), dtype=np.int64)
    vals = np.array([entries[int(d)] for d in dofs], dtype=float)
    return dofs, vals


# --------------------------------------------------------------------------
# Evaluation (space/evaluation.py)
# --------------------------------------------------------------------------


def evaluate(space, elems, n_q=None, order=1, ref=None, weights=None):
    """BasisData on the interior Gauss set for ``elems`` (evaluation.py:305-467),
    or on the reference points ``ref`` (n_q, dim) shared by every element with
    reference weights ``weights`` (pointset.py:27-75; unit weights if None).

    Returns dict with R (n_e,n_q,n_loc), dR (n_e,n_q,dim,n_loc),
    d2R (n_e,n_q,n_d2,n_loc) or None, x (n_e,n_q,dim), w (n_e,n_q).
    """
    dim = space.dim
    if ref is None:
        nq = [(p + 1) if n_q is None else int(n_q) for p in space.degree]
        ref, wq = gauss_rule(nq)
    else:
        ref = np.asarray(ref, dtype=float).reshape(-1, dim)
        wq = np.ones(len(ref)) if weights is None else np.asarray(weights, dtype=float)
    B, dB, d2B = bernstein_tensor(ref, space.degree, order=order)
    elems = np.asarray(elems)
    boxes = space.elem_vertex[elems]
    scale = 2.0 / (boxes[:, dim:] - boxes[:, :dim])
    C = space.extraction(elems)
    dofs = space.elem_dofs[elems]
    cpts = space.cpts[dofs]
    wgts = space.wgts[dofs]

    N = np.einsum("eij,qj->eqi", C, B)
    dN = np.einsum("eij,qdj->eqdi", C, dB) * scale[:, None, :, None]
    pairs = voigt_pairs(dim) if order >= 2 else []
    d2N = None
    if order >= 2:
        pair_scale = np.stack([scale[:, a] * scale[:, b] for a, b in pairs], axis=1)
        d2N = np.einsum("eij,qkj->eqki", C, d2B) * pair_scale[:, None, :, None]

    # _rational_and_pushforward (evaluation.py:95-172), vectorised over (e, q)
    M = N * wgts[:, None, :]
    dM = dN * wgts[:, None, None, :]
    W = M.sum(-1)
    dW = dM.sum(-1)
    R = M / W[..., None]
    dR = dM / W[..., None, None] - M[:, :, None, :] * dW[..., None] / W[..., None, None] ** 2
    d2R = None
    if order >= 2:
        d2M = d2N * wgts[:, None, None, :]
        d2W = d2M.sum(-1)
        rows = []
        for k, (a, b) in enumerate(pairs):
            rows.append(
                d2M[:, :, k] / W[..., None]
                - (dM[:, :, a] * dW[..., b, None] + dM[:, :, b] * dW[..., a, None] + M * d2W[..., k, None]) / W[..., None] ** 2
                + 2 * M * dW[..., a, None] * dW[..., b, None] / W[..., None] ** 3
            )
        d2R = np.stack(rows, axis=2)
    x = np.einsum("eqn,eni->eqi", R, cpts)
    J = np.einsum("eqan,eni->eqai", dR, cpts)  # dxdxi[a, i]
    detJ = np.linalg.det(J)
    dR_phys = np.linalg.solve(J, dR)
    d2R_phys = None
    if order >= 2:
        d2x = np.einsum("eqkn,eni->eqki", d2R, cpts)
        T = np.zeros(J.shape[:2] + (len(pairs), len(pairs)))
        for r, (a, b) in enumerate(pairs):
            for c, (i, j) in enumerate(pairs):
                T[..., r, c] = J[..., a, i] * J[..., b, j] + (J[..., a, j] * J[..., b, i] if i != j else 0.0)
        d2R_phys = np.linalg.solve(T, d2R - np.einsum("eqki,eqin->eqkn", d2x, dR_phys))
    jac = np.prod(2.0 / scale, axis=1) / 2.0 ** dim
    w = wq[None, :] * np.abs(detJ) * jac[:, None]
    return {"R": R, "dR": dR_phys, "d2R": d2R_phys, "x": x, "w": w, "dofs": dofs}


def evaluate_boundary(space, elems, sides, ref, wref):
    """Boundary BasisData (evaluation.py:174-193, 432-455): per face f (side
    sides[f] = 2 direction + end of element elems[f]) and point q at ref[f, q]
    with reference weight wref[f, q]: R, x, outward unit normal and
    w = wref |surface Jacobian| prod of tangential half-widths."""
    dim = space.dim
    R, X, N, W = [], [], [], []
    for f, (e, code) in enumerate(zip(np.asarray(elems), np.asarray(sides))):
        b = evaluate(space, [e], ref=ref[f], weights=np.ones(len(ref[f])))
        direction, end = divmod(int(code), 2)
        lo, hi = space.elem_vertex[e, :dim], space.elem_vertex[e, dim:]
        # dxdxi[a, i] rows are the parametric tangents, from the (rational) basis
        C = space.extraction([e])[0]
        B, dB, _ = bernstein_tensor(ref[f], space.degree, order=1)
        scale = 2.0 / (hi - lo)
        Nb = B @ C.T
        dNb = np.einsum("qdj,ij->qdi", dB, C) * scale[None, :, None]
        dofs = space.elem_dofs[e]
        wts = space.wgts[dofs]
        M, dM = Nb * wts, dNb * wts
        Wq, dW = M.sum(-1), dM.sum(-1)
        dR = dM / Wq[:, None, None] - M[:, None, :] * dW[:, :, None] / Wq[:, None, None] ** 2
        J = np.einsum("qan,ni->qai", dR, space.cpts[dofs])
        tang = [a for a in range(dim) if a != direction]
        if dim == 2:
            sj = np.linalg.norm(J[:, tang[0]], axis=1)
        else:
            sj = np.linalg.norm(np.cross(J[:, tang[0]], J[:, tang[1]]), axis=1)
        e_d = np.zeros(dim)
        e_d[direction] = 1.0
        nrm = np.linalg.solve(J, np.broadcast_to(e_d, (len(J), dim))[..., None])[..., 0]
        nrm = nrm / np.linalg.norm(nrm, axis=1, keepdims=True) * (1.0 if end == 1 else -1.0)
        half = np.prod([(hi[a] - lo[a]) / 2.0 for a in tang])
        R.append(b["R"][0])
        X.append(b["x"][0])
        N.append(nrm)
        W.append(wref[f] * sj * half)
    return {"R": np.stack(R), "x": np.stack(X), "normal": np.stack(N), "w": np.stack(W),
            "dofs": space.elem_dofs[np.asarray(elems)]}


def neumann_load(space, elems, sides, ref, wref, traction):
    """F_i,c = sum_q w t_c(x, n) R_i on the faces (the negative gradient of
    neumann_work, methods/_common.py:312-318); traction(x, n) -> (n_pts, vec)."""
    b = evaluate_boundary(space, elems, sides, ref, wref)
    nf, nq = b["w"].shape
    t = np.asarray(traction(b["x"].reshape(-1, space.dim), b["normal"].reshape(-1, space.dim)), dtype=float)
    t = t.reshape(nf, nq, space.vec)
    Fe = np.einsum("fq,fqc,fqi->fic", b["w"], t, b["R"]).reshape(nf, -1)
    F = np.zeros(space.n_dofs)
    np.add.at(F, space.expand(b["dofs"]), Fe)
    return F


# --------------------------------------------------------------------------
# Element tangents (forms/library.py, forms/materials.py)
# --------------------------------------------------------------------------


def isotropic(E, nu, dim, plane="stress"):
    """forms/materials.py:53-88."""
    if dim == 3:
        z, s = 0.0, (1 - 2 * nu) / 2
        return E / ((1 + nu) * (1 - 2 * nu)) * np.array([
            [1 - nu, nu, nu, z, z, z], [nu, 1 - nu, nu, z, z, z], [nu, nu, 1 - nu, z, z, z],
            [z, z, z, s, z, z], [z, z, z, z, s, z], [z, z, z, z, z, s]])
    if plane == "stress":
        return E / (1 - nu**2) * np.array([[1, nu, 0], [nu, 1, 0], [0, 0, (1 - nu) / 2]])
    return E / ((1 + nu) * (1 - 2 * nu)) * np.array([[1 - nu, nu, 0], [nu, 1 - nu, 0], [0, 0, (1 - 2 * nu) / 2]])


def strain_displacement(dR):
    """forms/library.py:17-37 (engineering Voigt, interleaved components)."""
    n_e, n_q, dim, n_loc = dR.shape
    ns = 3 if dim == 2 else 6
    B = np.zeros((n_e, n_q, ns, n_loc, dim))
    if dim == 2:
        B[:, :, 0, :, 0] = dR[:, :, 0]
        B[:, :, 1, :, 1] = dR[:, :, 1]
        B[:, :, 2, :, 0] = dR[:, :, 1]
        B[:, :, 2, :, 1] = dR[:, :, 0]
    else:
        B[:, :, 0, :, 0] = dR[:, :, 0]
        B[:, :, 1, :, 1] = dR[:, :, 1]
        B[:, :, 2, :, 2] = dR[:, :, 2]
        B[:, :, 3, :, 1] = dR[:, :, 2]
        B[:, :, 3, :, 2] = dR[:, :, 1]
        B[:, :, 4, :, 0] = dR[:, :, 2]
        B[:, :, 4, :, 2] = dR[:, :, 0]
        B[:, :, 5, :, 0] = dR[:, :, 1]
        B[:, :, 5, :, 1] = dR[:, :, 0]
    return B.reshape(n_e, n_q, ns, n_loc * dim)


def element_tangents(op, basis, params, vec=1):
    """K_e for op in {"poisson", "elasticity", "plate"}.

    poisson:    library.py:54-65  K = sum_q w a0 dR^T dR (x) I_vec
    elasticity: library.py:174-181 K = sum_q w B^T C B
    plate:      library.py:125-132 K = sum_q w B_k^T D B_k, B_k = -(d2R_xx, d2R_yy, 2 d2R_xy)
    """
    w = basis["w"]
    if op == "poisson":
        a0 = params.get("a0", 1.0)
        a0 = np.broadcast_to(np.asarray(a0, dtype=float), w.shape)
        scalar = np.einsum("eq,eqdi,eqdj->eij", w * a0, basis["dR"], basis["dR"])
        if vec == 1:
            return scalar
        n = scalar.shape[1]
        return np.einsum("eij,cd->eicjd", scalar, np.eye(vec)).reshape(-1, n * vec, n * vec)
    if op == "elasticity":
        dim = basis["dR"].shape[2]
        C = isotropic(params["E"], params["nu"], dim, params.get("plane", "stress"))
        return _btdb(w, strain_displacement(basis["dR"]), C)
    if op == "plate":
        E, nu, t = params["E"], params["nu"], params["t"]
        D = E * t**3 / (12 * (1 - nu**2)) * np.array([[1, nu, 0], [nu, 1, 0], [0, 0, (1 - nu) / 2]])
        d2R = basis["d2R"]
        B = -np.stack([d2R[:, :, 0], d2R[:, :, 2], 2.0 * d2R[:, :, 1]], axis=2)
        return _btdb(w, B, D)
    raise ValueError(op)


def _btdb(w, B, D):
    """sum_q w_q B_q^T D B_q per element, as one batched matrix product over the
    stacked (point, strain) rows (the contraction of library.py:125-132, 174-181)."""
    e, q, ns, n = B.shape
    DB = np.einsum("st,eqtj->eqsj", D, B) * w[:, :, None, None]
    return np.matmul(B.reshape(e, q * ns, n).transpose(0, 2, 1), DB.reshape(e, q * ns, n))


# --------------------------------------------------------------------------
# Assembly (methods/_common.py, methods/galerkin.py)
# --------------------------------------------------------------------------


class Assembled:
    """Free-free CSR operator plus the full operator for the Dirichlet lift."""

    def __init__(self, space, op, params, prescribed, values, source_qp=None,
                 n_q=None, chunk=2048, need_full=True):
        self.space = space
        vec = space.vec
        n = space.n_dofs
        self.prescribed = np.asarray(prescribed, dtype=np.int64)
        self.values = np.asarray(values, dtype=float)
        self.free = np.setdiff1d(np.arange(n), self.prescribed)
        order = 2 if op == "plate" else 1
        gd_all = space.expand(space.elem_dofs)
        rows, cols, vals = [], [], []
        F = np.zeros(n)
        diag_full = np.zeros(n)
        for lo in range(0, space.n_elems, chunk):
            el = np.arange(lo, min(lo + chunk, space.n_elems))
            basis = evaluate(space, el, n_q=n_q, order=order)
            p = dict(params)
            if "a0_qp" in params:
                p["a0"] = params["a0_qp"][el]
            Ke = element_tangents(op, basis, p, vec)
            gd = gd_all[el]
            np.add.at(diag_full, gd.ravel(), np.diagonal(Ke, axis1=1, axis2=2).ravel())
            rows.append(np.repeat(gd, gd.shape[1], axis=1).ravel())
            cols.append(np.tile(gd, (1, gd.shape[1])).ravel())
            vals.append(Ke.ravel())
            if source_qp is not None:
                fq = np.asarray(source_qp)[el].reshape(len(el), basis["w"].shape[1], vec)
                Fe = np.einsum("eq,eqc,eqi->eic", basis["w"], fq, basis["R"]).reshape(len(el), -1)
                np.add.at(F, gd.ravel(), Fe.ravel())
        rows = np.concatenate(rows)
        cols = np.concatenate(cols)
        vals = np.concatenate(vals)
        K = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
        K.sum_duplicates()
        K.sort_indices()
        self.K_full = K if need_full else None
        self.K = K[self.free][:, self.free].tocsr()
        self.K.sort_indices()
        self.F = F
        g = np.zeros(n)
        g[self.prescribed] = self.values
        self.g = g
        self.b = (F - K @ g)[self.free]
        self.diag = diag_full[self.free]

    def lift(self, u_free):
        """function_space.py:576-584."""
        u = np.zeros(self.space.n_dofs)
        u[self.free] = u_free
        u[self.prescribed] = self.values
        return u


def csr_pattern(elem_dofs, n_dofs, vec, free):
    """methods/_common.py:203-264: unique free-free keys in CSR order plus scatter map."""
    n = len(free)
    full_to_free = np.full(n_dofs + vec, -1, dtype=np.int64)
    full_to_free[np.asarray(free)] = np.arange(n, dtype=np.int64)
    ed = np.asarray(elem_dofs)
    if vec > 1:
        ed = (vec * ed[..., :, None] + np.arange(vec)).reshape(ed.shape[0], -1)
    f = full_to_free[ed]
    keys = f[:, :, None] * n + f[:, None, :]
    valid = (f[:, :, None] >= 0) & (f[:, None, :] >= 0)
    unique = np.unique(keys[valid])
    scatter = np.full(keys.shape, len(unique), dtype=np.int32)
    scatter[valid] = np.searchsorted(unique, keys[valid]).astype(np.int32)
    rows = (unique // n).astype(np.int32)
    columns = (unique % n).astype(np.int32)
    indptr = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32)
    return indptr, columns, rows, scatter


# --------------------------------------------------------------------------
# Solvers (solvers/linear.py, solvers/diagnostics.py)
# --------------------------------------------------------------------------


def scipy_superlu(A, b):
    """solvers/linear.py:221-258 with the symmetric Galerkin pattern (MMD_AT_PLUS_A)."""
    factor = spla.splu(A.tocsc(), permc_spec="MMD_AT_PLUS_A", options={"SymmetricMode": True})
    return factor.solve(np.asarray(b)).astype(np.float64)


def scipy_cg(A, b, tol, maxiter=None, preconditioner="jacobi"):
    """solvers/linear.py:261-321: SciPy CG with up to three true-residual restarts.

    Returns (u, iterations used).
    """
    precond = None
    if preconditioner == "jacobi":
        diagonal = A.diagonal()
        inverse = np.ones_like(diagonal)
        np.divide(1.0, diagonal, out=inverse, where=diagonal != 0)
        precond = spla.LinearOperator(A.shape, matvec=lambda v: inverse * v, dtype=A.dtype)
    rhs = np.asarray(b)
    u = np.zeros_like(rhs)
    residual = rhs.copy()
    norm = np.linalg.norm(residual)
    target = 0.5 * tol * norm
    remaining = maxiter if maxiter is not None else 10 * len(rhs)
    total = 0
    for attempt in range(4):
        if norm <= target or remaining <= 0:
            break
        used = 0

        def count(_):
            nonlocal used
            used += 1

        correction, info = spla.cg(A, residual, M=precond, rtol=min(0.5, 0.5 * target / norm),
                                   atol=0.0, maxiter=remaining, callback=count)
        remaining -= used
        total += used
        candidate = u + correction
        actual = rhs - A @ candidate
        actual_norm = np.linalg.norm(actual)
        if attempt > 0 and actual_norm >= norm:
            break
        u, residual, norm = candidate, actual, actual_norm
        if info != 0 or used == 0 or not np.isfinite(norm):
            break
    return u, total


def jax_cg(matvec, b, tol, maxiter=None, inv_diag=None, atol=0.0, x0=None):
    """Restatement of jax.scipy.sparse.linalg.cg (jax 0.11.1, ``_cg_solve``).

    x0 = 0; stop when r.r <= max(tol^2 b.b, atol^2) (unpreconditioned r when a
    preconditioner is given) or after ``maxiter`` (default 10 n) iterations.
    Returns (x, iterations).
    """
    b = np.asarray(b, dtype=float)
    if maxiter is None:
        maxiter = 10 * b.size
    M = (lambda v: v) if inv_diag is None else (lambda v: inv_diag * v)
    bs = b @ b
    atol2 = max(tol**2 * bs, atol**2)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=float)
    r = b - matvec(x)
    z = M(r)
    p = z.copy()
    gamma = r @ z
    k = 0
    while True:
        rs = gamma if inv_diag is None else r @ r
        if not (rs > atol2 and k < maxiter):
            break
        Ap = matvec(p)
        alpha = gamma / (p @ Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = M(r)
        gamma_new = r @ z
        beta = gamma_new / gamma
        p = z + beta * p
        gamma = gamma_new
        k += 1
    return x, k


def bicgstab(matvec, b, tol, maxiter=None, inv_diag=None, atol=0.0):
    """BiCGSTAB (van der Vorst, 1992) with right preconditioning M, in the
    stopping semantics of jax.scipy.sparse.linalg.bicgstab (the reference's
    method="bicgstab", solvers/linear.py:152-171): x0 = 0, stop when r.r <=
    max(tol^2 b.b, atol^2), or when s.s already is (x then takes the half step).
    Returns (x, iterations)."""
    b = np.asarray(b, dtype=float)
    maxiter = 10 * b.size if maxiter is None else maxiter
    M = (lambda v: v) if inv_diag is None else (lambda v: inv_diag * v)
    atol2 = max(tol**2 * (b @ b), atol**2)
    x = np.zeros_like(b)
    r = b.copy()
    rhat = r.copy()
    rho = alpha = omega = 1.0
    p = np.zeros_like(b)
    v = np.zeros_like(b)
    k = 0
    while r @ r > atol2 and k < maxiter:
        rho_new = rhat @ r
        beta = (rho_new / rho) * (alpha / omega)
        rho = rho_new
        p = r + beta * (p - omega * v)
        ph = M(p)
        v = matvec(ph)
        alpha = rho / (rhat @ v)
        s = r - alpha * v
        if s @ s <= atol2:
            x = x + alpha * ph
            r = s
            k += 1
            break
        sh = M(s)
        t = matvec(sh)
        omega = (t @ s) / (t @ t)
        x = x + alpha * ph + omega * sh
        r = s - omega * t
        k += 1
    return x, k


def reliable_cg(matvec, matvec32, b, tol, delta=1e-2, inv_diag=None, maxiter=None):
    """FP32 Jacobi-PCG with reliable FP64 updates, as the device solver runs it.

    Not part of the reference (its solves are FP64 only): this restates the
    reliable-update scheme of Sleijpen and van der Vorst (1996), in the form the
    CUDA path ``jxb_mixed_pcg`` uses, so that its convergence can be checked.
    The FP32 iteration runs on the residual scaled to unit norm. A segment ends
    when the FP32 recursive residual has fallen by ``delta`` or below
    ``tol ||b||``; then x += ||r_seg|| x32, the residual is recomputed in FP64
    (``matvec``), and the FP32 iteration resumes from it with the search
    direction kept (rescaled to the new units). Dot products are FP64 sums of
    FP32 products; alpha and beta are rounded to FP32 as on the device.
    Returns (x, FP32 iterations, updates).
    """
    b = np.asarray(b, dtype=float)
    if maxiter is None:
        maxiter = 10 * b.size
    f32 = np.float32
    inv32 = (np.ones_like(b) if inv_diag is None else np.asarray(inv_diag)).astype(f32)

    def dot(u, v):
        return float(np.dot(u.astype(float), v.astype(float)))

    x = np.zeros_like(b)
    res = b.copy()
    bn = float(np.linalg.norm(b))
    rn = bn
    k = updates = 0
    p = None
    rn_seg = rn
    while rn > tol * bn and k < maxiter:
        r = (res * (1.0 / rn)).astype(f32)
        z = inv32 * r
        p = z.copy() if p is None else p * f32(rn_seg / rn)
        rn_seg = rn
        gamma, rr = dot(r, z), dot(r, r)
        seg2 = max(delta, tol * bn / rn) ** 2 * rr
        xs = np.zeros_like(r)
        while rr > seg2 and k < maxiter:
            Ap = np.asarray(matvec32(p), dtype=f32)
            alpha = f32(gamma / dot(p, Ap))
            xs += alpha * p
            r -= alpha * Ap
            z = inv32 * r
            gnew, rr = dot(r, z), dot(r, r)
            p = z + f32(gnew / gamma) * p
            gamma = gnew
            k += 1
        x = x + rn_seg * xs.astype(float)
        res = b - matvec(x)
        rn = float(np.linalg.norm(res))
        updates += 1
        if not rn < rn_seg:
            break
    return x, k, updates


def jacobi_inverse(diagonal):
    """solvers/linear.py:427-431: 1/d where |d| > 0, else 1."""
    diagonal = np.asarray(diagonal)
    safe = np.where(np.abs(diagonal) > 0, diagonal, 1.0)
    return np.where(np.abs(diagonal) > 0, 1.0 / safe, 1.0)


def linear_diagnostics(matvec, u, b, tol):
    """solvers/diagnostics.py:8-19."""
    norm = float(np.linalg.norm(matvec(u) - b))
    scale = float(np.linalg.norm(b))
    rel = norm / (scale if scale > 0 else 1.0)
    finite = bool(np.isfinite(norm) and np.all(np.isfinite(u)))
    return {"residual": norm, "relative_residual": rel,
            "converged": bool(finite and norm <= tol * scale), "finite": finite}


def errornorm_l2(space, u, exact, n_q=None, chunk=4096):
    """post/norms.py:59-111, relative L2 error against ``exact(x) -> (n, vec)``."""
    num = den = 0.0
    for lo in range(0, space.n_elems, chunk):
        el = np.arange(lo, min(lo + chunk, space.n_elems))
        basis = evaluate(space, el, n_q=n_q)
        ul = u[space.expand(basis["dofs"])].reshape(len(el), -1, space.vec)
        uh = np.einsum("eqn,enc->eqc", basis["R"], ul)
        ue = np.asarray(exact(basis["x"].reshape(-1, space.dim))).reshape(uh.shape)
        num += np.sum(basis["w"] * np.sum((uh - ue) ** 2, -1))
        den += np.sum(basis["w"] * np.sum(ue**2, -1))
    return float(np.sqrt(num / den))


def interpolate_qp(space, coef, n_q=None, chunk=4096):
    """Field sum_i R_i c_i at the Gauss points, (n_e, n_q, ncomp)."""
    coef = np.asarray(coef, dtype=float)
    coef2 = coef.reshape(space.n_scalar, -1)
    out = []
    for lo in range(0, space.n_elems, chunk):
        el = np.arange(lo, min(lo + chunk, space.n_elems))
        basis = evaluate(space, el, n_q=n_q)
        out.append(np.einsum("eqn,enc->eqc", basis["R"], coef2[basis["dofs"]]))
    return np.concatenate(out)


def residual_indicator(space, u, problem_kind, params, source=None, n_q=None, elems=None):
    """Explicit residual indicators (post/estimators.py:33-88): eta_e^2 = h_e^2
    sum_q w |r|^2, h_e = |e|^(1/dim), on n_q = p + 2 Gauss points per
    direction, r = -a0 lap u - f (Poisson) or r = -((lam + mu) grad div u +
    mu lap u) - f (isotropic elasticity; plane stress in 2D); ``source(x)`` ->
    (n_pts, vec); ``space`` any view ``evaluate`` takes (tensor or padded THB)."""
    dim, vec = space.dim, (1 if problem_kind == "poisson" else space.dim)
    n_q = max(space.degree) + 2 if n_q is None else n_q
    elems = np.arange(space.n_elems) if elems is None else np.asarray(elems)
    b = evaluate(space, elems, n_q=n_q, order=2)
    pairs = voigt_pairs(dim)
    U = np.concatenate([np.asarray(u, dtype=float).reshape(-1, vec), np.zeros((1, vec))])[b["dofs"]]  # (e, n, vec)
    H = np.zeros(b["w"].shape + (vec, dim, dim))
    for k, (a, c) in enumerate(pairs):
        H[..., a, c] = H[..., c, a] = np.einsum("eqn,enc->eqc", b["d2R"][:, :, k], U)[..., None][..., 0]
    f = np.zeros(b["w"].shape + (vec,))
    if source is not None:
        f = np.asarray(source(b["x"].reshape(-1, dim)), dtype=float).reshape(f.shape)
    lap = np.trace(H, axis1=-2, axis2=-1)                                   # (e, q, vec)
    if problem_kind == "poisson":
        r = -params["a0"] * lap - f
    else:
        E, nu = params["E"], params["nu"]
        mu = E / (2 * (1 + nu))
        lam = E * nu / ((1 + nu) * (1 - 2 * nu)) if dim == 3 else E * nu / (1 - nu**2)
        graddiv = np.einsum("eqjij->eqi", H)                                # d_i sum_j d_j u_j
        r = -((lam + mu) * graddiv + mu * lap) - f
    h = b["w"].sum(1) ** (1.0 / dim)
    return np.sqrt(h**2 * np.sum(b["w"] * np.sum(r**2, -1), 1))
