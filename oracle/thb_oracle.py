"""CPU restatement of the Galerkin operator on truncated hierarchical spaces
(test infrastructure).

TEST INFRASTRUCTURE ONLY: the tests use it to check the device operator on
THB spaces (csrc/thb.cu, jaxiga_b200/thb.py). Nothing in the product package
imports it.

A THB space is in the padded-element form of the reference
(src/jaxiga/space/function_space.py:23-38): per element the supported
functions (padding index n_scalar_basis) and the extraction rows mapping the
element's Bernstein polynomials to them (zero rows for the padding). The
reference evaluates such a space with the same code as a tensor one
(src/jaxiga/space/evaluation.py:305-467), gathering control data through
one-longer arrays whose extra entry is inert; ``ThbSpace`` gives the tensor
oracle's ``evaluate`` exactly that view, so the element tangents
(src/jaxiga/forms/library.py:54-65) and the CSR scatter
(src/jaxiga/methods/galerkin.py:122-148) are the tensor oracle's.

Pinned by tests/golden/thb_golden.npz (make_thb_golden.py runs the
reference's own construction and assembly).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import iga_oracle as O


class ThbSpace:
    """Padded-element space view for ``iga_oracle.evaluate``."""

    def __init__(self, elem_dofs, extraction, elem_vertex, cpts, wgts, degree):
        self.elem_dofs = np.asarray(elem_dofs, dtype=np.int64)
        self._ext = np.asarray(extraction, dtype=float)
        self.elem_vertex = np.asarray(elem_vertex, dtype=float)
        self.n_scalar = len(wgts)
        # one-longer control data: the padding index reads an inert entry
        self.cpts = np.concatenate([np.asarray(cpts, dtype=float), np.zeros((1, np.shape(cpts)[1]))])
        self.wgts = np.concatenate([np.asarray(wgts, dtype=float), np.ones(1)])
        self.degree = tuple(int(p) for p in degree)
        self.dim = len(self.degree)
        self.vec = 1
        self.n_elems = len(self.elem_dofs)

    @classmethod
    def of(cls, space):
        return cls(space.elem_dofs, space.extraction, space.elem_vertex, space.cpts, space.wgts, space.degree)

    def extraction(self, elems):
        return self._ext[np.asarray(elems)]


def assemble_poisson(S, a0, prescribed, source_qp=None, chunk=1024):
    """(K_ff CSR, F on all DOFs, free DOFs, Gauss-point x and w) of
    -div(a0 grad u) = f on the THB space ``S``; a0 scalar or (n_e, n_q)."""
    n = S.n_scalar
    rows, cols, vals = [], [], []
    F = np.zeros(n + 1)
    xs, ws = [], []
    for lo in range(0, S.n_elems, chunk):
        el = np.arange(lo, min(lo + chunk, S.n_elems))
        basis = O.evaluate(S, el)
        a = a0 if np.ndim(a0) == 0 else np.asarray(a0)[el]
        Ke = O.element_tangents("poisson", basis, {"a0": a})
        gd = S.elem_dofs[el]
        rows.append(np.repeat(gd, gd.shape[1], axis=1).ravel())
        cols.append(np.tile(gd, (1, gd.shape[1])).ravel())
        vals.append(Ke.ravel())
        if source_qp is not None:
            Fe = np.einsum("eq,eq,eqi->ei", basis["w"], np.asarray(source_qp)[el], basis["R"])
            np.add.at(F, gd.ravel(), Fe.ravel())
        xs.append(basis["x"])
        ws.append(basis["w"])
    K = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n + 1, n + 1)).tocsr()[:n, :n]
    K.sum_duplicates()
    free = np.setdiff1d(np.arange(n), np.asarray(prescribed, dtype=np.int64))
    K_ff = K[free][:, free].tocsr()
    return K_ff, F[:n], free, np.concatenate(xs), np.concatenate(ws)


def assemble_plate(S, E, nu, t, prescribed, source_qp=None, chunk=1024):
    """(K_ff CSR, F on all DOFs, free DOFs) of the Kirchhoff plate
    (library.py:68-143: K_e = sum_q w B^T D B, B = -(R_xx, R_yy, 2 R_xy)) on the
    2D THB space ``S``, through the tensor oracle's second-derivative
    evaluation on the padded view; ``source_qp`` (n_e, n_q) is the load."""
    n = S.n_scalar
    rows, cols, vals = [], [], []
    F = np.zeros(n + 1)
    for lo in range(0, S.n_elems, chunk):
        el = np.arange(lo, min(lo + chunk, S.n_elems))
        basis = O.evaluate(S, el, order=2)
        Ke = O.element_tangents("plate", basis, {"E": E, "nu": nu, "t": t})
        gd = S.elem_dofs[el]
        rows.append(np.repeat(gd, gd.shape[1], axis=1).ravel())
        cols.append(np.tile(gd, (1, gd.shape[1])).ravel())
        vals.append(Ke.ravel())
        if source_qp is not None:
            Fe = np.einsum("eq,eq,eqi->ei", basis["w"], np.asarray(source_qp)[el], basis["R"])
            np.add.at(F, gd.ravel(), Fe.ravel())
    K = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n + 1, n + 1)).tocsr()[:n, :n]
    K.sum_duplicates()
    free = np.setdiff1d(np.arange(n), np.asarray(prescribed, dtype=np.int64))
    return K[free][:, free].tocsr(), F[:n], free, K


def assemble_elasticity(S, E, nu, prescribed, source_qp=None, chunk=512):
    """(K_ff CSR, F on all DOFs, free DOFs) of small-strain isotropic
    elasticity (library.py:174-181, plane stress in 2D) on the THB space ``S``
    with vec = dim; ``source_qp`` (n_e, n_q, dim). DOF c of function i is
    dim * i + c (function_space.py:300-312)."""
    vec = S.dim
    n = S.n_scalar * vec
    rows, cols, vals = [], [], []
    F = np.zeros(n + vec)
    for lo in range(0, S.n_elems, chunk):
        el = np.arange(lo, min(lo + chunk, S.n_elems))
        basis = O.evaluate(S, el)
        Ke = O.element_tangents("elasticity", basis, {"E": E, "nu": nu}, vec)
        gd = (vec * S.elem_dofs[el][..., None] + np.arange(vec)).reshape(len(el), -1)
        rows.append(np.repeat(gd, gd.shape[1], axis=1).ravel())
        cols.append(np.tile(gd, (1, gd.shape[1])).ravel())
        vals.append(Ke.ravel())
        if source_qp is not None:
            Fe = np.einsum("eq,eqc,eqi->eic", basis["w"], np.asarray(source_qp)[el], basis["R"]).reshape(len(el), -1)
            np.add.at(F, gd.ravel(), Fe.ravel())
    K = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n + vec, n + vec)).tocsr()[:n, :n]
    K.sum_duplicates()
    free = np.setdiff1d(np.arange(n), np.asarray(prescribed, dtype=np.int64))
    return K[free][:, free].tocsr(), F[:n], free, K


def neumann_load(S, vec, elems, sides, ref, wref, traction):
    """F_i,c = sum_q w t_c(x, n) R_i over boundary faces of the THB space ``S``
    (the negative gradient of neumann_work, src/jaxiga/methods/_common.py:312-318),
    the tensor oracle's boundary evaluation on the padded view; traction(x, n)
    -> (n_pts, vec); DOF c of function i is vec * i + c, the padding entry is
    dropped."""
    b = O.evaluate_boundary(S, elems, sides, ref, wref)
    nf, nq = b["w"].shape
    t = np.asarray(traction(b["x"].reshape(-1, S.dim), b["normal"].reshape(-1, S.dim)), dtype=float)
    Fe = np.einsum("fq,fqc,fqi->fic", b["w"], t.reshape(nf, nq, vec), b["R"])
    F = np.zeros((S.n_scalar + 1, vec))
    np.add.at(F, b["dofs"], Fe)
    return F[:-1].ravel()
