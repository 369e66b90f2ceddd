"""Golden fixtures for truncated hierarchical (THB) spaces, from the reference.

Run where the reference sources are available, as for make_golden.py:

    python tests/golden/make_thb_golden.py <reference checkout>
    JAXIGA_REFERENCE=<reference checkout> python tests/golden/make_thb_golden.py

The reference's own ``refine_elements`` (src/jaxiga/space/hierarchical.py)
runs under the NumPy jax stand-in of ``_jax_stub.py`` on a few patches and
markings; per case it records the padded connectivity, extraction operators,
element boxes and keys, the control net, the hierarchy and the boundary DOF
sets. For two Poisson cases it also records, from the reference's element
tangents and CSR scatter (src/jaxiga/methods/galerkin.py), the free-DOF
operator's K.v for a seeded v, its diagonal, the load vector with the Dirichlet
lift and the SuperLU solution. Output: tests/golden/thb_golden.npz.
"""

from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _jax_stub  # noqa: E402
from make_golden import reference_src  # noqa: E402

SEED = 20260903
SQ = [[0, 0], [1, 0], [1, 1], [0, 1]]


def main():
    m = _jax_stub.load_reference(reference_src())
    H = importlib.import_module("jaxiga.space.hierarchical")
    prim, fs, lib, prob_mod = m["primitives"], m["function_space"], m["library"], m["problem"]
    common, gal, lin, P, ev = m["_common"], m["galerkin"], m["linear"], m["pointset"], m["evaluation"]
    out = {}
    rng = np.random.default_rng(SEED)

    def deepen(V, rounds, **kw):
        """Refine the last two and the first element of the current space, ``rounds`` times."""
        for _ in range(rounds):
            V = H.refine_elements(V, [V.n_elems - 1, V.n_elems - 2, 0], **kw)
        return V

    cases = {
        "sq_p2": (lambda: prim.quadrilateral(SQ).elevate(2).refine(2), [[0, 1, 4]], {}),
        "sq_p3_deep": (lambda: prim.quadrilateral(SQ).elevate(3).refine(2), 3, {}),
        "sq_p2_hb": (lambda: prim.quadrilateral(SQ).elevate(2).refine(2), 3, {"truncate": False}),
        "sq_p2_nonadm": (lambda: prim.quadrilateral(SQ).elevate(2).refine(2), 2, {"admissible": False}),
        "annulus_p2": (lambda: prim.quarter_annulus(1.0, 2.0).elevate(2).refine(2), [[5, 6], [1, 2, 3]], {}),
        "cube_p2": (lambda: prim.cuboid([0, 0, 0], [1, 1, 1]).elevate(2).refine(1), [[0, 1]], {}),
    }
    spaces = {}
    for tag, (make, marks, kw) in cases.items():
        patch = make()
        V = fs.FunctionSpace([patch])
        if isinstance(marks, int):
            W = deepen(V, marks, **kw)
        else:
            W = V
            for mk in marks:
                W = H.refine_elements(W, mk, **kw)
        spaces[tag] = W
        out[f"{tag}/marks"] = np.asarray(marks if isinstance(marks, int) else -1)
        for d, kv in enumerate(patch.knots):
            out[f"{tag}/knots{d}"] = np.asarray(kv)
        out[f"{tag}/degree"] = np.asarray(patch.degree)
        out[f"{tag}/cpts0"] = np.asarray(patch.ctrl_pts) if hasattr(patch, "ctrl_pts") else np.zeros(0)
        out[f"{tag}/elem_dofs"] = np.asarray(W.elem_dofs).astype(np.int64)
        out[f"{tag}/extraction"] = np.asarray(W.extraction)
        out[f"{tag}/elem_vertex"] = np.asarray(W.elem_vertex)
        out[f"{tag}/elem_key"] = np.asarray(W.elem_key).astype(np.int64)
        out[f"{tag}/cpts"] = np.asarray(W.cpts)
        out[f"{tag}/wgts"] = np.asarray(W.wgts)
        for lv, ref in enumerate(W.hierarchy.refined[0]):
            out[f"{tag}/refined{lv}"] = np.asarray(ref, dtype=np.int64)
        for label, bset in W.boundaries.items():
            out[f"{tag}/bnd_dofs/{label}"] = np.asarray(bset.dofs).astype(np.int64)
            out[f"{tag}/bnd_elems/{label}"] = np.asarray(bset.elems).astype(np.int64)

    # ---- Poisson on two THB spaces: the reference's assembled operator ----
    ALL = lambda x: np.full(x.shape[0], True)  # noqa: E731
    for tag, src in (("sq_p3_deep", lambda x: 8 * np.pi**2 * np.sin(2 * np.pi * x[0]) * np.sin(2 * np.pi * x[1])),
                     ("annulus_p2", lambda x: 1.0 + x[0] * x[1])):
        W = spaces[tag]
        a0 = 1.7
        problem = lib.Poisson(W, dirichlet=[prob_mod.DirichletBC(0.0, where=ALL)], source=lambda x, p: src(x))
        ctx = common.build_context(problem, {"a0": a0})
        basis = ctx.interior
        free = np.asarray(ctx.dofmap.free)
        prescribed = np.asarray(ctx.dofmap.prescribed)
        out[f"{tag}/prescribed"] = prescribed.astype(np.int64)
        blocks = [np.asarray(K) for _, K in gal.element_tangents(ctx, {"a0": a0})]
        Ke = np.concatenate(blocks, axis=0)
        pattern = ctx.assembly
        data = np.asarray(gal._assemble_csr_values(pattern, iter([Ke])))
        n = len(free)
        K_ff = sp.csr_matrix((data, pattern.column_indices, pattern.indptr), shape=(n, n))
        x = np.asarray(ev.evaluate(W, P.gauss(W)).x)
        f_qp = src(np.moveaxis(x, -1, 0))
        R, w = np.asarray(basis.R), np.asarray(basis.w)
        Fe = np.einsum("eq,eq,eqi->ei", w, f_qp, R)
        F = np.zeros(W.n_scalar_basis + 1)
        np.add.at(F, np.asarray(W.elem_dofs).ravel(), Fe.ravel())
        F = F[:-1]
        v = rng.standard_normal(n)
        b = F[free]
        u_free = np.asarray(lin._scipy_csr_solve(lin.LinearOptions(), pattern, data, b))
        out[f"{tag}/a0"] = np.asarray(a0)
        out[f"{tag}/gauss_x"] = x
        out[f"{tag}/gauss_w"] = w
        out[f"{tag}/load_F"] = F
        out[f"{tag}/v"] = v
        out[f"{tag}/Kv"] = K_ff @ v
        out[f"{tag}/diag"] = K_ff.diagonal()
        u = np.zeros(W.n_scalar_basis)
        u[free] = u_free
        out[f"{tag}/u"] = u
        out[f"{tag}/nnz"] = np.asarray(pattern.nnz)

    path = os.path.join(HERE, "thb_golden.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays")


if __name__ == "__main__":
    main()
