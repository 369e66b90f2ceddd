"""Generate golden fixtures from the reference JAXIGA code.

Run where the reference sources are available (read-only is enough), giving
the reference checkout's root as an argument or in ``JAXIGA_REFERENCE``:

    python tests/golden/make_golden.py <reference checkout>
    JAXIGA_REFERENCE=<reference checkout> python tests/golden/make_golden.py

jax/jaxlib are not installed there, so the reference's setup stage and its
basis evaluation / element kernels run under the NumPy stand-in in
``_jax_stub.py`` (loops in place of ``vmap``). What is recorded, per case:

* geometry after the reference's ``elevate``/``refine``/``insert_knots``
  (knots, control points, weights);
* per-direction Bezier extraction operators (``space/bernstein.py``);
* connectivity ``elem_dofs`` and element boxes (``space/function_space.py``);
* the prescribed/free DOF partition (``forms/problem.py``);
* ``BasisData`` (R, dR, d2R, x, w) and element tangents K_e for a sample of
  elements (``space/evaluation.py``, ``forms/library.py``);
* the CSR pattern's size and checksum (``methods/_common.py``);
* the right-hand side, Jacobi diagonal and K.v for a seeded v, assembled
  from the reference's own element tangents through its CSR scatter
  (``methods/galerkin.py:_assemble_csr_values``);
* the solution from the reference's SuperLU host solve
  (``solvers/linear.py:_scipy_csr_solve``).

The right-hand side b = F_f - K_fp g is formed here from the reference's
basis data because the reference obtains it by reverse-mode AD of the
energy (``methods/galerkin.py:rhs``), which the stub cannot run.
"""

from __future__ import annotations

import hashlib
import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _jax_stub  # noqa: E402

SEED = 20260901


def reference_src(argv=None):
    """``src`` directory of the reference checkout named on the command line
    or by ``JAXIGA_REFERENCE``."""
    argv = sys.argv[1:] if argv is None else argv
    root = argv[0] if argv else os.environ.get("JAXIGA_REFERENCE")
    if not root:
        raise SystemExit("usage: make_golden.py <reference checkout> (or set JAXIGA_REFERENCE)")
    src = os.path.join(root, "src")
    if not os.path.isdir(os.path.join(src, "jaxiga")):
        raise SystemExit(f"{src} holds no jaxiga package")
    return src


def sha(a):
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.tobytes()).hexdigest()


def main():
    m = _jax_stub.load_reference(reference_src())
    prim, fs, P, ev = m["primitives"], m["function_space"], m["pointset"], m["evaluation"]
    prob_mod, lib, lin, common, gal = m["problem"], m["library"], m["linear"], m["_common"], m["galerkin"]
    bern = m["bernstein"]
    PointField = common.PointField
    out = {}

    def record_space(tag, V, patch):
        out[f"{tag}/degree"] = np.asarray(patch.degree)
        for d, kv in enumerate(patch.knots):
            out[f"{tag}/knots{d}"] = np.asarray(kv)
            C, nb = bern.bezier_extraction(np.asarray(kv), patch.degree[d])
            out[f"{tag}/extraction{d}"] = np.stack(C[:nb])
            lo, hi, first = bern.element_spans(np.asarray(kv), patch.degree[d])
            out[f"{tag}/first{d}"] = first
        out[f"{tag}/cpts"] = np.asarray(V.cpts)
        out[f"{tag}/wgts"] = np.asarray(V.wgts)
        out[f"{tag}/elem_dofs"] = np.asarray(V.elem_dofs).astype(np.int32)
        out[f"{tag}/elem_vertex"] = np.asarray(V.elem_vertex)

    def solve_case(tag, problem, params, source_qp, sample, rng, order=1):
        """Everything downstream of the space, from the reference's code."""
        V = problem.space
        vec = V.vec
        ctx = common.build_context(problem, params)
        basis = ctx.interior
        prescribed = np.asarray(ctx.dofmap.prescribed)
        values = np.asarray(ctx.dofmap.values, dtype=float)
        free = np.asarray(ctx.dofmap.free)
        out[f"{tag}/prescribed"] = prescribed.astype(np.int64)
        out[f"{tag}/prescribed_values"] = values
        gp = P.gauss(V, problem.quadrature)
        out[f"{tag}/gauss_ref"] = np.asarray(gp.ref)
        out[f"{tag}/gauss_w"] = np.asarray(gp.weights)

        for name in ("R", "dR", "d2R", "x", "w"):
            arr = getattr(basis, name)
            if arr is not None:
                out[f"{tag}/basis_{name}"] = np.asarray(arr)[sample]
        out[f"{tag}/sample"] = np.asarray(sample)
        out[f"{tag}/wsum"] = np.asarray(np.sum(basis.w))

        blocks = [np.asarray(K) for _, K in gal.element_tangents(ctx, params)]
        Ke = np.concatenate(blocks, axis=0)
        out[f"{tag}/Ke"] = Ke[sample]

        pattern = ctx.assembly
        data = np.asarray(gal._assemble_csr_values(pattern, iter([Ke])))
        out[f"{tag}/nnz"] = np.asarray(pattern.nnz)
        out[f"{tag}/csr_sha"] = np.asarray(sha(pattern.indptr) + sha(pattern.column_indices))
        n = len(free)
        K_ff = sp.csr_matrix((data, pattern.column_indices, pattern.indptr), shape=(n, n))

        # full K (prescribed rows/columns included) for the Dirichlet lift term
        gd = fs.expand_dofs(np.asarray(V.elem_dofs), vec)
        rows = np.repeat(gd, gd.shape[1], axis=1).ravel()
        cols = np.tile(gd, (1, gd.shape[1])).ravel()
        K_full = sp.coo_matrix((Ke.ravel(), (rows, cols)), shape=(V.n_dofs, V.n_dofs)).tocsr()

        # load vector F_i,c = sum_q w f_c R_i  (element_energy's source work)
        R = np.asarray(basis.R)
        w = np.asarray(basis.w)
        fq = np.asarray(source_qp).reshape(R.shape[0], R.shape[1], vec)
        Fe = np.einsum("eq,eqc,eqi->eic", w, fq, R).reshape(R.shape[0], -1)
        F = np.zeros(V.n_dofs)
        np.add.at(F, gd.ravel(), Fe.ravel())
        g = np.zeros(V.n_dofs)
        g[prescribed] = values
        b = (F - K_full @ g)[free]
        out[f"{tag}/load_F"] = F
        out[f"{tag}/rhs"] = b
        out[f"{tag}/diag"] = K_ff.diagonal()
        v = rng.standard_normal(n)
        out[f"{tag}/v"] = v
        out[f"{tag}/Kv"] = K_ff @ v

        opts = lin.LinearOptions()
        u_free = np.asarray(lin._scipy_csr_solve(opts, pattern, data, b))
        u = np.zeros(V.n_dofs)
        u[free] = u_free
        u[prescribed] = values
        out[f"{tag}/u"] = u
        out[f"{tag}/true_residual"] = np.asarray(np.linalg.norm(K_ff @ u_free - b))
        # energy norm of the discrete solution, u_f^T K_ff u_f
        out[f"{tag}/energy"] = np.asarray(u_free @ (K_ff @ u_free))
        return ctx, basis, u

    rng = np.random.default_rng(SEED)

    # ---- 1. 2D Poisson, unit square, cubic, 32x32 spans (1225 DOFs) ----
    tag = "poisson2d"
    patch = prim.quadrilateral([[0, 0], [1, 0], [1, 1], [0, 1]]).elevate(3).refine(5)
    V = fs.FunctionSpace(patch)
    record_space(tag, V, patch)
    ALL = lambda x: np.full(x.shape[0], True)  # noqa: E731
    problem = lib.Poisson(V, dirichlet=[prob_mod.DirichletBC(0.0, where=ALL)],
                          source=lambda x, p: 8 * np.pi**2 * np.sin(2 * np.pi * x[0]) * np.sin(2 * np.pi * x[1]))
    basis_x = np.asarray(ev.evaluate(V, P.gauss(V)).x)
    f_qp = 8 * np.pi**2 * np.sin(2 * np.pi * basis_x[..., 0]) * np.sin(2 * np.pi * basis_x[..., 1])
    ctx, basis, u = solve_case(tag, problem, {"a0": 1.0}, f_qp, [0, 1, 33, 500, 1023], rng)
    dofs = np.asarray(V.elem_dofs)
    uh = np.einsum("eqn,en->eq", np.asarray(basis.R), u[dofs])
    ex = np.sin(2 * np.pi * basis_x[..., 0]) * np.sin(2 * np.pi * basis_x[..., 1])
    w = np.asarray(basis.w)
    out[f"{tag}/errornorm_L2"] = np.asarray(np.sqrt(np.sum(w * (uh - ex) ** 2) / np.sum(w * ex**2)))

    # ---- 2. patch test: inhomogeneous linear Dirichlet data, no source ----
    tag = "patch2d"
    patch = prim.quadrilateral([[0, 0], [1, 0], [1, 1], [0, 1]]).elevate(2).refine(2)
    V = fs.FunctionSpace(patch)
    record_space(tag, V, patch)
    problem = lib.Poisson(V, dirichlet=[prob_mod.DirichletBC(lambda x, p: 1.0 + 2.0 * x[0] - 3.0 * x[1], where=ALL)],
                          source=lambda x, p: 0.0)
    nq = 9
    solve_case(tag, problem, {"a0": 1.0}, np.zeros((V.n_elems, nq)), [0, 5, 15], rng)

    # ---- 3. rational quarter annulus, cubic, 8x8 spans, lognormal a0, random source ----
    tag = "annulus2d"
    base = prim.quarter_annulus(1.0, 2.0).elevate(3)
    kn = np.linspace(0, 1, 9)[1:-1]
    patch = base.insert_knots(kn, kn)
    V = fs.FunctionSpace(patch)
    record_space(tag, V, patch)
    a0 = float(rng.lognormal(0.0, 0.5))
    coef = rng.standard_normal(V.n_scalar_basis)
    bset = [prob_mod.DirichletBC(0.0, where=lbl) for lbl in ("inner", "outer", "sym_y", "sym_x")]
    problem = lib.Poisson(V, dirichlet=bset, source=lambda x, p: 0.0)
    Rb = np.asarray(ev.evaluate(V, P.gauss(V)).R)
    f_qp = np.einsum("eqn,en->eq", Rb, coef[np.asarray(V.elem_dofs)])
    out[f"{tag}/a0"] = np.asarray(a0)
    out[f"{tag}/source_coef"] = coef
    solve_case(tag, problem, {"a0": a0}, f_qp, [0, 9, 63], rng)

    # geometry-only fixtures for the batched annulus family (degrees 2..4)
    for p in (2, 3, 4):
        g = prim.quarter_annulus(1.0, 2.0).elevate(p).insert_knots(np.linspace(0, 1, 6)[1:-1], np.linspace(0, 1, 4)[1:-1])
        out[f"annulus_p{p}/cpts"] = np.asarray(g.ctrl_pts)
        out[f"annulus_p{p}/wgts"] = np.asarray(g.weights)
        for d in range(2):
            out[f"annulus_p{p}/knots{d}"] = np.asarray(g.knots[d])

    # ---- 4. 3D linear elasticity, unit cube, cubic, 4^3 spans, x=0 clamped ----
    tag = "elast3d"
    kn = np.linspace(0, 1, 5)[1:-1]
    patch = prim.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kn)
    V = fs.FunctionSpace(patch, vec=3)
    record_space(tag, V, patch)
    eta = rng.normal(0.0, 0.1, size=(V.n_scalar_basis, 3))
    Rb = np.asarray(ev.evaluate(V, P.gauss(V)).R)
    f_qp = np.einsum("eqn,enc->eqc", Rb, eta[np.asarray(V.elem_dofs)]) + np.array([0.0, 0.0, -1.0])
    out[f"{tag}/eta"] = eta
    problem = lib.LinearElasticity(V, dirichlet=[prob_mod.DirichletBC([0.0, 0.0, 0.0], where="left")],
                                   source=lambda x, p: 0.0)
    solve_case(tag, problem, {"E": 1.0, "nu": 0.3}, f_qp, [0, 21, 63], rng)

    # ---- 5. 3D Darcy with a per-point log-normal permeability, 5^3 spans ----
    tag = "darcy3d"
    kn = np.linspace(0, 1, 6)[1:-1]
    patch = prim.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kn)
    V = fs.FunctionSpace(patch)
    record_space(tag, V, patch)
    loga = rng.standard_normal(V.n_scalar_basis)
    Rb = np.asarray(ev.evaluate(V, P.gauss(V)).R)
    a_qp = np.exp(np.einsum("eqn,en->eq", Rb, loga[np.asarray(V.elem_dofs)]))
    out[f"{tag}/loga"] = loga
    problem = lib.Poisson(V, dirichlet=[prob_mod.DirichletBC(0.0, where=ALL)], source=lambda x, p: 1.0)
    solve_case(tag, problem, {"a0": PointField(a_qp)}, np.ones(a_qp.shape), [0, 62, 124], rng)

    # ---- 6. clamped Kirchhoff plate, quartic, 8x8 spans, D = 1 ----
    tag = "plate2d"
    kn = np.linspace(0, 1, 9)[1:-1]
    patch = prim.rectangle(0, 0, 1, 1).elevate(4).insert_knots(kn, kn)
    V = fs.FunctionSpace(patch)
    record_space(tag, V, patch)
    problem = lib.KirchhoffPlate(V, dirichlet=[prob_mod.ClampedBC(where=s) for s in ("left", "right", "bottom", "top")],
                                 source=lambda x, p: 1.0)
    nq = 25
    solve_case(tag, problem, {"E": 12 * (1 - 0.3**2), "nu": 0.3, "t": 1.0}, np.ones((V.n_elems, nq)), [0, 27, 63], rng, order=2)

    # ---- 7. Bezier extraction / Bernstein known answers ----
    for deg in (1, 2, 3, 4, 5):
        for n_elem in (1, 2, 5):
            for rep in (0, 1):
                if rep >= deg:
                    continue
                interior = np.repeat(np.linspace(0, 1, n_elem + 1)[1:-1], 1 + rep)
                kv = np.concatenate([np.zeros(deg + 1), interior, np.ones(deg + 1)])
                C, nb = bern.bezier_extraction(kv, deg)
                out[f"bezier/p{deg}_n{n_elem}_r{rep}/knots"] = kv
                out[f"bezier/p{deg}_n{n_elem}_r{rep}/C"] = np.stack(C[:nb])
        pts = np.linspace(-1, 1, 7)
        out[f"bernstein/p{deg}/B"] = bern.bernstein_basis(pts, deg)
        out[f"bernstein/p{deg}/dB"] = bern.bernstein_basis_deriv(pts, deg)
        out[f"bernstein/p{deg}/d2B"] = bern.bernstein_basis_2nd_deriv(pts, deg)

    # ---- 8. connectivity at 16^3 (cubic, vec=3) by checksum ----
    kn = np.linspace(0, 1, 17)[1:-1]
    patch = prim.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kn)
    V = fs.FunctionSpace(patch, vec=3)
    out["cube16/elem_dofs_sha"] = np.asarray(sha(np.asarray(V.elem_dofs).astype(np.int64)))
    out["cube16/elem_vertex_sha"] = np.asarray(sha(np.asarray(V.elem_vertex, dtype=np.float64)))
    out["cube16/ops_sample"] = np.asarray(V.extraction)[[0, 17, 4095]]
    left = prob_mod.Problem(V, dirichlet=[prob_mod.DirichletBC([0.0, 0.0, 0.0], where="left")])
    out["cube16/prescribed_sha"] = np.asarray(sha(np.asarray(left.resolve_dirichlet()[0], dtype=np.int64)))

    # full-size per-direction extraction for the 3D and plate workloads
    for tag, p, n in (("ext_c2", 3, 64), ("ext_c4", 3, 96), ("ext_c5", 4, 256)):
        kv = np.concatenate([np.zeros(p + 1), np.linspace(0, 1, n + 1)[1:-1], np.ones(p + 1)])
        C, nb = bern.bezier_extraction(kv, p)
        out[f"{tag}/C"] = np.stack(C[:nb])

    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path) / 1e6:.2f} MB")


if __name__ == "__main__":
    main()
