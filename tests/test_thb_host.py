"""Truncated hierarchical spaces on the host: the construction against the
reference's own (tests/golden/thb_golden.npz, made by make_thb_golden.py from
src/jaxiga/space/hierarchical.py), the oracle's assembled Poisson operator
against the reference's, and the properties the reference's tests check
(tests/test_hierarchical.py): partition of unity for THB and not for HB, the
geometry of the level-0 patch, admissibility bounding the local count, bulk
marking."""

import os

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200 import hierarchical as H
from oracle import iga_oracle as O
from oracle import thb_oracle as TO

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "thb_golden.npz"))
SQ = [[0, 0], [1, 0], [1, 1], [0, 1]]


def _deepen(V, rounds, **kw):
    for _ in range(rounds):
        V = H.refine_elements(V, [V.n_elems - 1, V.n_elems - 2, 0], **kw)
    return V


def _marked(V, marks, **kw):
    for mk in marks:
        V = H.refine_elements(V, mk, **kw)
    return V


CASES = {
    "sq_p2": lambda: _marked(jx.FunctionSpace(jx.primitives.quadrilateral(SQ).elevate(2).refine(2)), [[0, 1, 4]]),
    "sq_p3_deep": lambda: _deepen(jx.FunctionSpace(jx.primitives.quadrilateral(SQ).elevate(3).refine(2)), 3),
    "sq_p2_hb": lambda: _deepen(jx.FunctionSpace(jx.primitives.quadrilateral(SQ).elevate(2).refine(2)), 3,
                                truncate=False),
    "sq_p2_nonadm": lambda: _deepen(jx.FunctionSpace(jx.primitives.quadrilateral(SQ).elevate(2).refine(2)), 2,
                                    admissible=False),
    "annulus_p2": lambda: _marked(jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 2.0).elevate(2).refine(2)),
                                  [[5, 6], [1, 2, 3]]),
    "cube_p2": lambda: _marked(jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(2).refine(1)),
                               [[0, 1]]),
}


@pytest.mark.parametrize("tag", sorted(CASES))
def test_construction_matches_the_reference(tag):
    W = CASES[tag]()
    assert np.array_equal(W.elem_dofs, G[f"{tag}/elem_dofs"])
    assert np.array_equal(W.elem_key, G[f"{tag}/elem_key"])
    assert np.abs(W.extraction - G[f"{tag}/extraction"]).max() <= 1e-14
    assert np.abs(W.elem_vertex - G[f"{tag}/elem_vertex"]).max() == 0.0
    assert np.abs(W.cpts - G[f"{tag}/cpts"]).max() <= 1e-14
    assert np.abs(W.wgts - G[f"{tag}/wgts"]).max() <= 1e-14
    for lv, ref in enumerate(W.hierarchy.refined):
        assert np.array_equal(np.asarray(ref), G[f"{tag}/refined{lv}"])
    labels = sorted(k.split("/", 2)[2] for k in G.files if k.startswith(f"{tag}/bnd_dofs/"))
    assert sorted(W.boundaries) == labels
    for lbl in labels:
        assert np.array_equal(W.boundary(lbl).dofs, G[f"{tag}/bnd_dofs/{lbl}"])
        assert np.array_equal(W.boundary(lbl).elems, G[f"{tag}/bnd_elems/{lbl}"])


@pytest.mark.parametrize("tag", ["sq_p3_deep", "annulus_p2"])
def test_oracle_operator_matches_the_reference(tag):
    W = CASES[tag]()
    S = TO.ThbSpace.of(W)
    pres = G[f"{tag}/prescribed"]
    x = O.evaluate(S, np.arange(S.n_elems))["x"]
    assert np.abs(x - G[f"{tag}/gauss_x"]).max() <= 1e-13  # the level-0 geometry, as the reference's
    f = (8 * np.pi**2 * np.sin(2 * np.pi * x[..., 0]) * np.sin(2 * np.pi * x[..., 1]) if tag == "sq_p3_deep"
         else 1.0 + x[..., 0] * x[..., 1])
    K, F, free, _, w = TO.assemble_poisson(S, float(G[f"{tag}/a0"]), pres, source_qp=f)
    assert np.abs(w - G[f"{tag}/gauss_w"]).max() <= 1e-14
    Kv, ref = K @ G[f"{tag}/v"], G[f"{tag}/Kv"]
    assert np.abs(Kv - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.abs(K.diagonal() - G[f"{tag}/diag"]).max() <= 1e-12 * np.abs(G[f"{tag}/diag"]).max()
    assert np.abs(F - G[f"{tag}/load_F"]).max() <= 1e-12 * np.abs(G[f"{tag}/load_F"]).max()
    u = np.zeros(S.n_scalar)
    u[free] = O.scipy_superlu(K, F[free])
    assert np.linalg.norm(u - G[f"{tag}/u"]) <= 1e-10 * np.linalg.norm(G[f"{tag}/u"])
    assert K.nnz == int(G[f"{tag}/nnz"])


def test_thb_is_a_partition_of_unity_and_hb_is_not():
    for truncate, pou in ((True, True), (False, False)):
        W = _deepen(jx.FunctionSpace(jx.primitives.quadrilateral(SQ).elevate(2).refine(2)), 2, truncate=truncate)
        # the B-spline (not the rational) basis: sum_i N_i = sum_a (sum_i C_ia) B_a
        ref, _ = O.gauss_rule([3, 3])
        B = O.bernstein_tensor(ref, W.degree)[0]
        err = np.abs(np.einsum("ea,qa->eq", W.extraction.sum(1), B) - 1.0).max()
        assert (err <= 1e-13) if pou else (err > 1e-3), (truncate, err)


def test_empty_refinement_is_the_tensor_space():
    V = jx.FunctionSpace(jx.primitives.quadrilateral(SQ).elevate(3).refine(2))
    W = H.refine_elements(V, [])
    assert W.n_elems == V.n_elems and W.n_scalar_basis == V.n_scalar_basis and W.n_local_max == V.n_local
    assert np.array_equal(W.elem_dofs, V.elem_dofs)
    assert np.abs(W.extraction - V.extraction()).max() == 0.0


def test_admissibility_bounds_the_local_count():
    V = jx.FunctionSpace(jx.primitives.quadrilateral(SQ).elevate(2).refine(2))
    adm = _deepen(V, 3)
    assert adm.n_local_max <= 2 * V.n_local  # two levels of functions at most act on an element
    raw = _deepen(V, 3, admissible=False)
    assert raw.n_local_max >= adm.n_local_max


def test_refinement_argument_checks_and_bulk_marking():
    V = jx.FunctionSpace(jx.primitives.quadrilateral(SQ).elevate(2).refine(1))
    with pytest.raises(IndexError):
        H.refine_elements(V, [V.n_elems])
    eta = np.array([0.1, 3.0, 0.2, 2.0, 0.05])
    assert np.array_equal(H.dorfler_mark(eta, 0.5), [1])
    assert np.array_equal(H.dorfler_mark(eta, 0.9), [1, 3])
    assert H.dorfler_mark(np.zeros(4)).size == 0
    with pytest.raises(ValueError):
        H.dorfler_mark(eta, 0.0)


def test_gauss_point_values_and_gradients_match_the_oracle():
    """The host read-back of a field on a THB space (values and physical
    gradients at the Gauss points, used by errornorm and Solution.at) against
    the oracle's basis on the same padded view."""
    from jaxiga_b200.thb import ThbGeometry

    for tag in ("sq_p3_deep", "annulus_p2", "cube_p2"):
        W = CASES[tag]()
        S = TO.ThbSpace.of(W)
        b = O.evaluate(S, np.arange(W.n_elems))
        c = np.random.default_rng(2).standard_normal((W.n_scalar_basis, 2))
        cp = np.concatenate([c, np.zeros((1, 2))])[W.elem_dofs]  # (e, i, comp)
        g = ThbGeometry(W)
        val = g.interpolate(c).numpy()
        assert np.abs(val - np.einsum("eqi,eic->eqc", b["R"], cp)).max() <= 1e-12
        grad = g.interpolate_grad(c).numpy()
        ref = np.einsum("eqdi,eic->eqcd", b["dR"], cp)
        assert np.abs(grad - ref).max() <= 1e-11 * np.abs(ref).max()
        assert np.abs(g.qp_coords().numpy() - b["x"]).max() <= 1e-13


@pytest.mark.parametrize("tag", ["annulus_p2", "cube_p2", "sq_p3_deep"])
def test_boundary_points_match_the_oracle(tag):
    """Face points, outward normals and surface weights of every labelled side
    (host side data of the Neumann load) against the oracle's boundary
    evaluation on the padded view; side centres lie on the sides' points."""
    from jaxiga_b200.pointset import boundary_gauss
    from jaxiga_b200.thb import reference_tables, side_centres, side_points, tables_at

    W = CASES[tag]()
    S = TO.ThbSpace.of(W)
    u = np.polynomial.legendre.leggauss(W.degree[0] + 1)[0]
    grid = np.stack([g.ravel(order="F") for g in np.meshgrid(*([u] * W.dim), indexing="ij")], -1)
    assert np.array_equal(tables_at(grid, W.degree[0]), reference_tables(W.dim, W.degree[0])[0])
    for label in sorted(W.boundaries):
        ps = boundary_gauss(W, W.boundary(label))
        b = O.evaluate_boundary(S, ps.elems, ps.sides, ps.ref, ps.weights)
        for code in np.unique(ps.sides):
            sel = np.flatnonzero(ps.sides == code)
            x, n, w, _, _ = side_points(W, ps.elems[sel], code, ps.ref[sel[0]], ps.weights[sel[0]])
            assert np.abs(x - b["x"][sel]).max() < 1e-14
            assert np.abs(n - b["normal"][sel]).max() < 1e-13
            assert np.abs(w - b["w"][sel]).max() < 1e-14 * np.abs(b["w"]).max()
        c = side_centres(W, ps.elems, ps.sides)
        assert c.shape == (len(ps.elems), W.dim) and np.isfinite(c).all()


@pytest.mark.parametrize("tag", ["sq_p2", "sq_p3_deep", "annulus_p2"])
def test_plate_metric_reproduces_the_oracle_tangents(tag):
    """The Kirchhoff plate's per-point metric (the channels of the rational
    numerator mapped to the curvatures) contracted with the element's channel
    values gives the oracle's element tangents (library.py:68-143), on the
    rational annulus too."""
    from jaxiga_b200.thb import plate_point_data

    W = CASES[tag]()
    fac, _, X, w, T = plate_point_data(W, 2.0, 0.3, 0.1)
    iu = np.triu_indices(6)
    M = np.zeros(fac.shape[:2] + (6, 6))
    M[..., iu[0], iu[1]] = fac
    M[..., iu[1], iu[0]] = fac
    wl = np.concatenate([W.wgts, [0.0]])[W.elem_dofs]
    G = np.einsum("cqa,eia->eqci", T, W.extraction) * wl[:, None, None, :]
    Ke = np.einsum("eqci,eqcd,eqdj->eij", G, M, G)
    b = O.evaluate(TO.ThbSpace.of(W), np.arange(W.n_elems), order=2)
    Ko = O.element_tangents("plate", b, {"E": 2.0, "nu": 0.3, "t": 0.1})
    assert np.abs(Ke - Ko).max() <= 1e-12 * np.abs(Ko).max()
    assert np.abs(X - b["x"]).max() < 1e-14 and np.abs(w - b["w"]).max() < 1e-14 * np.abs(b["w"]).max()


def test_clamped_conditions_are_rejected_on_hierarchical_spaces():
    """A clamped side needs the second control-point layer of every level; the
    reference rejects it on hierarchical spaces (src/jaxiga/forms/problem.py:249-262)
    and so does this package, while the simply supported plate is accepted."""
    W = CASES["sq_p2"]()
    with pytest.raises(NotImplementedError):
        jx.KirchhoffPlate(W, dirichlet=[jx.ClampedBC(where=sorted(W.boundaries)[0])])
    jx.KirchhoffPlate(W, dirichlet=[jx.DirichletBC(0.0, where=sorted(W.boundaries)[0])])


@pytest.mark.parametrize("tag", ["annulus_p2", "cube_p2", "sq_p3_deep"])
def test_point_evaluation_matches_the_oracle(tag):
    """Values, physical gradients, coordinates and |det J| of a field at random
    points of random leaf elements (Solution.at / grad on any PointSet) against
    the oracle's evaluation on the padded view."""
    from jaxiga_b200.solve import Solution
    from jaxiga_b200.thb import ThbGeometry

    W = CASES[tag]()
    S = TO.ThbSpace.of(W)
    rng = np.random.default_rng(2)
    el, ref = rng.integers(0, W.n_elems, 40), rng.uniform(-1, 1, (40, W.dim))
    c = rng.standard_normal((W.n_scalar_basis, 2))
    out = ThbGeometry(W).eval_points(el, ref, c, val=True, grad=True, x=True, jac=True)
    cp = np.concatenate([c, np.zeros((1, 2))])
    b = [O.evaluate(S, [e], ref=r[None], weights=np.ones(1)) for e, r in zip(el, ref)]
    val = np.array([bk["R"][0, 0] @ cp[bk["dofs"][0]] for bk in b])
    grad = np.array([(bk["dR"][0, 0] @ cp[bk["dofs"][0]]).T for bk in b])
    assert np.abs(out["val"].numpy() - val).max() <= 1e-13 * np.abs(val).max()
    assert np.abs(out["grad"].numpy() - grad).max() <= 1e-12 * np.abs(grad).max()
    assert np.abs(out["x"].numpy() - np.array([bk["x"][0, 0] for bk in b])).max() < 1e-14
    assert np.abs(out["jac"].numpy() - np.array([bk["w"][0, 0] for bk in b])).max() < 1e-15
    ps = jx.gauss(W, 3)
    assert Solution(W, c[:, 0]).at(ps).shape == (W.n_elems, 3 ** W.dim, 1)
