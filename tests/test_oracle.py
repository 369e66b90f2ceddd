"""The oracle pinned against the reference's fixtures (CPU only).

tests/golden/golden.npz was produced by tests/golden/make_golden.py from the
reference's own setup, evaluation and element-kernel code. Connectivity and
extraction must match bit for bit; basis data, element tangents, assembled
operators and solutions to round-off (1e-12 relative or better).
"""

import numpy as np
import pytest

from oracle import iga_oracle as O
from tests.cases import golden

CASES = [("poisson2d", 1, "poisson"), ("patch2d", 1, "poisson"), ("annulus2d", 1, "poisson"),
         ("elast3d", 3, "elasticity"), ("darcy3d", 1, "poisson"), ("plate2d", 1, "plate")]


def space(tag, vec):
    g = golden()
    deg = g[tag + "/degree"]
    return O.Space([g[f"{tag}/knots{d}"] for d in range(len(deg))], deg, g[tag + "/cpts"], g[tag + "/wgts"], vec)


def params_and_source(tag, S):
    g = golden()
    if tag == "poisson2d":
        x = O.evaluate(S, np.arange(S.n_elems))["x"]
        return {"a0": 1.0}, 8 * np.pi**2 * np.sin(2 * np.pi * x[..., 0]) * np.sin(2 * np.pi * x[..., 1])
    if tag == "patch2d":
        return {"a0": 1.0}, np.zeros((S.n_elems, 9))
    if tag == "annulus2d":
        return {"a0": float(g["annulus2d/a0"])}, O.interpolate_qp(S, g["annulus2d/source_coef"])[..., 0]
    if tag == "elast3d":
        return {"E": 1.0, "nu": 0.3}, O.interpolate_qp(S, g["elast3d/eta"]) + np.array([0, 0, -1.0])
    if tag == "darcy3d":
        return {"a0_qp": np.exp(O.interpolate_qp(S, g["darcy3d/loga"])[..., 0])}, np.ones((S.n_elems, 64))
    return {"E": 12 * (1 - 0.09), "nu": 0.3, "t": 1.0}, np.ones((S.n_elems, 25))


def rel(a, b):
    return np.abs(np.asarray(a) - b).max() / np.abs(b).max()


@pytest.mark.parametrize("tag,vec,op", CASES)
def test_connectivity_and_extraction_are_bit_exact(tag, vec, op):
    g = golden()
    S = space(tag, vec)
    np.testing.assert_array_equal(S.elem_dofs, g[tag + "/elem_dofs"])
    np.testing.assert_array_equal(S.elem_vertex, g[tag + "/elem_vertex"])
    for d in range(S.dim):
        np.testing.assert_array_equal(S.ext1d[d], g[f"{tag}/extraction{d}"])
        np.testing.assert_array_equal(S.spans[d][2], g[f"{tag}/first{d}"])


@pytest.mark.parametrize("tag,vec,op", CASES)
def test_basis_and_element_tangents(tag, vec, op):
    g = golden()
    S = space(tag, vec)
    sample = g[tag + "/sample"]
    b = O.evaluate(S, sample, order=2 if op == "plate" else 1)
    for k in ("R", "dR", "x", "w") + (("d2R",) if op == "plate" else ()):
        assert rel(b[k], g[f"{tag}/basis_{k}"]) < 1e-12, k
    params, _ = params_and_source(tag, S)
    p = dict(params)
    if "a0_qp" in p:
        p["a0"] = p.pop("a0_qp")[sample]
    assert rel(O.element_tangents(op, b, p, vec), g[tag + "/Ke"]) < 1e-13


@pytest.mark.parametrize("tag,vec,op", CASES)
def test_assembly_rhs_and_solution(tag, vec, op):
    g = golden()
    S = space(tag, vec)
    params, f = params_and_source(tag, S)
    A = O.Assembled(S, op, params, g[tag + "/prescribed"], g[tag + "/prescribed_values"], source_qp=f)
    assert A.K.nnz == int(g[tag + "/nnz"])
    assert rel(A.b, g[tag + "/rhs"]) < 1e-13
    assert rel(A.diag, g[tag + "/diag"]) < 1e-13
    assert rel(A.K @ g[tag + "/v"], g[tag + "/Kv"]) < 1e-13
    u = A.lift(O.scipy_superlu(A.K, A.b))
    assert np.linalg.norm(u - g[tag + "/u"]) <= 1e-12 * np.linalg.norm(g[tag + "/u"])


def test_csr_pattern_checksum_matches_reference():
    import hashlib

    g = golden()
    S = space("poisson2d", 1)
    free = np.setdiff1d(np.arange(S.n_dofs), g["poisson2d/prescribed"])
    indptr, cols, rows, scatter = O.csr_pattern(S.elem_dofs, S.n_dofs, 1, free)
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()  # noqa: E731
    assert sha(indptr) + sha(cols) == str(g["poisson2d/csr_sha"])


@pytest.mark.parametrize("key", [k for k in golden().files if k.startswith("bezier/") and k.endswith("/C")])
def test_bezier_extraction_known_answers(key):
    g = golden()
    deg = int(key.split("/")[1].split("_")[0][1:])
    np.testing.assert_array_equal(np.stack(O.bezier_extraction(g[key[:-2] + "/knots"], deg)), g[key])


@pytest.mark.parametrize("deg", [1, 2, 3, 4, 5])
def test_bernstein_known_answers(deg):
    g = golden()
    u = np.linspace(-1, 1, 7)
    np.testing.assert_array_equal(O.bernstein_basis(u, deg), g[f"bernstein/p{deg}/B"])
    np.testing.assert_allclose(O.bernstein_basis_deriv(u, deg), g[f"bernstein/p{deg}/dB"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(O.bernstein_basis_2nd_deriv(u, deg), g[f"bernstein/p{deg}/d2B"], rtol=0, atol=1e-14)


def test_jax_cg_restatement_converges_like_scipy():
    g = golden()
    S = space("poisson2d", 1)
    params, f = params_and_source("poisson2d", S)
    A = O.Assembled(S, "poisson", params, g["poisson2d/prescribed"], g["poisson2d/prescribed_values"], source_qp=f)
    x, k = O.jax_cg(lambda v: A.K @ v, A.b, 1e-12, inv_diag=O.jacobi_inverse(A.diag))
    assert 0 < k < 10 * len(A.b)
    d = O.linear_diagnostics(lambda v: A.K @ v, x, A.b, 1e-10)
    assert d["converged"] and d["finite"]
    u = A.lift(x)
    assert np.linalg.norm(u - g["poisson2d/u"]) <= 1e-9 * np.linalg.norm(g["poisson2d/u"])
    xs, used = O.scipy_cg(A.K, A.b, 1e-12)
    assert np.linalg.norm(A.lift(xs) - g["poisson2d/u"]) <= 1e-9 * np.linalg.norm(g["poisson2d/u"])


def test_truncated_cg_reports_non_convergence():
    """tests/test_solver_robustness.py:85-93 of the reference, on the oracle."""
    g = golden()
    S = space("poisson2d", 1)
    params, f = params_and_source("poisson2d", S)
    A = O.Assembled(S, "poisson", params, g["poisson2d/prescribed"], g["poisson2d/prescribed_values"], source_qp=f)
    x, k = O.jax_cg(lambda v: A.K @ v, A.b, 1e-12, maxiter=3, inv_diag=O.jacobi_inverse(A.diag))
    assert k == 3
    assert not O.linear_diagnostics(lambda v: A.K @ v, x, A.b, 1e-12)["converged"]


@pytest.mark.parametrize("tag,vec,op", [("elast3d", 3, "elasticity"), ("darcy3d", 1, "poisson"),
                                        ("annulus2d", 1, "poisson")])
def test_reliable_update_cg_keeps_the_fp64_iteration_count(tag, vec, op):
    """FP32 iterations with FP64 reliable updates reach an FP64 tolerance in about
    as many iterations as FP64 CG (the Krylov recurrence is kept across updates).
    The cases take 50-250 FP64 iterations; on a system so small that FP64 CG ends
    by finite termination (the 64-DOF plate: 10 iterations) FP32 rounding loses
    that and the comparison says nothing."""
    g = golden()
    S = space(tag, vec)
    params, f = params_and_source(tag, S)
    A = O.Assembled(S, op, params, g[tag + "/prescribed"], g[tag + "/prescribed_values"], source_qp=f)
    inv = O.jacobi_inverse(A.diag)
    K32 = A.K.astype(np.float32)
    x64, k64 = O.jax_cg(lambda v: A.K @ v, A.b, 1e-11, inv_diag=inv)
    x, k, updates = O.reliable_cg(lambda v: A.K @ v, lambda v: K32 @ v, A.b, 1e-11, delta=1e-2, inv_diag=inv)
    assert np.linalg.norm(A.b - A.K @ x) <= 1e-11 * np.linalg.norm(A.b)
    assert updates >= 5  # one per two decades at least
    assert k <= 1.15 * k64 + 10, (k, k64)
    assert np.linalg.norm(A.lift(x) - g[tag + "/u"]) <= 1e-7 * np.linalg.norm(g[tag + "/u"])


@pytest.mark.parametrize("fine", [(7, 6, 5), (8, 9, 3), (1, 2, 3)])
def test_cnn_oracle_trilinear_upsampling(fine):
    """The pooled network's output interpolation: rows of each 1D prolongation sum
    to one, a constant stays constant, and the gradient map is its adjoint."""
    from oracle import cnn_oracle as C

    coarse = C.half(fine)
    for nf, nc in zip(fine, coarse):
        P = C.lin_matrix(nf, nc)
        np.testing.assert_allclose(P.sum(axis=1), 1.0)
        assert all(P[X, X // 2] == 1.0 for X in range(0, nf, 2))  # even fine points copy their coarse point
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2,) + coarse)
    g = rng.standard_normal((2,) + fine)
    assert abs((C.up_lin(x, fine) * g).sum() - (x * C.up_lin_grad(g, coarse)).sum()) < 1e-12
    np.testing.assert_allclose(C.up_lin(np.full((1,) + coarse, 3.0), fine), 3.0)


def test_cnn_oracle_pooled_forward_is_the_coarse_network_interpolated():
    from oracle import cnn_oracle as C

    rng = np.random.default_rng(1)
    ch = (4, 8)
    n = sum(ci * co * k ** 3 + co for ci, co, k, _ in C.layer_shapes(2, ch))
    p = rng.uniform(-0.3, 0.3, n)
    x = rng.standard_normal((2, 7, 6, 5))
    out, _ = C.forward(p, x, 2, ch, pool_input=True)
    coarse, _ = C.forward(p, C.pool(x), 2, ch)
    np.testing.assert_allclose(out, C.up_lin(coarse, x.shape[1:]))
    g = rng.standard_normal((1, 7, 6, 5))
    np.testing.assert_allclose(C.backward(p, x, g, 2, ch, pool_input=True),
                               C.backward(p, C.pool(x), C.up_lin_grad(g, C.half(x.shape[1:])), 2, ch))


def test_boundary_measures_and_normals_of_the_annulus():
    """Boundary Gauss sets of the quarter annulus (radii 1 and 4, cubic, refined
    three times): side lengths 2 pi, pi/2, 3, 3 to 1e-12 and radial outward
    normals, the known answers of the reference's tests/test_evaluation.py:47-70."""
    import jaxiga_b200 as jx
    from jaxiga_b200.pointset import boundary_gauss

    V = jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 4.0).elevate(3).refine(3))
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 1)
    exact = {"outer": 2 * np.pi, "inner": np.pi / 2, "sym_y": 3.0, "sym_x": 3.0}
    for label, length in exact.items():
        ps = boundary_gauss(V, V.boundary(label))
        b = O.evaluate_boundary(S, ps.elems, ps.sides, ps.ref, ps.weights)
        assert abs(b["w"].sum() - length) < 1e-12 * length, label
        assert np.abs(np.linalg.norm(b["normal"], axis=-1) - 1.0).max() < 1e-13
        if label in ("outer", "inner"):
            r = np.linalg.norm(b["x"], axis=-1)[..., None]
            sign = 1.0 if label == "outer" else -1.0
            assert np.abs(b["normal"] - sign * b["x"] / r).max() < 1e-12


def test_neumann_load_of_a_constant_flux_sums_to_the_side_length():
    import jaxiga_b200 as jx
    from jaxiga_b200.pointset import boundary_gauss

    V = jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 4.0).elevate(3).refine(3))
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 1)
    ps = boundary_gauss(V, V.boundary("outer"))
    F = O.neumann_load(S, ps.elems, ps.sides, ps.ref, ps.weights, lambda x, n: np.ones((len(x), 1)))
    assert abs(F.sum() - 2 * np.pi) < 1e-12 * 2 * np.pi  # partition of unity: sum_i int R_i = arc length
