"""Mixed-precision solves (FP32 iterations, FP64 corrections) through the libjxb C ABI.

Both schemes -- FP32 PCG with reliable FP64 updates (jxb_mixed_pcg) and FP64
iterative refinement around FP32 inner solves (jxb_refine_solve) -- must reach
an FP64 tolerance and give the reference's solution to the accuracy that FP64
CG gives at the same tolerance. The reliable-update iteration count is checked
against the oracle's restatement of the same scheme and against FP64 CG.
"""

import numpy as np
import pytest

import jaxiga_b200 as jx
from oracle import iga_oracle as O
from tests.cases import OPS, build, golden, with_fields
from tests.test_gpu_parity import device_interp, rel_l2

pytestmark = pytest.mark.gpu


def f32_operator(tag):
    V, problem, params = build(tag)
    params = with_fields(tag, V, params, device_interp(V))
    pres, vals = problem.resolve_dirichlet(params)
    mask = np.zeros(V.n_dofs, bool)
    mask[pres] = True
    coef, field = problem.operator_coefficients(params)
    coef_qp = None if field is None else np.asarray(field.values)
    op = jx.Operator(V, OPS[tag], coef, prescribed=mask, coef_qp=coef_qp, want_f32=True)
    return V, problem, params, op, pres, coef, field


@pytest.mark.parametrize("refinement", ["reliable", "restart"])
@pytest.mark.parametrize("tag", ["poisson2d", "annulus2d", "elast3d", "darcy3d", "plate2d"])
def test_mixed_solve_matches_reference(tag, refinement):
    g = golden()
    V, problem, params = build(tag)
    params = with_fields(tag, V, params, device_interp(V))
    plain = jx.solve(problem, params=params, linear=jx.LinearOptions(tol=1e-12))
    sol = jx.solve(problem, params=params,
                   linear=jx.LinearOptions(tol=1e-12, precision="mixed", refinement=refinement))
    assert sol.stats["converged"] and sol.stats["relative_residual"] <= 1e-12
    if tag == "plate2d":  # the plate's mixed form keeps the FP64 operator (FP32 cannot resolve it at size)
        assert sol.stats["fp32_operator"] is False and sol.stats["refinement"] is None
    else:
        assert sol.stats["refinement"] == refinement and sol.stats["outer"] >= 1
    # as close to the reference's solution as FP64 CG at the same tolerance
    err, err64 = rel_l2(sol.u, g[f"{tag}/u"]), rel_l2(plain.u, g[f"{tag}/u"])
    assert err < max(1e-9, 10 * err64), (err, err64)


@pytest.mark.parametrize("tag", ["annulus2d", "elast3d", "darcy3d"])
def test_reliable_update_iterations_match_oracle(tag):
    """Same scheme on the oracle's assembled matrix (FP32 CSR products): the
    FP32 rounding differs, so the counts agree to a few percent, not exactly."""
    g = golden()
    V, problem, params, op, pres, coef, field = f32_operator(tag)
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec)
    names = {"poisson": ("a0",), "elasticity": ("E", "nu"), "plate": ("E", "nu", "t")}[OPS[tag]]
    oparams = dict(zip(names, coef))
    if field is not None:
        oparams["a0_qp"] = np.asarray(field.values)
    A = O.Assembled(S, OPS[tag], oparams, pres, problem.resolve_dirichlet(params)[1], need_full=False)
    b = g[f"{tag}/rhs"]
    inv = O.jacobi_inverse(A.diag)
    K32 = A.K.astype(np.float32)
    x_o, k_o, u_o = O.reliable_cg(lambda v: A.K @ v, lambda v: K32 @ v, b, 1e-11, delta=1e-2, inv_diag=inv)
    _, k64 = O.jax_cg(lambda v: A.K @ v, b, 1e-11, inv_diag=inv)
    bf = np.zeros(V.n_dofs)
    bf[A.free] = b
    x, st = op.mixed_pcg(bf, tol=1e-11, delta=1e-2)
    assert st["converged"] and st["relative_residual"] <= 1e-11
    assert abs(st["iterations"] - k_o) <= 0.05 * k_o + 3, (st["iterations"], k_o)
    assert st["iterations"] <= 1.15 * k64 + 10, (st["iterations"], k64)
    assert abs(st["outer"] - u_o) <= 2, (st["outer"], u_o)
    assert rel_l2(x.cpu().numpy()[A.free], x_o) < 1e-8
    op.close()


def test_reliable_update_at_size_keeps_fp64_iteration_count():
    """3D elasticity, 16^3 cubic elements (15,000 DOFs): to 1e-8 the reliable-
    update solver needs about as many iterations as FP64 PCG, restarted
    refinement more, and all three solutions agree."""
    import torch

    from jaxiga_b200 import workloads

    V, problem, params = workloads.config2(n=16)
    pres, _ = problem.resolve_dirichlet(params)
    mask = np.zeros(V.n_dofs, bool)
    mask[pres] = True
    op = jx.Operator(V, "elasticity", (1.0, 0.3), prescribed=mask, want_f32=True)
    rng = np.random.default_rng(3)
    b = rng.standard_normal(V.n_dofs)
    x64, s64 = op.pcg(b, tol=1e-8, check_every=8)
    xr, sr = op.mixed_pcg(b, tol=1e-8, delta=1e-2, check_every=8)
    xf, sf = op.refine_solve(b, tol=1e-8, inner_tol=1e-3, check_every=8)
    for st in (s64, sr, sf):
        assert st["converged"] and st["relative_residual"] <= 1e-8
    assert sr["iterations"] <= 1.2 * s64["iterations"] + 16, (sr["iterations"], s64["iterations"])
    assert sr["iterations"] < sf["iterations"]
    for x in (xr, xf):
        assert float(torch.linalg.norm(x - x64) / torch.linalg.norm(x64)) < 1e-5
    op.close()


def test_mixed_solvers_with_a_zero_right_hand_side():
    """b = 0: no iteration runs, x = 0, and the stats report convergence, as for jxb_pcg."""
    V, problem, params, op, pres, coef, field = f32_operator("elast3d")
    b = np.zeros(V.n_dofs)
    for solve in (op.pcg, op.mixed_pcg, op.refine_solve):
        x, st = solve(b, tol=1e-10)
        assert st["iterations"] == 0 and st["converged"] and st["finite"], (solve.__name__, st)
        assert float(x.abs().max()) == 0.0
    op.close()
