"""BiCGSTAB on the device (the reference's method="bicgstab") against its oracle
restatement on the assembled operators, and the backends-agree check of the
reference's tests/test_galerkin.py:71-79 (CG and BiCGSTAB give one solution)."""

from __future__ import annotations

import numpy as np
import pytest
from cases import build, golden, make_operator_oracle

import jaxiga_b200 as jx
from oracle import iga_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["poisson2d", "elast3d", "plate2d"])
def test_bicgstab_matches_oracle(tag):
    from test_gpu_parity import make_operator

    g = golden()
    V, problem, params, op, pres, vals = make_operator(tag)
    A = make_operator_oracle(tag)
    b = g[f"{tag}/rhs"]
    bf = np.zeros(V.n_dofs)
    bf[A.free] = b
    x, st = op.bicgstab(bf, tol=1e-10)
    x_o, k_o = O.bicgstab(lambda v: A.K @ v, b, 1e-10, inv_diag=O.jacobi_inverse(A.diag))
    assert st["converged"] and st["relative_residual"] <= 1.01e-10
    # BiCGSTAB's residual history is erratic, so its iteration count moves more
    # with the summation order of K.v (matrix-free bricks against a CSR product)
    # than CG's does
    assert abs(st["iterations"] - k_o) <= max(2, 0.15 * k_o), (st["iterations"], k_o)
    assert np.linalg.norm(x.cpu().numpy()[A.free] - x_o) < 1e-7 * np.linalg.norm(x_o)
    op.close()


def test_backends_agree():
    """tests/test_galerkin.py:71-79: every LinearOptions method gives one solution
    (the direct ones and GMRES run the device CG, the operators being SPD)."""
    V, problem, params = build("poisson2d")
    a = jx.solve(problem, params=params, linear=jx.LinearOptions(method="cg", tol=1e-12))
    assert a.stats["converged"]
    for m in ("bicgstab", "scipy", "dense", "gmres"):
        b = jx.solve(problem, params=params, linear=jx.LinearOptions(method=m, tol=1e-12))
        assert b.stats["converged"] and b.stats["requested_method"] == m
        assert np.linalg.norm(a.u - b.u) <= 1e-7 * np.linalg.norm(a.u)
