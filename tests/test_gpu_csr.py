"""Device Jacobi-PCG on assembled CSR matrices (the phase-field DeviceCG,
src/jaxiga/solvers/phase_field.py:305-390) against the jax-CG restatement on
the oracle's assembled operators, including the warm start across calls."""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
from cases import make_operator_oracle

import jaxiga_b200 as jx
from oracle import iga_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["poisson2d", "elast3d", "plate2d"])
def test_csr_pcg_matches_jax_cg_with_warm_start(tag):
    A = make_operator_oracle(tag)
    K = A.K.tocsr()
    K.sort_indices()
    pat = jx.CSRPattern.from_scipy(K)
    cg = jx.DeviceCG(pat, tol=1e-10, maxiter=20000)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(K.shape[0])
    assert np.abs(cg.matvec(K.data, x).cpu().numpy() - K @ x).max() < 1e-13 * np.abs(K @ x).max()
    b = rng.standard_normal(K.shape[0])
    inv = O.jacobi_inverse(K.diagonal())
    x1 = cg.solve(K.data, b).cpu().numpy()
    r1, k1 = O.jax_cg(lambda v: K @ v, b, 1e-10, inv_diag=inv)
    assert abs(cg.last_stats["iterations"] - k1) <= max(1, 0.02 * k1)
    assert np.linalg.norm(x1 - r1) < 1e-7 * np.linalg.norm(r1)
    # second sweep: new values and right-hand side, warm start from x1
    data2 = K.data * 1.1
    b2 = b + 0.01 * rng.standard_normal(K.shape[0])
    x2 = cg.solve(data2, b2).cpu().numpy()
    K2 = sp.csr_matrix((data2, K.indices, K.indptr), shape=K.shape)
    r2, k2 = O.jax_cg(lambda v: K2 @ v, b2, 1e-10, inv_diag=O.jacobi_inverse(K2.diagonal()), x0=x1)
    assert abs(cg.last_stats["iterations"] - k2) <= max(1, 0.02 * k2)
    assert np.linalg.norm(x2 - r2) < 1e-7 * np.linalg.norm(r2)
    assert cg.relative_residual(data2, b2, x2) <= 1e-10 * 1.01
    assert cg.calls == 2 and cg.failures == 0
    cg.release()


def test_csr_pcg_reports_a_truncated_solve():
    A = make_operator_oracle("elast3d")
    pat = jx.CSRPattern.from_scipy(A.K)
    cg = jx.DeviceCG(pat, tol=1e-12, maxiter=5)
    cg.solve(A.K.tocsr().data, np.ones(A.K.shape[0]))
    assert cg.failures == 1 and not cg.last_stats["converged"] and cg.last_stats["iterations"] == 5
    cg.release()
