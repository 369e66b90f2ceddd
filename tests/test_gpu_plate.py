"""The clamped Kirchhoff plate (biharmonic, quartic, condition number ~h^-4)
solved to a true relative residual of 1e-8 in every form.

Plain FP64 Jacobi-PCG needs the true-residual restarts (the correction solves
of the reference's CPU CG, src/jaxiga/solvers/linear.py:261-321): at 256^2
CG's recursive residual meets 1e-8 while b - K u is still 1.09e-8. The mixed
form keeps the FP64 operator (its FP32 counterpart cannot resolve the plate)
and the learned form runs flexible CG with the committed plate network.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200 import workloads

pytestmark = pytest.mark.gpu

CKPT = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "jaxiga_b200", "checkpoints")
TOL = 1e-8


def _check(sol, ref=None):
    st = sol.stats
    assert st["finite"] and st["converged"], st
    assert st["relative_residual"] <= TOL, st
    if ref is not None:
        # both solutions have true residuals below TOL ||b||: their difference
        # is what K^-1 makes of a residual of at most 2 TOL ||b||
        d = np.linalg.norm(sol.u - ref.u) / np.linalg.norm(ref.u)
        assert d < 1e-5, d


@pytest.mark.parametrize("n", [128, 256])
def test_plate_plain_fp64_reaches_true_tolerance(n):
    V, problem, params = workloads.config5(n=n)
    sol = jx.solve(problem, params=params, linear=jx.LinearOptions(tol=TOL, maxiter=40000))
    _check(sol)


def test_plate_128_mixed_and_learned_reach_true_tolerance():
    V, problem, params = workloads.config5(n=128)
    plain = jx.solve(problem, params=params, linear=jx.LinearOptions(tol=TOL, maxiter=40000))
    _check(plain)
    mixed = jx.solve(problem, params=params, linear=jx.LinearOptions(tol=TOL, maxiter=40000, precision="mixed"))
    assert mixed.stats["fp32_operator"] is False
    _check(mixed, plain)
    ckpt = os.path.join(CKPT, "plate128.npz")
    for precision in ("fp64", "mixed"):
        learned = jx.solve(problem, params=params,
                           linear=jx.LinearOptions(tol=TOL, maxiter=40000, precision=precision,
                                                   preconditioner="learned", checkpoint=ckpt))
        _check(learned, plain)
        assert learned.stats["outer"] > 0  # iterations that used the network
