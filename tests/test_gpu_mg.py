"""The multigrid V-cycle on the device against its oracle restatement
(oracle/mg_oracle.py, built on the oracle's assembled operators), its symmetry,
and multigrid-preconditioned CG against plain Jacobi-PCG."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import jaxiga_b200 as jx
from jaxiga_b200 import workloads
from jaxiga_b200.multigrid import Multigrid
from jaxiga_b200.solve import geometry_operator
from oracle import iga_oracle as O
from oracle import mg_oracle as MO

pytestmark = pytest.mark.gpu


def _case(which):
    if which == "plate":
        V, pr, params = workloads.config5(n=32)
        return pr, dict(params), "plate", dict(params)
    if which == "annulus":
        V = jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 4.0).elevate(3).refine(4), vec=2)
        pr = jx.LinearElasticity(V, dirichlet=[jx.DirichletBC(0.0, where="sym_y", component=1),
                                               jx.DirichletBC(0.0, where="sym_x", component=0)])
        return pr, {"E": 2.0, "nu": 0.3}, "elasticity", {"E": 2.0, "nu": 0.3}
    if which == "elasticity":
        V, pr, params = workloads.config2(n=8)
        return pr, {"E": 1.0, "nu": 0.3}, "elasticity", {"E": 1.0, "nu": 0.3}
    V, pr, params = workloads.config4(n=8)
    a = np.exp(geometry_operator(V).interpolate(params["loga"])[..., 0].cpu().numpy())
    return pr, {"a0": jx.PointField(a)}, "poisson", None


@pytest.mark.parametrize("which", ["plate", "annulus", "elasticity", "darcy"])
def test_vcycle_matches_oracle(which):
    pr, params, op, oparams = _case(which)
    mg = Multigrid(pr, params, degree=3, smooth_range=20.0, max_coarse=200)
    assert mg.levels >= 3 and all(mg.exact)
    levels = []
    for l, (S, m) in enumerate(zip(mg.spaces, mg.masks)):
        p = dict(oparams) if oparams is not None else {"a0_qp": mg.coefs[l].reshape(S.n_elems, -1)}
        levels.append((O.Space(S.knots, S.degree, S.cpts, S.wgts, S.vec), op, p, np.nonzero(m)[0]))
    V = MO.VCycle(levels, mg.transfers, mg.lmax, 3, 20.0)
    rng = np.random.default_rng(2)
    free = ~mg.masks[0]
    for _ in range(2):
        r = rng.standard_normal(len(free)) * free
        z = mg.vcycle(r).cpu().numpy()
        zo = V(r[free])
        assert np.abs(z[free] - zo).max() < 1e-11 * np.abs(zo).max()
        assert np.all(z[~free] == 0)
    mg.close()


def test_vcycle_is_symmetric():
    pr, params, _, _ = _case("elasticity")
    mg = Multigrid(pr, params, max_coarse=200)
    free = torch.as_tensor(~mg.masks[0], device="cuda", dtype=torch.float64)
    g = torch.Generator("cuda").manual_seed(5)
    r1 = torch.randn(len(free), dtype=torch.float64, device="cuda", generator=g) * free
    r2 = torch.randn(len(free), dtype=torch.float64, device="cuda", generator=g) * free
    a, b = float(mg.vcycle(r1) @ r2), float(r1 @ mg.vcycle(r2))
    assert abs(a - b) < 1e-12 * abs(a)
    mg.close()


def test_multigrid_pcg_on_the_plate():
    V, pr, params = workloads.config5(n=128)
    plain = jx.solve(pr, params=params, linear=jx.LinearOptions(tol=1e-8, maxiter=40000))
    mg = jx.solve(pr, params=params, linear=jx.LinearOptions(tol=1e-8, preconditioner="multigrid"))
    assert mg.stats["converged"] and mg.stats["relative_residual"] <= 1e-8
    assert mg.stats["iterations"] <= 30 < plain.stats["iterations"]
    assert np.linalg.norm(mg.u - plain.u) < 1e-5 * np.linalg.norm(plain.u)
    # a second solve reuses the hierarchy and the captured graph
    again = jx.solve(pr, params=params, linear=jx.LinearOptions(tol=1e-8, preconditioner="multigrid"))
    assert again.stats["iterations"] == mg.stats["iterations"] and np.array_equal(again.u, mg.u)


def test_multigrid_pcg_on_a_rational_patch_with_neumann_loads():
    V = jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 4.0).elevate(4).refine(5), vec=2)
    pr = jx.LinearElasticity(V, plane="stress",
                             dirichlet=[jx.DirichletBC(0.0, where="sym_y", component=1),
                                        jx.DirichletBC(0.0, where="sym_x", component=0)],
                             neumann=[jx.Neumann(lambda x, n, p: -10.0 * n, where="inner")])
    params = {"E": 1e5, "nu": 0.3}
    a = jx.solve(pr, params=params, linear=jx.LinearOptions(tol=1e-10))
    b = jx.solve(pr, params=params, linear=jx.LinearOptions(tol=1e-10, preconditioner="multigrid"))
    assert b.stats["converged"] and b.stats["iterations"] < a.stats["iterations"]
    assert np.linalg.norm(a.u - b.u) < 1e-7 * np.linalg.norm(a.u)
