"""The slab decomposition on the device: every slab's libjxb plan on one GPU,
exchanged through the in-process loopback transport (no ranks waiting on one
another), against the single-plan apply and Jacobi-PCG of the whole patch."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import jaxiga_b200 as jx
from jaxiga_b200 import workloads
from jaxiga_b200.slab import device_slab_solver
from jaxiga_b200.solve import geometry_operator

pytestmark = pytest.mark.gpu


def _mask(V, problem, params):
    pres, _ = problem.resolve_dirichlet(params)
    m = np.zeros(V.n_dofs, bool)
    m[pres] = True
    return m


@pytest.mark.parametrize("world", [2, 3])
def test_device_slabs_match_the_whole_patch_elasticity(world):
    V, problem, params = workloads.config2(n=12)
    mask = _mask(V, problem, params)
    whole = jx.Operator(V, "elasticity", (1.0, 0.3), prescribed=mask)
    slab = device_slab_solver(V, "elasticity", (1.0, 0.3), mask, world)
    x = torch.randn(V.n_dofs, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    y = whole.apply(x)
    ys = slab.apply(slab.scatter(x))
    yg = slab.gather(ys, V.n_dofs)
    assert float((yg - y).abs().max() / y.abs().max()) < 1e-13
    fq = geometry_operator(V).interpolate(params["eta"])
    fq[..., 2] -= 1.0
    b = whole.load(fq)
    u, st = whole.pcg(b, tol=1e-10)
    xs, k, rel = slab.pcg(slab.scatter(b), tol=1e-10)
    ug = slab.gather(xs, V.n_dofs)
    assert abs(k - st["iterations"]) <= max(1, 0.02 * st["iterations"])
    assert float(torch.linalg.norm(ug - u) / torch.linalg.norm(u)) < 1e-7
    for op in slab.ops:
        op.close()
    whole.close()


def test_device_slabs_with_a_pointfield_coefficient():
    V, problem, params = workloads.config4(n=12)
    a = torch.exp(geometry_operator(V).interpolate(params["loga"])[..., 0]).cpu().numpy()
    mask = _mask(V, problem, params)
    whole = jx.Operator(V, "poisson", (1.0,), prescribed=mask, coef_qp=a)
    slab = device_slab_solver(V, "poisson", (1.0,), mask, 3, coef_qp=a)
    x = torch.randn(V.n_dofs, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(4))
    yg = slab.gather(slab.apply(slab.scatter(x)), V.n_dofs)
    y = whole.apply(x)
    assert float((yg - y).abs().max() / y.abs().max()) < 1e-13
    for op in slab.ops:
        op.close()
    whole.close()
