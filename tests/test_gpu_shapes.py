"""Operator parity with the oracle across degrees, dimensions, operators and
knot layouts (uniform, graded, a repeated interior knot), at sizes the oracle
assembles in seconds. Bar: 1e-12 relative on K.v and diag K."""

import numpy as np
import pytest

import jaxiga_b200 as jx
from oracle import iga_oracle as O

pytestmark = pytest.mark.gpu


def patch(dim, p, n, layout, rational=False):
    P = jx.primitives
    if dim == 2:
        base = P.quarter_annulus(1.0, 2.0) if rational else P.rectangle(0, 0, 1.0, 0.7)
    else:
        base = P.cuboid([0, 0, 0], [1.0, 0.8, 1.2])
    base = base.elevate(p)
    kn = np.linspace(0, 1, n + 1)[1:-1]
    if layout == "graded":
        kn = kn**1.7
    elif layout == "repeated" and p >= 2:
        kn = np.sort(np.concatenate([kn, [kn[len(kn) // 2]]]))
    return base.insert_knots(*([kn] * dim))


def oracle_K(V, op, params, prescribed):
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec)
    return O.Assembled(S, op, params, prescribed, np.zeros(len(prescribed)), need_full=False)


CASES = [
    # dim, p, n, layout, op, rational
    (2, 1, 9, "uniform", "poisson", False),
    (2, 2, 37, "graded", "poisson", False),
    (2, 3, 35, "repeated", "poisson", False),
    (2, 4, 20, "uniform", "poisson", True),
    (2, 5, 12, "graded", "poisson", False),
    (2, 2, 11, "uniform", "poisson", True),
    (2, 3, 10, "graded", "elasticity", False),
    (2, 2, 9, "uniform", "elasticity", True),
    (2, 2, 14, "uniform", "plate", False),
    (2, 3, 10, "repeated", "plate", False),
    (2, 4, 9, "graded", "plate", True),
    (3, 1, 6, "uniform", "poisson", False),
    (3, 2, 7, "graded", "poisson", False),
    (3, 3, 9, "repeated", "poisson", False),
    (3, 4, 5, "uniform", "poisson", False),
    (3, 2, 5, "uniform", "elasticity", False),
    (3, 3, 6, "graded", "elasticity", False),
]


@pytest.mark.parametrize("dim,p,n,layout,op,rational", CASES)
def test_operator_matches_oracle(dim, p, n, layout, op, rational):
    vec = dim if op == "elasticity" else 1
    V = jx.FunctionSpace(patch(dim, p, n, layout, rational), vec=vec)
    rng = np.random.default_rng(dim * 100 + p * 10 + n)
    # Dirichlet on the first side (and the next layer for the plate)
    side = V.side_indices("u0")
    if op == "plate":
        side = np.union1d(side, V.side_indices("u0", offset=1))
    pres = np.sort(jx.expand_dofs(side[:, None], vec).ravel()) if vec > 1 else side
    mask = np.zeros(V.n_dofs, bool)
    mask[pres] = True
    coef = {"poisson": (1.3,), "elasticity": (2.0, 0.27), "plate": (2.0, 0.27, 0.1)}[op]
    params = {"poisson": {"a0": 1.3}, "elasticity": {"E": 2.0, "nu": 0.27},
              "plate": {"E": 2.0, "nu": 0.27, "t": 0.1}}[op]
    A = oracle_K(V, op, params, pres)
    dev = jx.Operator(V, op, coef, prescribed=mask)
    v = rng.standard_normal(len(A.free))
    x = np.zeros(V.n_dofs)
    x[A.free] = v
    y = dev.apply(x).cpu().numpy()[A.free]
    ref = A.K @ v
    assert np.abs(y - ref).max() / np.abs(ref).max() < 1e-12
    d = dev.diag().cpu().numpy()[A.free]
    assert np.abs(d - A.diag).max() / np.abs(A.diag).max() < 1e-12
    dev.close()


@pytest.mark.parametrize("p", [2, 3])
def test_poisson_load_and_interpolation_match_oracle(p):
    V = jx.FunctionSpace(patch(2, p, 13, "graded", rational=True))
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 1)
    dev = jx.Operator(V, "poisson", (1.0,))
    rng = np.random.default_rng(p)
    c = rng.standard_normal(V.n_scalar_basis)
    fq = dev.interpolate(c).cpu().numpy()
    ref = O.interpolate_qp(S, c)
    assert np.abs(fq - ref).max() < 1e-13 * np.abs(ref).max()
    F = dev.load(fq[..., 0]).cpu().numpy()
    A = O.Assembled(S, "poisson", {"a0": 1.0}, np.zeros(0, dtype=int), np.zeros(0), source_qp=fq[..., 0], need_full=False)
    assert np.abs(F - A.F).max() < 1e-13 * np.abs(A.F).max()
    dev.close()


@pytest.mark.parametrize("op", ["poisson", "elasticity", "plate"])
def test_brick_rows_leave_the_operator_unchanged(op):
    """2D bricks of 1 to 64 element rows (a runtime choice; small patches get
    short bricks by default) give the same K.v and diag K, also for the load."""
    vec = 2 if op == "elasticity" else 1
    V = jx.FunctionSpace(patch(2, 3, 23, "graded", rational=True), vec=vec)
    side = V.side_indices("u0")
    mask = np.zeros(V.n_dofs, bool)
    mask[np.unique(jx.expand_dofs(side, vec))] = True
    coef = {"poisson": (1.3,), "elasticity": (2.0, 0.27), "plate": (2.0, 0.27, 0.1)}[op]
    rng = np.random.default_rng(5)
    x = rng.standard_normal(V.n_dofs)
    ref = jx.Operator(V, op, coef, prescribed=mask)
    y0, d0 = ref.apply(x).cpu().numpy(), ref.diag().cpu().numpy()
    for tile in [(32, 1), (32, 3), (32, 8), (32, 64)]:
        dev = jx.Operator(V, op, coef, prescribed=mask, tile=tile)
        y, d = dev.apply(x).cpu().numpy(), dev.diag().cpu().numpy()
        assert np.abs(y - y0).max() <= 1e-12 * np.abs(y0).max(), tile
        assert np.abs(d - d0).max() <= 1e-12 * np.abs(d0).max(), tile
        dev.close()
    ref.close()
