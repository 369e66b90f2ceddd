"""Multipatch spaces on the device: the composite plan (jxb_mp_create) against
the oracle's per-patch assembly summed through the same global numbering, to
1e-12 on K.v and diag K; the glued solve against SuperLU; and the reference's
own downstream check (tests/test_multipatch.py:199-213): a glued space
reproduces a linear field across the interface."""

import numpy as np
import pytest
import scipy.sparse as sp

import jaxiga_b200 as jx
from oracle import iga_oracle as O

pytestmark = pytest.mark.gpu

rect = jx.primitives.rectangle


def cases():
    return {
        "squares": ([rect(0, 0, 1, 1).elevate(2).refine(2), rect(1, 0, 2, 1).elevate(2).refine(2)], 1, "poisson"),
        "annuli": ([jx.primitives.quarter_annulus(1.0, 2.0).elevate(2).refine(2),
                    jx.primitives.quarter_annulus(2.0, 3.0).elevate(2).refine(2)], 2, "elasticity"),
        "cubes": ([jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(2).refine(1),
                   jx.primitives.cuboid([1, 0, 0], [2, 1, 1]).elevate(2).refine(1)], 1, "poisson"),
        "cubes_p3": ([jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).refine(1),
                      jx.primitives.cuboid([0, 1, 0], [1, 2, 1]).elevate(3).refine(1)], 3, "elasticity"),
    }


def oracle_global(V, op, params):
    """sum_p P_p^T K_p P_p with the oracle's patch assembly."""
    n = V.n_dofs
    K = sp.csr_matrix((n, n))
    for i, s in enumerate(V.spaces):
        S = O.Space(s.knots, s.degree, s.cpts, s.wgts, V.vec)
        A = O.Assembled(S, op, params, np.zeros(0, dtype=int), np.zeros(0))
        g = jx.expand_dofs(V.topology.local_to_global[i][:, None], V.vec).reshape(-1) if V.vec > 1 else \
            V.topology.local_to_global[i]
        P = sp.csr_matrix((np.ones(len(g)), (np.arange(len(g)), g)), shape=(len(g), n))
        K = K + P.T @ A.K_full @ P
    return K.tocsr()


@pytest.mark.parametrize("name", list(cases()))
def test_composite_apply_and_diagonal_match_oracle(name):
    patches, vec, op = cases()[name]
    V = jx.FunctionSpace(patches, vec=vec)
    coef = (1.3,) if op == "poisson" else (2.0, 0.3)
    params = {"a0": 1.3} if op == "poisson" else {"E": 2.0, "nu": 0.3}
    K = oracle_global(V, op, params)
    from jaxiga_b200.multipatch import MultiPatchOperator

    dev = MultiPatchOperator(V, op, coef)
    x = np.random.default_rng(3).standard_normal(V.n_dofs)
    y = dev.apply(x, masked=False).cpu().numpy()
    assert np.abs(y - K @ x).max() <= 1e-12 * np.abs(K @ x).max()
    d = dev.diag().cpu().numpy()
    assert np.abs(d - K.diagonal()).max() <= 1e-12 * np.abs(K.diagonal()).max()
    dev.close()


def test_glued_solve_matches_superlu():
    patches, vec, op = cases()["squares"]
    V = jx.FunctionSpace(patches)
    problem = jx.Poisson(V, dirichlet=[jx.DirichletBC(0.0, where="left"), jx.DirichletBC(1.0, where="right")],
                         source=lambda x, p: 4.0 + 0.0 * x[0])
    sol = jx.solve(problem, params={"a0": 1.3}, linear=jx.LinearOptions(tol=1e-13))
    assert sol.stats["converged"]
    K = oracle_global(V, "poisson", {"a0": 1.3})
    pres, vals = problem.resolve_dirichlet({"a0": 1.3})
    free = np.setdiff1d(np.arange(V.n_dofs), pres)
    # load by the oracle, patch by patch through the numbering
    F = np.zeros(V.n_dofs)
    for i, s in enumerate(V.spaces):
        S = O.Space(s.knots, s.degree, s.cpts, s.wgts, 1)
        A = O.Assembled(S, "poisson", {"a0": 1.3}, np.zeros(0, dtype=int), np.zeros(0),
                        source_qp=np.full((s.n_elems, 9), 4.0), need_full=False)
        np.add.at(F, V.topology.local_to_global[i], A.F)
    u = np.zeros(V.n_dofs)
    u[pres] = vals
    rhs = F - K @ u
    u[free] = O.scipy_superlu(K[free][:, free], rhs[free])
    assert np.abs(sol.u - u).max() <= 1e-9 * np.abs(u).max()


def test_a_glued_space_reproduces_a_linear_field_across_the_interface():
    patches = [rect(0, 0, 1, 1).elevate(2).refine(2), rect(1, 0, 2, 1).elevate(2).refine(2)]
    V = jx.FunctionSpace(patches)
    exact = lambda x: 2.0 * x[0] - 3.0 * x[1] + 1.0  # noqa: E731
    sol = jx.solve(jx.Poisson(V, dirichlet=[jx.DirichletBC(lambda x, p: exact(x),
                                                           where=lambda X: np.ones(len(X), bool))]),
                   params={"a0": 1.0})
    assert jx.errornorm(sol, lambda x: exact(x.T), "L2") < 1e-10


def test_neumann_load_on_a_glued_space_matches_the_single_patch():
    """A traction on the far side of two glued squares equals the traction on
    the same side of one rectangle covering both, with identical knots (the
    rectangle's discretization is the two patches' union)."""
    import torch

    left, right = rect(0, 0, 1, 1).elevate(2).refine(2), rect(1, 0, 2, 1).elevate(2).refine(2)
    V = jx.FunctionSpace([left, right], vec=2)
    trac = [jx.Neumann(lambda x, n, p: np.stack([np.full(len(x), 1.5), x[:, 1] ** 2], axis=1), where="right"),
            jx.Neumann(lambda x, n, p: np.stack([0.5 * x[:, 0], np.full(len(x), -1.0)], axis=1), where="top")]
    problem = jx.LinearElasticity(V, plane="strain", dirichlet=[jx.DirichletBC([0.0, 0.0], where="left")],
                                  neumann=trac)
    sol = jx.solve(problem, params={"E": 10.0, "nu": 0.3}, linear=jx.LinearOptions(tol=1e-13))
    assert sol.stats["converged"]
    # one patch over [0, 2] x [0, 1] with the union's knots
    # 8 elements along x, the interface x = 1 (parameter 0.5) only C0 (multiplicity p = 2) as in the glued space
    kn = np.concatenate([np.linspace(0, 0.5, 5)[1:-1], [0.5, 0.5], 0.5 + np.linspace(0, 0.5, 5)[1:-1]])
    one = rect(0, 0, 2, 1).elevate(2).insert_knots(kn, np.linspace(0, 1, 5)[1:-1])
    W = jx.FunctionSpace(one, vec=2)
    p1 = jx.LinearElasticity(W, plane="strain", dirichlet=[jx.DirichletBC([0.0, 0.0], where="left")], neumann=trac)
    s1 = jx.solve(p1, params={"E": 10.0, "nu": 0.3}, linear=jx.LinearOptions(tol=1e-13))
    # compare at the Gauss points of both (same physical elements, patch order differs): use norms
    assert abs(jx.norm(sol, "L2") - jx.norm(s1, "L2")) <= 1e-9 * jx.norm(s1, "L2")
    assert abs(jx.norm(sol, "H1") - jx.norm(s1, "H1")) <= 1e-9 * jx.norm(s1, "H1")
    del torch
