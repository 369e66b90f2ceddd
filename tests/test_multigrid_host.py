"""The multigrid hierarchy on the host: coarse knot vectors, exact knot-insertion
prolongation (checked through the oracle's basis evaluation), the Galerkin
identity P^T K_h P = K_H of the rediscretised coarse operator, Dirichlet sets
that nest, and the coarse coefficient of a per-point field."""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

import jaxiga_b200 as jx
from jaxiga_b200 import workloads
from jaxiga_b200.multigrid import _coarse_problem, coarse_coefficients, coarse_knots, coarsen
from oracle import iga_oracle as O


def test_coarse_knots_remove_every_other_interior_knot():
    kv = np.array([0, 0, 0, 0.25, 0.5, 0.5, 0.75, 1, 1, 1])
    kc, back = coarse_knots(kv)
    assert list(kc) == [0, 0, 0, 0.5, 0.5, 1, 1, 1]
    assert list(back) == [0.25, 0.75]


def _full_P(Ps, vec):
    P = sp.csr_matrix(Ps[0])
    for d in range(1, len(Ps)):
        P = sp.kron(sp.csr_matrix(Ps[d]), P)
    return sp.kron(P, sp.eye(vec)).tocsr() if vec > 1 else P.tocsr()


@pytest.mark.parametrize("which", ["annulus", "cube"])
def test_prolongation_reproduces_the_coarse_function(which):
    if which == "annulus":
        V = jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 2.0).elevate(2).refine(3))
    else:
        kn = np.linspace(0, 1, 7)[1:-1]
        V = jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 2, 1]).elevate(3).insert_knots(kn, kn, kn))
    Vc, Ps, exact = coarsen(V)
    assert exact
    assert [n for n in Vc.n_span] == [(n + 1) // 2 for n in V.n_span]
    c = np.random.default_rng(0).standard_normal(Vc.n_scalar_basis)
    f = (_full_P(Ps, 1) @ (Vc.wgts * c)) / V.wgts  # knot insertion on homogeneous coefficients
    S, Sc = O.Space(V.knots, V.degree, V.cpts, V.wgts, 1), O.Space(Vc.knots, Vc.degree, Vc.cpts, Vc.wgts, 1)
    # the same physical points: fine element 0's Gauss points lie in coarse element 0 at known reference coords
    bf = O.evaluate(S, [0])
    from jaxiga_b200.pointset import tensor_rule

    rf, _ = tensor_rule([V.degree[0] + 1] * V.dim)
    # fine element 0 is [0, h_f]^d, coarse element 0 is [0, h_c]^d with h_c = 2 h_f
    scale = np.array([(V.span_hi[d][0] - V.span_lo[d][0]) / (Vc.span_hi[d][0] - Vc.span_lo[d][0]) for d in range(V.dim)])
    rc = -1.0 + (rf + 1.0) * scale
    bc = O.evaluate(Sc, [0], ref=rc)
    vf = bf["R"][0] @ f[bf["dofs"][0]]
    vc = bc["R"][0] @ c[bc["dofs"][0]]
    assert np.abs(bf["x"][0] - bc["x"][0]).max() < 1e-13
    assert np.abs(vf - vc).max() < 1e-12 * np.abs(vc).max()


@pytest.mark.parametrize("case", ["plate", "elasticity"])
def test_rediscretised_coarse_operator_is_galerkin(case):
    if case == "plate":
        V, pr, params = workloads.config5(n=8)
        op, par = "plate", dict(params)
    else:
        V, pr, params = workloads.config2(n=4)
        op, par = "elasticity", {"E": 1.0, "nu": 0.3}
    Vc, Ps, exact = coarsen(V)
    cpr = _coarse_problem(pr, Vc)
    S, Sc = O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec), O.Space(Vc.knots, Vc.degree, Vc.cpts, Vc.wgts, V.vec)
    pf, _ = pr.resolve_dirichlet(params)
    pc, _ = cpr.resolve_dirichlet(params)
    Af = O.Assembled(S, op, par, pf, np.zeros(len(pf)), need_full=False)
    Ac = O.Assembled(Sc, op, par, pc, np.zeros(len(pc)), need_full=False)
    P = _full_P(Ps, V.vec)
    # coarse free functions prolong to fine functions that vanish on the fine prescribed DOFs
    assert abs(P[pf][:, Ac.free]).max() < 1e-13
    G = (P[Af.free][:, Ac.free].T @ Af.K @ P[Af.free][:, Ac.free]).toarray()
    assert np.abs(G - Ac.K.toarray()).max() < 1e-11 * np.abs(Ac.K).max()


def test_coarse_coefficient_is_the_containing_fine_element_mean():
    kn = np.linspace(0, 1, 5)[1:-1]
    V = jx.FunctionSpace(jx.primitives.quadrilateral([[0, 0], [1, 0], [1, 1], [0, 1]]).elevate(2).insert_knots(kn, kn))
    Vc, _, _ = coarsen(V)
    fine = np.repeat(np.arange(V.n_elems, dtype=float)[:, None], 9, axis=1)
    c = coarse_coefficients(V, Vc, fine)
    assert c.shape == (Vc.n_elems, 9)
    # coarse element 0 covers fine elements 0, 1, 4, 5 (4 x 4 fine elements)
    assert set(np.unique(c[0]).tolist()) == {0.0, 1.0, 4.0, 5.0}
