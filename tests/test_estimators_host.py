"""Residual indicators (jaxiga_b200.estimators, after src/jaxiga/post/estimators.py)
against the oracle's restatement on tensor and THB spaces, with a known answer
and the argument checks of the reference's adapt driver. The oracle writes the
elasticity residual in its Lame form, the product from the constitutive
matrix, so the two are independent derivations."""

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200 import hierarchical as H
from jaxiga_b200.solve import Solution
from oracle import iga_oracle as O
from oracle import thb_oracle as TO

SQ = [[0, 0], [1, 0], [1, 1], [0, 1]]


def _thb(vec=1):
    return H.refine_elements(jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 2.0).elevate(3).refine(2), vec=vec),
                             [5, 6, 10])


def test_poisson_indicators_match_the_oracle_on_tensor_and_thb_spaces():
    rng = np.random.default_rng(0)
    src = lambda x, p: np.sin(x[0]) * x[1]  # noqa: E731
    V = jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 2.0).elevate(2).refine(2))
    for W, S in ((V, O.Space(V.knots, V.degree, V.cpts, V.wgts, 1)), (_thb(), None)):
        S = TO.ThbSpace.of(W) if S is None else S
        u = rng.standard_normal(W.n_dofs)
        eta = jx.residual_indicator(Solution(W, u, {"a0": 1.7}, jx.Poisson(W, source=src)))
        ref = O.residual_indicator(S, u, "poisson", {"a0": 1.7}, source=lambda x: np.sin(x[:, 0]) * x[:, 1])
        assert eta.shape == (W.n_elems,)
        assert np.abs(eta - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("dim", [2, 3])
def test_elasticity_indicators_match_the_oracle(dim):
    rng = np.random.default_rng(dim)
    if dim == 2:
        W = _thb(vec=2)
    else:
        W = H.refine_elements(jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(2).refine(1),
                                               vec=3), [0, 1])
    u = rng.standard_normal(W.n_dofs)
    src = lambda x, p: np.stack([x[0] * 0 + 0.5] + [x[1]] * (len(x) - 1))  # noqa: E731
    eta = jx.residual_indicator(Solution(W, u, {"E": 2.0, "nu": 0.3}, jx.LinearElasticity(W, source=src)))
    ref = O.residual_indicator(TO.ThbSpace.of(W), u, "elasticity", {"E": 2.0, "nu": 0.3},
                               source=lambda x: np.stack([x[:, 0] * 0 + 0.5] + [x[:, 1]] * (dim - 1), 1))
    assert np.abs(eta - ref).max() <= 1e-12 * np.abs(ref).max()


def test_known_answer_and_exact_fields():
    """u_h = 0 under f = 1 on the unit square: r = -1, so eta_e = h_e |e|^(1/2) =
    |e|. A linear field (its control values are the field at the control
    points, by linear precision) has no residual without a source."""
    V = jx.FunctionSpace(jx.primitives.quadrilateral(SQ).elevate(2).refine(2))
    one = lambda x, p: np.ones_like(x[0])  # noqa: E731
    eta = jx.residual_indicator(Solution(V, np.zeros(V.n_dofs), {"a0": 1.0}, jx.Poisson(V, source=one)))
    assert np.abs(eta - 1.0 / 16).max() < 1e-15
    u = V.cpts[:, 0] + 2.0 * V.cpts[:, 1]  # linear precision: control values of a linear field reproduce it
    eta = jx.residual_indicator(Solution(V, u, {"a0": 1.0}, jx.Poisson(V)))
    assert np.abs(eta).max() < 1e-12


def test_adapt_argument_checks():
    V = jx.FunctionSpace(jx.primitives.quadrilateral(SQ).elevate(2).refine(2))
    with pytest.raises(TypeError, match="factory"):
        jx.adapt(jx.Poisson(V))
    with pytest.raises(TypeError, match="starting space"):
        jx.adapt(lambda W: jx.Poisson(W))
    with pytest.raises(NotImplementedError):
        jx.residual_indicator(Solution(V, np.zeros(V.n_dofs), {"E": 1.0, "nu": 0.3, "t": 0.1},
                                       jx.KirchhoffPlate(V)))


def test_multipatch_indicators_are_the_patches_own():
    """On a conforming two-patch space the indicators are, patch by patch, the
    oracle's on each patch with its share of the global coefficients."""
    rect = jx.primitives.rectangle
    V = jx.FunctionSpace([rect(0, 0, 1, 1).elevate(2).refine(2), rect(1, 0, 2, 1).elevate(2).refine(2)])
    u = np.random.default_rng(3).standard_normal(V.n_dofs)
    eta = jx.residual_indicator(Solution(V, u, {"a0": 1.0}, jx.Poisson(V, source=lambda x, p: x[0] * x[1])))
    ref = np.concatenate([
        O.residual_indicator(O.Space(s.knots, s.degree, s.cpts, s.wgts, 1), u[V.topology.local_to_global[i]],
                             "poisson", {"a0": 1.0}, source=lambda x: x[:, 0] * x[:, 1])
        for i, s in enumerate(V.spaces)])
    assert np.abs(eta - ref).max() <= 1e-12 * np.abs(ref).max()
