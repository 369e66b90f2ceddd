"""Multipatch topology on the host (jaxiga_b200/multipatch.py): the gluing
and refusals the reference's own tests pin (tests/test_multipatch.py:30-197),
and the global numbering and boundaries of a glued space
(src/jaxiga/space/function_space.py:372-535)."""

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200.multipatch import MultiPatchSpace, NonConformingError, OrientationError, compute_topology

rect = jx.primitives.rectangle
cube = jx.primitives.cuboid


def test_abutting_squares_share_one_interface():
    left, right = rect(0, 0, 1, 1).elevate(2), rect(1, 0, 2, 1).elevate(2)
    topo = compute_topology([left, right])
    assert len(topo.interfaces) == 1
    assert topo.n_global_dofs == left.n_cp + right.n_cp - 3


def test_corner_contact_is_not_an_interface():
    topo = compute_topology([rect(0, 0, 1, 1).elevate(1), rect(1, 1, 2, 2).elevate(1)])
    assert len(topo.interfaces) == 0 and topo.n_global_dofs == 7


def test_disjoint_patches_are_left_alone():
    topo = compute_topology([rect(0, 0, 1, 1).elevate(1), rect(3, 3, 4, 4).elevate(1)])
    assert len(topo.interfaces) == 0 and topo.n_global_dofs == 8


def test_three_dimensional_edge_contact_is_allowed():
    topo = compute_topology([cube([0, 0, 0], [1, 1, 1]).elevate(1), cube([1, 1, 0], [2, 2, 1]).elevate(1)])
    assert len(topo.interfaces) == 0 and topo.n_global_dofs == 14


def test_curved_nurbs_patches_glue():
    inner = jx.primitives.quarter_annulus(1.0, 2.0).elevate(2)
    outer = jx.primitives.quarter_annulus(2.0, 3.0).elevate(2)
    assert len(compute_topology([inner, outer]).interfaces) == 1


def test_three_dimensional_face_glues_and_counts():
    a = cube([0, 0, 0], [1, 1, 1]).elevate(2).refine(1)
    b = cube([1, 0, 0], [2, 1, 1]).elevate(2).refine(1)
    topo = compute_topology([a, b])
    assert len(topo.interfaces) == 1
    assert topo.n_global_dofs == a.n_cp + b.n_cp - 16  # a 4 x 4 face shared


def test_reversed_interface_glues():
    """The right patch's u direction runs the other way along the shared edge."""
    left = rect(0, 0, 1, 1).elevate(2)
    right = rect(1, 0, 2, 1).elevate(2)
    n = right.n_cp_per_dir
    grid = np.arange(right.n_cp).reshape(n[::-1])[::-1, :].ravel()  # flip v
    flipped = jx.Patch.create(right.knots, right.degree, right.ctrl_pts[grid], right.weights[grid])
    topo = compute_topology([left, flipped])
    assert len(topo.interfaces) == 1 and topo.interfaces[0].reversed
    assert topo.n_global_dofs == left.n_cp + right.n_cp - 3


@pytest.mark.parametrize("patches", [
    [rect(0, 0, 1, 1).elevate(2), rect(0, 0, 1, 1).elevate(2)],                       # duplicated
    [cube([0, 0, 0], [1, 1, 1]).elevate(1), cube([0, 0, 0], [1, 1, 1]).elevate(1)],   # duplicated cuboid
    [rect(0, 0, 1, 1).elevate(2).refine(1), rect(1, 0, 2, 1).elevate(2)],             # mismatched refinement
    [rect(0, 0, 1, 2).elevate(1).refine(1), rect(1, 0, 2, 1).elevate(1)],             # partial abutment
])
def test_non_conforming_contact_is_rejected(patches):
    with pytest.raises((NonConformingError, OrientationError)):
        compute_topology(patches)


def test_glued_space_numbering_and_boundaries():
    V = jx.FunctionSpace([rect(0, 0, 1, 1).elevate(2).refine(2), rect(1, 0, 2, 1).elevate(2).refine(2)], vec=2)
    assert isinstance(V, MultiPatchSpace)
    assert V.n_scalar_basis == 2 * 36 - 6 and V.n_dofs == 2 * V.n_scalar_basis
    assert V.n_elems == 32
    # the shared edge is interior: no boundary label covers its inner points
    assert sorted(V.boundaries) == ["bottom", "left", "right", "top"]
    x = V.cpts
    right = V.boundary("right").dofs
    assert np.allclose(x[right, 0], 2.0)
    left = V.boundary("left").dofs
    assert np.allclose(x[left, 0], 0.0)
    # every element's DOFs are global indices, and the glued points appear in both patches
    shared = set(V.topology.local_to_global[0]) & set(V.topology.local_to_global[1])
    assert len(shared) == 6 and np.allclose(x[sorted(shared), 0], 1.0)
