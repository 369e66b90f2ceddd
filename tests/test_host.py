"""Host-side logic of the product (CPU only): geometry, space setup, boundary
conditions, options validation, and the C-ABI library's exported symbols."""

import ctypes
import hashlib
import os
import re

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200 import _lib
from tests.cases import CASES, build, golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("tag", CASES)
def test_space_setup_matches_reference(tag):
    g = golden()
    V, problem, params = build(tag)
    for d in range(V.dim):
        np.testing.assert_array_equal(np.asarray(V.patch.knots[d]), g[f"{tag}/knots{d}"])
        np.testing.assert_array_equal(V.ext1d[d], g[f"{tag}/extraction{d}"])
        np.testing.assert_array_equal(V.first[d], g[f"{tag}/first{d}"])
    np.testing.assert_array_equal(V.elem_dofs, g[f"{tag}/elem_dofs"])
    np.testing.assert_array_equal(V.elem_vertex, g[f"{tag}/elem_vertex"])
    np.testing.assert_allclose(V.cpts, g[f"{tag}/cpts"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(V.wgts, g[f"{tag}/wgts"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("tag", CASES)
def test_dirichlet_partition_matches_reference(tag):
    g = golden()
    V, problem, params = build(tag)
    pres, vals = problem.resolve_dirichlet(params)
    np.testing.assert_array_equal(pres, g[f"{tag}/prescribed"])
    np.testing.assert_allclose(vals, g[f"{tag}/prescribed_values"], rtol=0, atol=1e-14)


@pytest.mark.parametrize("p", [2, 3, 4])
def test_annulus_geometry_matches_reference(p):
    g = golden()
    patch = jx.primitives.quarter_annulus(1.0, 2.0).elevate(p).insert_knots(
        np.linspace(0, 1, 6)[1:-1], np.linspace(0, 1, 4)[1:-1])
    for d in range(2):
        np.testing.assert_array_equal(np.asarray(patch.knots[d]), g[f"annulus_p{p}/knots{d}"])
    np.testing.assert_allclose(patch.ctrl_pts, g[f"annulus_p{p}/cpts"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(patch.weights, g[f"annulus_p{p}/wgts"], rtol=0, atol=1e-15)


def test_full_size_extraction_is_bit_exact():
    g = golden()
    for tag, p, n in (("ext_c2", 3, 64), ("ext_c4", 3, 96), ("ext_c5", 4, 256)):
        kv = np.concatenate([np.zeros(p + 1), np.linspace(0, 1, n + 1)[1:-1], np.ones(p + 1)])
        np.testing.assert_array_equal(np.stack(jx.bezier_extraction(kv, p)), g[f"{tag}/C"])


@pytest.mark.parametrize("key", [k for k in golden().files if k.startswith("bezier/") and k.endswith("/C")])
def test_bezier_extraction_known_answers(key):
    g = golden()
    deg = int(key.split("/")[1].split("_")[0][1:])
    np.testing.assert_array_equal(np.stack(jx.bezier_extraction(g[key[:-2] + "/knots"], deg)), g[key])


def test_cube16_connectivity_checksums():
    g = golden()
    kn = np.linspace(0, 1, 17)[1:-1]
    V = jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kn), vec=3)
    assert sha(V.elem_dofs.astype(np.int64)) == str(g["cube16/elem_dofs_sha"])
    assert sha(V.elem_vertex) == str(g["cube16/elem_vertex_sha"])
    np.testing.assert_array_equal(V.extraction([0, 17, 4095]), g["cube16/ops_sample"])
    pr = jx.Problem(V, dirichlet=[jx.DirichletBC([0.0, 0.0, 0.0], where="left")])
    assert sha(pr.resolve_dirichlet()[0].astype(np.int64)) == str(g["cube16/prescribed_sha"])


def test_refinement_preserves_geometry():
    """Knot insertion and degree elevation leave the NURBS map unchanged."""
    from oracle import iga_oracle as O

    base = jx.primitives.quarter_annulus(1.0, 2.0)
    fine = base.elevate(4).insert_knots([0.2, 0.5, 0.5], [0.3, 0.7])
    for patch in (base, fine):
        S = O.Space(patch.knot_arrays(), patch.degree, patch.ctrl_pts, patch.weights)
        x = O.evaluate(S, np.arange(S.n_elems))["x"].reshape(-1, 2)
        r = np.hypot(x[:, 0], x[:, 1])
        assert np.all(r > 1 - 1e-12) and np.all(r < 2 + 1e-12)
    S = O.Space(fine.knot_arrays(), fine.degree, fine.ctrl_pts, fine.weights)
    w = O.evaluate(S, np.arange(S.n_elems))["w"]
    # rational integrand: Gauss quadrature on this coarse mesh is accurate to ~1e-11
    assert abs(w.sum() - 3 * np.pi / 4) < 1e-9


def test_clamping_constrains_two_layers():
    V = jx.FunctionSpace(jx.primitives.rectangle(0, 0, 1, 1).elevate(3).refine(2))
    simple = jx.KirchhoffPlate(V, dirichlet=[jx.DirichletBC(0.0, where="left")])
    clamped = jx.KirchhoffPlate(V, dirichlet=[jx.ClampedBC(where="left")])
    assert len(clamped.resolve_dirichlet()[0]) == 2 * len(simple.resolve_dirichlet()[0])


def test_problem_validation():
    V = jx.FunctionSpace(jx.primitives.rectangle(0, 0, 1, 1).refine(2))
    with pytest.raises(ValueError, match="degree"):
        jx.KirchhoffPlate(V)
    with pytest.raises(ValueError, match="vec == dim"):
        jx.LinearElasticity(V)
    with pytest.raises(ValueError, match="homogeneous"):
        jx.ClampedBC(value=1.0, where="left")
    with pytest.raises(ValueError, match="component"):
        jx.Poisson(V, dirichlet=[jx.DirichletBC(0.0, where="left", component=2)])


def test_linear_options_validation():
    """solvers/linear.py:102-127 of the reference plus the device fields."""
    with pytest.raises(ValueError, match="tol"):
        jx.LinearOptions(tol=0.0)
    with pytest.raises(ValueError, match="maxiter"):
        jx.LinearOptions(maxiter=0)
    with pytest.raises(ValueError, match="method"):
        jx.LinearOptions(method="lu")
    with pytest.raises(ValueError, match="preconditioner"):
        jx.LinearOptions(preconditioner="ilu")
    with pytest.raises(ValueError, match="SuperLU"):
        jx.LinearOptions(superlu_ordering="bad")
    with pytest.raises(ValueError, match="iterative"):
        jx.LinearOptions(method="scipy", matrix_free=True)
    with pytest.raises(ValueError, match="precision"):
        jx.LinearOptions(precision="fp16")
    assert jx.LinearOptions(precision="mixed").precision == "mixed"
    assert jx.LinearOptions(precision="mixed").refinement == "reliable"
    with pytest.raises(ValueError, match="refinement"):
        jx.LinearOptions(precision="mixed", refinement="defect")
    with pytest.raises(ValueError, match="update_delta"):
        jx.LinearOptions(precision="mixed", update_delta=1.0)


def header_symbols():
    text = open(os.path.join(ROOT, "include", "jxb.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(jxb_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = header_symbols()
    assert len(declared) >= 10
    for name in declared:
        assert hasattr(lib, name), name
    bound = {n for n, _ in _lib.SIGNATURES}
    assert set(declared) == bound


def test_library_reports_errors_without_a_gpu():
    lib = _lib.load()
    assert lib.jxb_version() >= 1
    out = ctypes.c_void_p()
    rc = lib.jxb_plan_create(None, ctypes.byref(out))
    assert rc == 1
    assert b"desc" in lib.jxb_last_error()
    # argument checks come before any device work
    assert lib.jxb_mixed_pcg(None, None, None, None, None, None) == 1
    assert b"jxb_mixed_pcg" in lib.jxb_last_error()
    assert lib.jxb_cnn_set_input_pooling(None, 1) == 1
    assert b"input_pooling" in lib.jxb_last_error()


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors have the sizes and field offsets the C compiler gives include/jxb.h."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"jxb_desc": _lib.Desc, "jxb_info": _lib.Info, "jxb_solve_opts": _lib.SolveOpts, "jxb_stats": _lib.Stats,
               "jxb_transfer1d": _lib.Transfer1d, "jxb_thb_desc": _lib.ThbDesc}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "jxb.h"', "int main(void){"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.split("\n") if line)
    for cname, cls in structs.items():
        assert int(out[cname]) == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(out[f"{cname}.{fname}"]) == getattr(cls, fname).offset, f"{cname}.{fname}"


def test_batch_rejects_a_plan_listed_twice():
    """A plan given twice would share its brick scratch inside one launch; the
    pointers are checked before any plan is read, so a stand-in pointer works."""
    lib = _lib.load()
    buf = ctypes.create_string_buffer(64)
    fake = ctypes.cast(buf, ctypes.c_void_p).value
    arr = (ctypes.c_void_p * 2)(fake, fake)
    out = ctypes.c_void_p()
    assert lib.jxb_batch_create(arr, 2, ctypes.byref(out)) == 1
    assert b"more than once" in lib.jxb_last_error()
    assert out.value is None


def test_solve_status_codes_map_to_stats():
    """NOT_CONVERGED and NONFINITE come back with x and stats written: they are
    reported through the stats, every other code raises."""
    assert _lib.check_solve(0) == 0
    assert _lib.check_solve(3) == 3
    assert _lib.check_solve(4) == 4
    with pytest.raises(_lib.JxbError):
        _lib.check_solve(4, raise_on_nonfinite=True)
    with pytest.raises(_lib.JxbError):
        _lib.check_solve(1)


def test_linear_options_learned_and_restarts():
    import jaxiga_b200 as jx

    with pytest.raises(ValueError, match="checkpoint"):
        jx.LinearOptions(preconditioner="learned")
    o = jx.LinearOptions(preconditioner="learned", checkpoint="net.npz", learned_map="multiplicative")
    assert o.learned_map == "multiplicative"
    with pytest.raises(ValueError, match="learned_map"):
        jx.LinearOptions(preconditioner="learned", checkpoint="net.npz", learned_map="other")
    for bad in (-1, 9, 1.5, True):
        with pytest.raises(ValueError, match="restarts"):
            jx.LinearOptions(restarts=bad)
    assert jx.LinearOptions().restarts == 3


def test_point_set_gauss_rule_matches_oracle_order():
    import jaxiga_b200 as jx
    from oracle import iga_oracle as O

    kn = np.linspace(0, 1, 4)[1:-1]
    V = jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(2).insert_knots(kn, kn, kn))
    for q in (None, 2, 5):
        ps = jx.gauss(V, q)
        pts, wts = O.gauss_rule([(p + 1) if q is None else q for p in V.degree])
        assert np.array_equal(ps.ref, pts) and np.array_equal(ps.weights, wts)
        e, r = ps.flat()
        assert e.shape == (V.n_elems * len(pts),) and r.shape == (V.n_elems * len(pts), 3)
        assert np.array_equal(e[: len(pts)], np.zeros(len(pts))) and np.array_equal(r[: len(pts)], pts)
    per_elem = jx.PointSet(elems=[3, 1], ref=np.zeros((2, 4, 3)))
    assert not per_elem.shared_ref and per_elem.n_pts == 8
    with pytest.raises(ValueError):
        jx.PointSet(elems=[0, 1, 2], ref=np.zeros((2, 4, 3)))


def test_error_norm_argument_checks_come_first():
    import jaxiga_b200 as jx

    sol = jx.Solution(space=None, u=None)
    with pytest.raises(ValueError, match="unknown norm"):
        jx.errornorm(sol, lambda x: x, "H2")
    with pytest.raises(ValueError, match="exact_grad"):
        jx.errornorm(sol, lambda x: x, "H1")
    with pytest.raises(ValueError, match="unknown norm"):
        jx.norm(sol, "energy")


def test_elasticity_constitutive_matches_oracle():
    import jaxiga_b200 as jx
    from oracle import iga_oracle as O

    for dim, plane in ((3, "stress"), (2, "stress"), (2, "strain")):
        kn = np.linspace(0, 1, 3)[1:-1]
        patch = (jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(2).insert_knots(kn, kn, kn) if dim == 3 else
                 jx.primitives.rectangle(0, 0, 1, 1).elevate(2).insert_knots(kn, kn))
        V = jx.FunctionSpace(patch, vec=dim)
        pr = jx.LinearElasticity(V, plane=plane)
        assert np.allclose(pr.C({"E": 2.0, "nu": 0.25}), O.isotropic(2.0, 0.25, dim, plane), rtol=1e-15, atol=0)


def test_direct_and_gmres_methods_are_accepted_like_the_reference():
    """LinearOptions(method="scipy") is the reference's default direct solve;
    the drop-in accepts it (and "dense", "gmres") and runs the device CG."""
    for m in ("scipy", "dense", "gmres", "cg", "bicgstab"):
        o = jx.LinearOptions(method=m)
        assert o.method == m and not o.matrix_free
    with pytest.raises(ValueError):
        jx.LinearOptions(method="dense", matrix_free=True)
