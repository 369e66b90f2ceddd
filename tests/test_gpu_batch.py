"""Batched solves of uneven instances (the configuration with 256 quarter annuli,
here at test size): the batch must agree with per-instance solves (the
reference's "batched solve equals the Python loop", tests/test_advanced.py:338-356),
every tile shape must give the same operator, and the autotuner must return one
of the supported shapes per degree."""

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200 import batch, workloads
from jaxiga_b200.solve import geometry_operator
from oracle import iga_oracle as O

pytestmark = pytest.mark.gpu


def interp(V, c):
    return geometry_operator(V).interpolate(c).cpu().numpy()


def small_batch(n=10):
    return workloads.config3(n_instances=n, interpolate=interp, span_range=(3, 20))


def test_batched_solve_equals_the_loop():
    import torch

    problems, params = small_batch(10)
    bs = batch.BatchSolver(problems, params)
    xs, stats, secs = bs.solve(tol=1e-12)
    assert secs > 0
    for pr, pa, x, st in zip(problems, params, xs, stats):
        assert st["converged"], st
        ref = jx.solve(pr, params=pa, linear=jx.LinearOptions(tol=1e-12))
        u = x.cpu().numpy()
        assert np.linalg.norm(u - ref.u) <= 1e-9 * np.linalg.norm(ref.u)
    bs.close()


def test_batched_solve_matches_oracle_superlu():
    problems, params = small_batch(4)
    bs = batch.BatchSolver(problems, params)
    xs, stats, _ = bs.solve(tol=1e-12)
    for pr, pa, x in zip(problems, params, xs):
        V = pr.space
        S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 1)
        pres, vals = pr.resolve_dirichlet(pa)
        f = np.asarray(pa["f"].values)
        A = O.Assembled(S, "poisson", {"a0": pa["a0"]}, pres, vals, source_qp=f)
        u_ref = A.lift(O.scipy_superlu(A.K, A.b))
        u = x.cpu().numpy()
        assert np.linalg.norm(u - u_ref) <= 1e-9 * np.linalg.norm(u_ref)
    bs.close()


@pytest.mark.parametrize("tile", batch.TILES)
def test_every_tile_shape_gives_the_same_operator(tile):
    problems, params = small_batch(3)
    rng = np.random.default_rng(0)
    for pr, pa in zip(problems, params):
        m = batch._mask(pr, pa)
        a = jx.Operator(pr.space, "poisson", (pa["a0"],), prescribed=m)
        b = jx.Operator(pr.space, "poisson", (pa["a0"],), prescribed=m, tile=tile)
        x = rng.standard_normal(pr.space.n_dofs)
        ya, yb = a.apply(x).cpu().numpy(), b.apply(x).cpu().numpy()
        assert np.abs(ya - yb).max() <= 1e-12 * np.abs(ya).max()
        da, db = a.diag().cpu().numpy(), b.diag().cpu().numpy()
        assert np.abs(da - db).max() <= 1e-12 * np.abs(da).max()
        a.close()
        b.close()


def test_autotuner_picks_a_supported_tile_per_degree():
    problems, params = small_batch(6)
    best, timings = batch.autotune_tiles(problems, params, reps=3)
    degrees = {pr.space.degree[0] for pr in problems}
    assert set(best) == degrees
    for p, tile in best.items():
        assert tile in batch.TILES
        assert timings[(p, tile)] == min(timings[(p, t)] for t in batch.TILES)


CHILD = r"""
import sys, numpy as np, torch
sys.path.insert(0, {root!r})
sys.path.insert(0, {tests!r})
from test_gpu_batch import small_batch
from jaxiga_b200 import batch, _lib
problems, params = small_batch(12)
bs = batch.BatchSolver(problems, params, tiles={{p: (32, 8) for p in (1, 2, 3, 4, 5)}})
assert not bs.batch.persistent
x = torch.from_numpy(np.load({xin!r})).cuda()
y = torch.empty_like(x)
_lib.check(bs.batch.lib.jxb_batch_apply(bs.batch.handle, torch.cuda.current_stream().cuda_stream, x.data_ptr(),
                                        y.data_ptr()))
np.save({out!r}, y.cpu().numpy())
"""


def test_persistent_launch_equals_the_per_degree_launches(tmp_path, monkeypatch):
    """With JXB_BATCH_PERSIST=1 and rows of 32 elements one persistent launch
    walks the bricks of every instance and degree; without it (a child process)
    the same bricks run as one launch per degree group. Same bricks, same
    per-brick arithmetic: the two K.u agree to rounding, and a second persistent
    apply (the work counter has reset itself) repeats the first."""
    import os
    import subprocess
    import sys

    import torch

    from jaxiga_b200 import _lib

    problems, params = small_batch(12)
    assert len({pr.space.degree[0] for pr in problems}) > 1
    tiles = {p: (32, 8) for p in (1, 2, 3, 4, 5)}
    monkeypatch.setenv("JXB_BATCH_PERSIST", "1")
    bs = batch.BatchSolver(problems, params, tiles=tiles)
    assert bs.batch.persistent and bs.batch.brick_launches == 1
    x = torch.randn(bs.batch.total, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    ys = []
    for _ in range(2):
        y = torch.empty_like(x)
        _lib.check(bs.batch.lib.jxb_batch_apply(bs.batch.handle, torch.cuda.current_stream().cuda_stream,
                                                x.data_ptr(), y.data_ptr()))
        ys.append(y.cpu().numpy())
    assert np.array_equal(ys[0], ys[1])
    # the persistent batch also solves: every instance converges
    xs, stats, _ = bs.solve(tol=1e-10)
    assert all(st["converged"] for st in stats)
    xin, out = str(tmp_path / "x.npy"), str(tmp_path / "y.npy")
    np.save(xin, x.cpu().numpy())
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    env.pop("JXB_BATCH_PERSIST", None)
    subprocess.run([sys.executable, "-c", CHILD.format(root=root, tests=os.path.join(root, "tests"), xin=xin, out=out)],
                   env=env, check=True, cwd=root, timeout=600)
    y_groups = np.load(out)
    assert np.abs(ys[0] - y_groups).max() <= 1e-14 * np.abs(y_groups).max()
    # and each instance's block equals its own operator's K.u
    for i, op in enumerate(bs.ops):
        lo, hi = bs.batch.offsets[i], bs.batch.offsets[i + 1]
        yi = op.apply(x[lo:hi].contiguous()).cpu().numpy()
        assert np.abs(ys[0][lo:hi] - yi).max() <= 1e-13 * max(np.abs(yi).max(), 1e-300)
    bs.close()
