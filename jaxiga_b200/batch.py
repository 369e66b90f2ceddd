"""Batched solves of many independent 2D Poisson problems, plus the tile autotuner.

``BatchSolver(problems, params)`` builds one device plan per problem (uneven
sizes and degrees are fine), the load vectors with the device load kernel,
and a libjxb batch: every Jacobi-PCG iteration of all instances runs as a
handful of launches captured in one CUDA graph (see include/jxb.h).

``autotune_tiles`` times the batched operator application for each supported
2D brick shape on the problems of each degree and returns the fastest shape
per degree; ``BatchSolver(..., tiles="auto")`` runs it first.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .forms import PointField, call_points, flat_params
from .operator import Operator
from .solve import qp_points

TILES = [(32, 8), (16, 8), (32, 16), (64, 4), (32, 2), (16, 2), (32, 1), (64, 1)]


def _s():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _mask(problem, params):
    pres, vals = problem.resolve_dirichlet(params)
    if np.any(vals != 0):
        raise NotImplementedError("batched solves take homogeneous Dirichlet data")
    m = np.zeros(problem.space.n_dofs, bool)
    m[pres] = True
    return m


class _Batch:
    def __init__(self, ops):
        self.lib = _lib.load()
        arr = (ctypes.c_void_p * len(ops))(*[op.handle.value for op in ops])
        h = ctypes.c_void_p()
        _lib.check(self.lib.jxb_batch_create(arr, len(ops), ctypes.byref(h)))
        self.handle = h
        total = ctypes.c_int64()
        offs = (ctypes.c_int64 * (len(ops) + 1))()
        _lib.check(self.lib.jxb_batch_size(h, ctypes.byref(total), offs))
        self.total = total.value
        self.offsets = np.array(offs[:], dtype=np.int64)
        pers, launches = ctypes.c_int(), ctypes.c_int()
        _lib.check(self.lib.jxb_batch_info(h, ctypes.byref(pers), ctypes.byref(launches)))
        self.persistent = bool(pers.value)  # one persistent launch over every degree
        self.brick_launches = launches.value

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.jxb_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def time_batch_apply(ops, reps=10):
    """Device ms of one batched masked K.u over all instances (CUDA events)."""
    import torch

    b = _Batch(ops)
    x = torch.randn(b.total, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    for _ in range(2):
        _lib.check(b.lib.jxb_batch_apply(b.handle, _s(), _p(x), _p(y)))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        _lib.check(b.lib.jxb_batch_apply(b.handle, _s(), _p(x), _p(y)))
    e1.record()
    torch.cuda.synchronize()
    b.close()
    return e0.elapsed_time(e1) / reps


def autotune_tiles(problems, params_list, candidates=TILES, reps=10):
    """Fastest 2D brick shape per degree, timed on the batch's own problems."""
    by_degree = {}
    for pr, pa in zip(problems, params_list):
        by_degree.setdefault(pr.space.degree[0], []).append((pr, pa))
    best, timings = {}, {}
    for p, items in by_degree.items():
        t_best = None
        for tile in candidates:
            ops = [Operator(pr.space, "poisson", pr.operator_coefficients(pa)[0], prescribed=_mask(pr, pa), tile=tile)
                   for pr, pa in items]
            ms = time_batch_apply(ops, reps)
            for op in ops:
                op.close()
            timings[(p, tile)] = ms
            if t_best is None or ms < t_best:
                t_best, best[p] = ms, tile
    return best, timings


class BatchSolver:
    """All instances solved together on the GPU (Jacobi-PCG, jax CG semantics)."""

    def __init__(self, problems, params_list, tiles=None):
        import torch

        self.problems = list(problems)
        self.params = list(params_list)
        for pr in self.problems:
            if pr.op != "poisson" or pr.space.dim != 2:
                raise NotImplementedError("batched solves take 2D Poisson problems")
        self.tune = None
        if tiles == "auto":
            tiles, self.tune = autotune_tiles(self.problems, self.params)
        # default: 16 x 8 element bricks for every degree (the autotuner's pick on
        # the 256-annuli batch); JXB_BATCH_PERSIST=1 with 32-wide tiles runs the
        # persistent launch instead
        self.tiles = tiles or {p: (16, 8) for p in (1, 2, 3, 4, 5)}
        self.ops = []
        loads = []
        for pr, pa in zip(self.problems, self.params):
            coef, field = pr.operator_coefficients(pa)
            if field is not None:
                raise NotImplementedError("batched solves take a constant a0 per instance")
            op = Operator(pr.space, "poisson", coef, prescribed=_mask(pr, pa), tile=self.tiles.get(pr.space.degree[0]))
            self.ops.append(op)
            if pr.source is None:
                loads.append(torch.zeros(op.n_dofs, dtype=torch.float64, device=op.device))
            else:
                x = qp_points(pr.space)
                f = call_points(pr.source, x, flat_params(pa, x.shape[0])).reshape(-1)
                loads.append(op.load(np.array(f, dtype=np.float64, copy=True)))
        self.batch = _Batch(self.ops)
        self.b = torch.cat(loads).contiguous()

    def solve(self, tol=1e-10, maxiter=None, check_every=16):
        import torch

        x = torch.empty_like(self.b)
        o = self.ops[0]._opts(tol, 0.0, maxiter, "jacobi", check_every, 0.0, 0)
        n = len(self.ops)
        stats = (_lib.Stats * n)()
        secs = ctypes.c_double()
        rc = self.batch.lib.jxb_batch_pcg(self.batch.handle, _s(), _p(self.b), _p(x), ctypes.byref(o), stats,
                                          ctypes.byref(secs))
        _lib.check_solve(rc)
        off = self.batch.offsets
        xs = [x[off[i]: off[i + 1]] for i in range(n)]
        st = [{k: getattr(stats[i], k) for k, _ in _lib.Stats._fields_} for i in range(n)]
        return xs, st, secs.value

    def close(self):
        self.batch.close()
        for op in self.ops:
            op.close()


if __name__ == "__main__":
    import argparse
    import json

    import torch

    from . import workloads
    from .solve import geometry_operator

    ap = argparse.ArgumentParser(description="batched K.u over the quarter-annulus instances")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--tiles", default="default",
                    help="'default' (rows of 32 elements: one persistent launch over every degree) or WxH for "
                         "every degree (e.g. 16x8: one launch per degree group)")
    a = ap.parse_args()
    problems, params = workloads.config3(n_instances=a.instances,
                                         interpolate=lambda V, c: geometry_operator(V).interpolate(c).cpu().numpy())
    tiles = None
    if a.tiles != "default":
        w, h = (int(v) for v in a.tiles.split("x"))
        tiles = {p: (w, h) for p in (1, 2, 3, 4, 5)}
    bs = BatchSolver(problems, params, tiles=tiles)
    b = bs.batch
    x = torch.randn(b.total, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    for _ in range(3):
        _lib.check(b.lib.jxb_batch_apply(b.handle, _s(), _p(x), _p(y)))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        _lib.check(b.lib.jxb_batch_apply(b.handle, _s(), _p(x), _p(y)))
    e1.record()
    torch.cuda.synchronize()
    n_qp = sum(pr.space.n_elems * (pr.space.degree[0] + 1) ** 2 for pr in problems)
    ms = e0.elapsed_time(e1) / a.reps
    print(json.dumps({"instances": a.instances, "tiles": a.tiles, "persistent": b.persistent,
                      "brick_launches": b.brick_launches, "n_dofs": int(b.total), "gauss_points": n_qp,
                      "ms_per_apply": ms, "algorithmic_gbs": (16 * b.total + 48 * n_qp) / (ms * 1e-3) / 1e9}))
    bs.close()
