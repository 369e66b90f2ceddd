"""The single-patch slab decomposition on CPU: partition, interface exchange and
the distributed Jacobi-PCG, with each slab's local operator emulated by the
oracle (its elements' tangents assembled into the slab's local DOF range).

Two gloo ranks exchange over torch.distributed; the loopback transport runs
three slabs in one process. Both must reproduce the global operator and the
global CG (the jax-CG restatement) of the same problem."""

from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import pytest
import scipy.sparse as sp
import torch
import torch.multiprocessing as mp

import jaxiga_b200 as jx
from jaxiga_b200.slab import LoopbackComm, SlabSolver, SlabSpace, partition
from oracle import iga_oracle as O


def _poisson2d():
    V = jx.FunctionSpace(jx.primitives.quadrilateral([[0, 0], [1, 0], [1, 1], [0, 1]]).elevate(3).refine(4))
    pr = jx.Poisson(V, dirichlet=[jx.DirichletBC(0.0, where="left")], source=lambda x, p: 1.0)
    return V, pr, "poisson", {"a0": 1.3}


def _elasticity3d():
    kx, kz = np.linspace(0, 1, 4)[1:-1], np.linspace(0, 1, 8)[1:-1]
    V = jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kx, kx, kz), vec=3)
    pr = jx.LinearElasticity(V, dirichlet=[jx.DirichletBC([0.0, 0.0, 0.0], where="left")])
    return V, pr, "elasticity", {"E": 1.0, "nu": 0.3}


CASES = {"poisson2d": _poisson2d, "elasticity3d": _elasticity3d}


def _setup(case):
    V, pr, op, params = CASES[case]()
    pres, _ = pr.resolve_dirichlet(params)
    mask = np.zeros(V.n_dofs, bool)
    mask[pres] = True
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, V.vec)
    return V, S, op, params, mask


def _local_operator(V, S, op, params, mask, slab):
    """The slab's elements assembled on its local DOF range (masked)."""
    ss = SlabSpace(V, slab)
    lo, hi = ss.dof_range()
    el = np.arange(V.n_elems)[ss.elem_slice()]
    basis = O.evaluate(S, el)
    Ke = O.element_tangents(op, basis, params, V.vec)
    gd = S.expand(S.elem_dofs[el]) - lo
    n = hi - lo
    rows = np.repeat(gd, gd.shape[1], axis=1).ravel()
    cols = np.tile(gd, (1, gd.shape[1])).ravel()
    K = sp.coo_matrix((Ke.ravel(), (rows, cols)), shape=(n, n)).tocsr()
    keep = (~mask[lo:hi]).astype(float)

    def apply(x):
        return torch.from_numpy(keep * (K @ (keep * x.numpy())))

    return ss, apply, torch.from_numpy(keep * K.diagonal()), torch.from_numpy(keep)


def _global(V, S, op, params, mask):
    pres = np.nonzero(mask)[0]
    A = O.Assembled(S, op, params, pres, np.zeros(len(pres)), need_full=False)
    return A


@pytest.mark.parametrize("case", list(CASES))
def test_partition_covers_elements_and_owns_every_layer(case):
    V = CASES[case]()[0]
    p = V.degree[-1]
    for world in (1, 2, 3):
        if V.n_span[-1] < world * p:
            continue
        slabs = partition(V, world)
        assert slabs[0].elem_lo == 0 and slabs[-1].elem_hi == V.n_span[-1]
        assert all(a.elem_hi == b.elem_lo for a, b in zip(slabs, slabs[1:]))
        assert slabs[0].own_lo == 0 and slabs[-1].own_hi == V.n_cp[-1]
        assert all(a.own_hi == b.own_lo for a, b in zip(slabs, slabs[1:]))
        for a, b in zip(slabs, slabs[1:]):
            assert a.cp_hi - b.cp_lo == p  # p shared layers between neighbours (C^{p-1})
            assert a.own_lo >= a.cp_lo and a.own_hi <= a.cp_hi
    with pytest.raises(ValueError):
        partition(V, V.n_span[-1])


@pytest.mark.parametrize("case", list(CASES))
def test_loopback_slabs_reproduce_global_apply_and_cg(case):
    V, S, op, params, mask = _setup(case)
    world = 3 if V.n_span[-1] >= 9 else 2
    slabs = partition(V, world)
    parts = [_local_operator(V, S, op, params, mask, s) for s in slabs]
    solver = SlabSolver(V, slabs, [p[0] for p in parts], [p[1] for p in parts], [p[2] for p in parts],
                        [p[3] for p in parts], LoopbackComm())
    A = _global(V, S, op, params, mask)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(V.n_dofs)
    ys = solver.apply(solver.scatter(torch.from_numpy(x)))
    y = np.zeros(V.n_dofs)
    y[A.free] = A.K @ x[A.free]
    for ss, yl in zip(solver.spaces, ys):
        lo, hi = ss.dof_range()
        assert np.abs(yl.numpy() - y[lo:hi]).max() < 1e-13 * np.abs(y).max()
    b = np.zeros(V.n_dofs)
    b[A.free] = rng.standard_normal(len(A.free))
    xs, k, rel = solver.pcg(solver.scatter(torch.from_numpy(b)), tol=1e-10)
    u = solver.gather(xs, V.n_dofs).numpy()
    x_o, k_o = O.jax_cg(lambda v: A.K @ v, b[A.free], 1e-10, inv_diag=O.jacobi_inverse(A.diag))
    assert _same_history(k, k_o), (k, k_o)
    assert np.linalg.norm(u[A.free] - x_o) < 1e-7 * np.linalg.norm(x_o)


def _same_history(k, k_o):
    """Iteration counts equal up to rounding: the slabs sum their dot products
    in another order than one array, which on an ill-conditioned system shifts
    a few hundred iterations by a few."""
    return abs(k - k_o) <= max(1, 0.02 * k_o)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, case, q):
    import torch.distributed as dist

    from jaxiga_b200.slab import TorchComm

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        V, S, op, params, mask = _setup(case)
        slabs = partition(V, world)
        ss, apply, diag, keep = _local_operator(V, S, op, params, mask, slabs[rank])
        solver = SlabSolver(V, slabs, [ss], [apply], [diag], [keep], TorchComm())
        rng = np.random.default_rng(0)
        x = rng.standard_normal(V.n_dofs)
        y = solver.apply(solver.scatter(torch.from_numpy(x)))[0].numpy()
        b = rng.standard_normal(V.n_dofs) * (~mask)
        xs, k, rel = solver.pcg(solver.scatter(torch.from_numpy(b)), tol=1e-10)
        u = solver.gather(xs, V.n_dofs).numpy()
        q.put((rank, ss.dof_range(), y, k, u))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", list(CASES))
def test_two_gloo_ranks_reproduce_global_apply_and_cg(case):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    V, S, op, params, mask = _setup(case)
    A = _global(V, S, op, params, mask)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(V.n_dofs)
    y = np.zeros(V.n_dofs)
    y[A.free] = A.K @ x[A.free]
    b = rng.standard_normal(V.n_dofs) * (~mask)
    x_o, k_o = O.jax_cg(lambda v: A.K @ v, b[A.free], 1e-10, inv_diag=O.jacobi_inverse(A.diag))
    us = []
    for rank, (lo, hi), yl, k, u in sorted(out, key=lambda t: t[0]):
        assert np.abs(yl - y[lo:hi]).max() < 1e-13 * np.abs(y).max()
        assert _same_history(k, k_o), (k, k_o)
        assert np.linalg.norm(u[A.free] - x_o) < 1e-7 * np.linalg.norm(x_o)
        us.append(u)
    assert np.array_equal(us[0], us[1])  # every rank ends with the same gathered solution
