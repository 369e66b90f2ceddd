"""One patch across GPUs: slabs of element layers with a p-layer exchange.

The reference runs one patch on one device (it has no multi-device code);
this module splits the matrix-free solve of ``matrix_free_solve``
(src/jaxiga/solvers/linear.py:414-442) over processes, one per GPU.

Partition. The elements are cut into ``world`` slabs of whole element layers
along the slowest parametric direction (z in 3D, y in 2D). A slab holds the
control-point layers its elements touch: global layers [cp_lo, cp_hi). For a
C^{p-1} spline neighbouring slabs share p layers, and each slab needs at
least p element layers so that only neighbours share. Every layer is owned
by exactly one slab -- slab r owns [cp_lo_r, cp_lo_{r+1}) -- for the dot
products. A slab's DOFs are a contiguous slice of the global DOF vector
(layers are the slowest index), so its plan is an ordinary libjxb plan of the
sliced space: the same extraction rows, first indices shifted by cp_lo.

Apply. Each slab applies its local operator (its elements only). On the
shared layers that gives partial sums; each slab sends its upper shared
layers to the slab above and its lower ones to the slab below, receives the
neighbours' partials for the same layers and adds them. Both copies of a
shared layer then hold a + b and b + a, which are equal bit for bit.

CG. Jacobi-PCG in jax CG semantics (x0 = 0, stop on r.r <= tol^2 b.b), with
the dot products over owned layers and one FP64 allreduce per reduction point
(p.Ap, then r.z and r.r packed together). Every rank takes the same
collective steps in the same order.

Transport. ``TorchComm`` uses torch.distributed (NCCL between GPUs, gloo on
CPU): batched point-to-point send/recv of the interface layers and
``all_reduce``. ``LoopbackComm`` holds every slab in one process and exchanges
by copies, so the decomposition can run on a single device with no ranks
waiting on one another.
"""

from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass(frozen=True)
class Slab:
    """Slab ``rank`` of a partition: element layers [elem_lo, elem_hi), control-point
    layers held [cp_lo, cp_hi) and owned [own_lo, own_hi), all along the slowest direction."""

    rank: int
    elem_lo: int
    elem_hi: int
    cp_lo: int
    cp_hi: int
    own_lo: int
    own_hi: int

    @property
    def n_layers(self):
        return self.cp_hi - self.cp_lo


def partition(space, world):
    """Balanced slabs of element layers along the slowest direction."""
    d = space.dim - 1
    ns, p = space.n_span[d], space.degree[d]
    first = np.asarray(space.first[d])
    if world < 1:
        raise ValueError("world must be >= 1")
    if world * p > ns:
        raise ValueError(f"{ns} element layers cannot give {world} slabs of at least p = {p} layers")
    bounds = [int(round(r * ns / world)) for r in range(world + 1)]
    slabs = []
    for r in range(world):
        e0, e1 = bounds[r], bounds[r + 1]
        c0, c1 = int(first[e0]), int(first[e1 - 1]) + p + 1
        own_hi = int(first[bounds[r + 1]]) if r + 1 < world else space.n_cp[d]
        slabs.append(Slab(r, e0, e1, c0, c1, c0, own_hi))
    for a, b in zip(slabs, slabs[1:]):
        if b.cp_lo < a.cp_lo or b.cp_lo > a.cp_hi:
            raise ValueError("knot multiplicities leave slabs without a shared interface")
    return slabs


class SlabSpace:
    """The space of one slab: the attributes a libjxb plan reads, sliced."""

    def __init__(self, space, slab):
        d = space.dim - 1
        self.parent, self.slab = space, slab
        self.dim, self.vec, self.degree = space.dim, space.vec, space.degree
        self.n_cp = list(space.n_cp)
        self.n_cp[d] = slab.n_layers
        self.n_span = list(space.n_span)
        self.n_span[d] = slab.elem_hi - slab.elem_lo
        sl = slice(slab.elem_lo, slab.elem_hi)
        self.first = [np.asarray(f) for f in space.first]
        self.first[d] = np.asarray(space.first[d])[sl] - slab.cp_lo
        self.span_lo = list(space.span_lo)
        self.span_hi = list(space.span_hi)
        self.ext1d = list(space.ext1d)
        self.span_lo[d] = np.asarray(space.span_lo[d])[sl]
        self.span_hi[d] = np.asarray(space.span_hi[d])[sl]
        self.ext1d[d] = np.asarray(space.ext1d[d])[sl]
        self.layer = int(np.prod(space.n_cp[:d]))  # control points per layer
        rows = slice(slab.cp_lo * self.layer, slab.cp_hi * self.layer)
        self.cpts = np.asarray(space.cpts)[rows]
        self.wgts = np.asarray(space.wgts)[rows]
        self.n_scalar_basis = slab.n_layers * self.layer
        self.n_elems = int(np.prod(self.n_span))
        self._plans = {}

    @property
    def n_dofs(self):
        return self.n_scalar_basis * self.vec

    def dof_range(self):
        """This slab's slice of the global DOF vector."""
        s = self.slab
        return s.cp_lo * self.layer * self.vec, s.cp_hi * self.layer * self.vec

    def local_range(self, lo_layer, hi_layer):
        """Local DOF slice of the global layers [lo_layer, hi_layer)."""
        k = self.layer * self.vec
        return slice((lo_layer - self.slab.cp_lo) * k, (hi_layer - self.slab.cp_lo) * k)

    def elem_slice(self):
        """This slab's elements in the global element order (a contiguous range)."""
        per = int(np.prod(self.parent.n_span[:-1]))
        return slice(self.slab.elem_lo * per, self.slab.elem_hi * per)


def interfaces(slabs, r):
    """Global layer ranges that slab r shares with the slab below and above (or None)."""
    s = slabs[r]
    lower = (s.cp_lo, slabs[r - 1].cp_hi) if r > 0 else None
    upper = (slabs[r + 1].cp_lo, s.cp_hi) if r + 1 < len(slabs) else None
    return lower, upper


class LoopbackComm:
    """Every slab in this process; exchanges are copies, reductions sums."""

    def ranks(self, world):
        return list(range(world))

    def exchange(self, ys, spaces, slabs):
        """Add the neighbours' partial sums on the shared layers of every slab."""
        parts = []
        for r in range(len(slabs)):
            _, upper = interfaces(slabs, r)
            if upper is None:
                continue
            a = spaces[r].local_range(*upper)
            b = spaces[r + 1].local_range(*upper)
            parts.append((r, a, b, ys[r][a].clone(), ys[r + 1][b].clone()))
        for r, a, b, ya, yb in parts:
            ys[r][a] += yb
            ys[r + 1][b] += ya

    def allreduce(self, vals):
        """vals: one tensor of scalars per local slab -> their sum."""
        out = vals[0].clone()
        for v in vals[1:]:
            out += v
        return out


class TorchComm:
    """One slab per process over torch.distributed (NCCL on GPUs, gloo on CPUs)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)

    def ranks(self, world):
        return [self.rank]

    def exchange(self, ys, spaces, slabs):
        dist, r = self.dist, self.rank
        y, sp = ys[0], spaces[0]
        lower, upper = interfaces(slabs, r)
        ops, recv = [], []
        for rng, peer in ((lower, r - 1), (upper, r + 1)):
            if rng is None:
                continue
            sl = sp.local_range(*rng)
            buf = y[sl].clone()
            got = y.new_empty(buf.shape)
            ops.append(dist.P2POp(dist.isend, buf, peer, self.group))
            ops.append(dist.P2POp(dist.irecv, got, peer, self.group))
            recv.append((sl, got, buf))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for sl, got, _ in recv:
            y[sl] += got

    def allreduce(self, vals):
        t = vals[0].clone()
        self.dist.all_reduce(t, group=self.group)
        return t


class SlabSolver:
    """Apply and Jacobi-PCG of one patch split into slabs.

    ``applies[i](x_i) -> y_i`` is the local masked operator of the i-th slab held
    by this process and ``diags[i]`` its local diagonal (partial sums on shared
    layers, completed here by the exchange); ``keeps[i]`` the free-DOF masks.
    """

    def __init__(self, space, slabs, spaces, applies, diags, keeps, comm):
        self.space, self.slabs, self.spaces, self.comm = space, slabs, spaces, comm
        self.applies, self.keeps = applies, keeps
        self.mine = comm.ranks(len(slabs))
        diags = [d.clone() for d in diags]
        comm.exchange(diags, spaces, slabs)
        self.inv = [k * _safe_inv(d) for d, k in zip(diags, keeps)]
        self.owned = []
        for sp in spaces:
            m = diags[0].new_zeros(sp.n_dofs)
            m[sp.local_range(sp.slab.own_lo, sp.slab.own_hi)] = 1.0
            self.owned.append(m)

    def apply(self, xs):
        ys = [f(x) for f, x in zip(self.applies, xs)]
        self.comm.exchange(ys, self.spaces, self.slabs)
        return ys

    def dots(self, pairs):
        """Global dot products of several vector pairs, one allreduce."""
        import torch

        loc = [torch.stack([torch.dot(a[i] * self.owned[i], b[i]) for a, b in pairs]) for i in range(len(self.owned))]
        return self.comm.allreduce(loc)

    def scatter(self, v):
        """Local slices of a global vector (host or device tensor)."""
        out = []
        for sp in self.spaces:
            lo, hi = sp.dof_range()
            out.append(v[lo:hi].clone())
        return out

    def pcg(self, bs, tol=1e-10, maxiter=None):
        """Jacobi-PCG from 0; returns (local solutions, iterations, relative residual norm)."""
        xs = [b.new_zeros(b.shape) for b in bs]
        rs = [b * k for b, k in zip(bs, self.keeps)]
        zs = [i * r for i, r in zip(self.inv, rs)]
        ps = [z.clone() for z in zs]
        rz, rr, bb = self.dots([(rs, zs), (rs, rs), (rs, rs)]).tolist()
        n_free = int(self.dots([(self.keeps, self.keeps)])[0].item())
        maxiter = 10 * n_free if maxiter is None else int(maxiter)
        atol2 = tol * tol * bb
        k = 0
        while rr > atol2 and k < maxiter:
            aps = self.apply(ps)
            pap = float(self.dots([(ps, aps)])[0].item())
            alpha = rz / pap
            for i in range(len(xs)):
                xs[i] += alpha * ps[i]
                rs[i] -= alpha * aps[i]
                zs[i] = self.inv[i] * rs[i]
            rz_new, rr = self.dots([(rs, zs), (rs, rs)]).tolist()
            beta = rz_new / rz
            rz = rz_new
            for i in range(len(ps)):
                ps[i] = zs[i] + beta * ps[i]
            k += 1
        return xs, k, float(np.sqrt(rr / bb)) if bb > 0 else 0.0

    def gather(self, locals_, n):
        """The global vector from the owned layers of the local ones (loopback:
        all slabs here; distributed: every rank contributes its owned part)."""
        import torch

        out = locals_[0].new_zeros(n)
        for sp, v in zip(self.spaces, locals_):
            lo, _ = sp.dof_range()
            sl = sp.local_range(sp.slab.own_lo, sp.slab.own_hi)
            out[lo + sl.start: lo + sl.stop] = v[sl]
        if isinstance(self.comm, TorchComm):
            self.comm.dist.all_reduce(out, group=self.comm.group)
        return out


def _safe_inv(d):
    """1/d where |d| > 0, else 1 (solvers/linear.py:427-431)."""
    import torch

    return torch.where(d.abs() > 0, 1.0 / torch.where(d.abs() > 0, d, torch.ones_like(d)), torch.ones_like(d))


def device_slab_solver(space, op_name, coef, prescribed_mask, world, comm=None, coef_qp=None):
    """SlabSolver on libjxb plans of the slabs this process holds (all of them
    with the default LoopbackComm; its own with a TorchComm)."""
    from .operator import Operator

    comm = comm or LoopbackComm()
    slabs = partition(space, world)
    spaces, applies, diags, keeps, ops = [], [], [], [], []
    for r in comm.ranks(world):
        sp = SlabSpace(space, slabs[r])
        lo, hi = sp.dof_range()
        mask = np.asarray(prescribed_mask, dtype=bool)[lo:hi]
        cq = None
        if coef_qp is not None:
            cq = np.asarray(coef_qp).reshape(space.n_elems, -1)[sp.elem_slice()]
        op = Operator(sp, op_name, coef, prescribed=mask, coef_qp=cq)
        spaces.append(sp)
        ops.append(op)
        applies.append(lambda x, op=op: op.apply(x))
        diags.append(op.diag())
        import torch

        keeps.append(torch.as_tensor(~mask, dtype=torch.float64, device=op.device))
    solver = SlabSolver(space, slabs if isinstance(comm, LoopbackComm) else slabs, spaces, applies, diags, keeps, comm)
    solver.ops = ops
    return solver
