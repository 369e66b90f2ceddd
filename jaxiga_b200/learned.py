"""Learned preconditioner: a 3D U-Net on the control-point grid inside flexible CG.

Pipeline (all arithmetic in libjxb's kernels; torch holds device memory):

1. ``pairs_from_solve``: one plain FP64 Jacobi-PCG solve records its iterates
   x_j; with the converged x*, e_j = x* - x_j and r_j = K e_j (exact, one
   operator application each) are the (residual, error) pairs CG actually
   meets, early rough residuals and late smooth ones alike.
2. ``train``: by default the energy-norm angle between the network's output
   z = N(in_scale r/||r||) and the error e, 1 - (z.r)^2 / ((z^T K z)(e^T K e))
   (r = K e), forward and backward through the network's own kernels and the
   operator apply, Adam on the flat parameter vector. The energy norm weighs
   the error the way CG convergence does, and the angle ignores the scale of
   z, which flexible CG does not use: for a smooth residual the error is
   orders of magnitude larger than for a rough one of the same norm, a range
   a network fed unit-norm inputs cannot span. The scaled energy norm
   (e - z)^T K (e - z) / e^T K e and a masked MSE are kept for comparison.
3. ``solve``: truncated flexible CG with z = ||r|| out_scale N(in_scale r/||r||)
   and Jacobi-PCG as the fallback (jxb_fcg_learned), optionally as FP32 inner
   solves inside FP64 iterative refinement.

Weights and scales are saved to / resumed from ``.npz`` files.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class _DeviceArray:
    """Zero-copy torch view of a raw device pointer (CUDA array interface)."""

    def __init__(self, ptr, n, typestr="<f4"):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2}


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _s():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class LearnedPreconditioner:
    """CNN preconditioner for an :class:`~jaxiga_b200.Operator` on a single patch.

    Parameters
    ----------
    op : Operator
        The operator (its Dirichlet mask defines the free DOFs).
    features : array (n_feat, n_scalar_basis) or None
        Static per-control-point input channels, e.g. a normalised log-coefficient.
    channels : sequence of int or None
        Channels per U-Net level (2..6 levels, each in {4,8,12,16,24,32,48,64});
        None picks :func:`default_channels` for the grid the network runs on.
    pool_input : bool
        Run the network on the 2x2x2-pooled residual (half resolution) and
        upsample its output: the network then supplies the smooth part of the
        correction, the Jacobi term of the additive two-level map the rest, at
        about an eighth of the finest level's cost.
    """

    def __init__(self, op, features=None, channels=None, seed=0, pool_input=False):
        import torch

        self.lib = _lib.load()
        self.op = op
        self.vec = op.vec
        sp = op.space
        self.grid = (sp.n_cp[0], sp.n_cp[1], sp.n_cp[2] if sp.dim == 3 else 1)
        self.ncp = sp.n_scalar_basis
        self.dev = op.device
        if features is not None:
            f = torch.as_tensor(np.asarray(features), dtype=torch.float32, device=self.dev).reshape(-1, self.ncp)
            self.features = f.contiguous()
        else:
            self.features = None
        self.n_feat = 0 if self.features is None else self.features.shape[0]
        self.pool_input = bool(pool_input)
        if channels is None:
            g = self.grid
            channels = default_channels(tuple((n + 1) // 2 for n in g) if self.pool_input else g)
        self.channels = tuple(int(c) for c in channels)
        ch = (ctypes.c_int32 * len(self.channels))(*self.channels)
        h = ctypes.c_void_p()
        _lib.check(self.lib.jxb_cnn_create(self.vec + self.n_feat, self.vec, len(self.channels), ch, int(seed),
                                           ctypes.byref(h)))
        self.handle = h
        if self.pool_input:
            _lib.check(self.lib.jxb_cnn_set_input_pooling(h, 1))
        ptr, n = ctypes.c_void_p(), ctypes.c_int64()
        _lib.check(self.lib.jxb_cnn_params(h, ctypes.byref(ptr), ctypes.byref(n)))
        self.params = torch.as_tensor(_DeviceArray(ptr.value, n.value), device=self.dev)
        self.n_params = n.value
        self.in_scale = 1.0
        self.out_scale = 1.0
        self.additive_weight = 1.0
        self.history = []
        self.inference_bf16 = False

    def set_inference_bf16(self, on=True):
        """Run the network's applications in the solver (and ``forward``) with
        the BF16 tensor-core convolution on its layers of at most 32 channels;
        training keeps FP32."""
        _lib.check(self.lib.jxb_cnn_set_inference_bf16(self.handle, 1 if on else 0))
        self.inference_bf16 = bool(on)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.jxb_cnn_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- layout helpers ----------------------------------------------------------
    def _to_grid(self, v):
        """DOF vector (vec*i + c) -> [vec, ncp] float32."""
        return v.reshape(self.ncp, self.vec).t().contiguous().float()

    def _input(self, r_grid):
        import torch

        if self.features is None:
            return r_grid.contiguous()
        return torch.cat([r_grid, self.features], 0).contiguous()

    # -- data ------------------------------------------------------------------
    def pairs_from_solve(self, b, n_pairs=2000, every=1, tol=1e-12, maxiter=None):
        """Residual/error pairs of one plain FP64 Jacobi-PCG solve of K x = b:
        the starting point x_0 = 0, then the iterate after every ``every`` steps.

        Returns (R, E, stats): R, E float32 [n, vec, ncp], each pair scaled by
        1/||r_j||, the solve's stats, and sets in_scale / out_scale.
        """
        import torch

        op = self.op
        b = op._vec(b)
        x = op._empty(op.n_dofs)
        snaps = torch.empty((int(n_pairs), op.n_dofs), dtype=torch.float64, device=self.dev)
        o = op._opts(tol, 0.0, maxiter, "jacobi", every, 0.0, 0)
        st = _lib.Stats()
        ns = ctypes.c_int64()
        _lib.check_solve(self.lib.jxb_pcg_snapshots(op.handle, _s(), _p(b), _p(x), ctypes.byref(o), int(every),
                                                    _p(snaps), int(n_pairs), ctypes.byref(ns), ctypes.byref(st)),
                         raise_on_nonfinite=True)
        m = min(ns.value + 1, int(n_pairs))
        R = torch.empty((m, self.vec, self.ncp), dtype=torch.float32, device=self.dev)
        E = torch.empty_like(R)
        for j in range(m):
            # pair 0 is the starting iterate x_0 = 0 (e_0 = x*, r_0 = b on the
            # free DOFs); CG iterates are zero on prescribed DOFs, so e_j is too,
            # and the masked operator gives the exact residual r_j = K e_j.
            e = x if j == 0 else x - snaps[j - 1]
            r = op.apply(e)
            rn = float(torch.linalg.norm(r))
            R[j] = self._to_grid(r / rn)
            E[j] = self._to_grid(e / rn)
        del snaps
        free = int(op.info["n_free"])
        self.in_scale = float(np.sqrt(free))
        self.out_scale = float(torch.sqrt((E.double() ** 2).sum() / max(m * free, 1)))
        stats = {k: getattr(st, k) for k, _ in _lib.Stats._fields_}
        return R, E, stats

    def pairs_random(self, n_pairs, tol=1e-10, seed=0, maxiter=None):
        """Pairs (r, K^-1 r) for seeded r ~ N(0, I) on the free DOFs.

        Each e = K^-1 r comes from a plain FP64 Jacobi-PCG solve to ``tol``.
        White-noise residuals cover the whole spectrum, which the iterates of a
        few Krylov solves do not. Returns float32 [n, vec, ncp] R, E normalised
        by ||r|| (the scales of ``pairs_from_solve`` are left unchanged).
        """
        import torch

        op = self.op
        gen = torch.Generator(device=self.dev).manual_seed(int(seed))
        free = torch.as_tensor(~op.prescribed_mask, device=self.dev)
        R = torch.empty((int(n_pairs), self.vec, self.ncp), dtype=torch.float32, device=self.dev)
        E = torch.empty_like(R)
        for j in range(int(n_pairs)):
            r = torch.randn(op.n_dofs, dtype=torch.float64, device=self.dev, generator=gen) * free
            e, st = op.pcg(r, tol=tol, maxiter=maxiter, preconditioner="jacobi")
            rn = float(torch.linalg.norm(r))
            R[j] = self._to_grid(r / rn)
            E[j] = self._to_grid(e / rn)
        return R, E

    @property
    def mask(self):
        """Loss mask on the grid: 1 where any component of the control point is free."""
        import torch

        free = ~self.op.prescribed_mask.reshape(self.ncp, self.vec)
        return torch.as_tensor(free.any(axis=1).astype(np.float32), device=self.dev)

    # -- training ----------------------------------------------------------------
    def train(self, R, E, epochs=4, lr=2e-3, batch=4, seed=0, loss="angle", log=None):
        """Adam on the energy-norm angle (or scaled energy norm, or masked-MSE) loss;
        returns the per-epoch mean losses. ``loss="additive"`` takes the angle of
        the additive two-level map z = n + D^-1 r, so that the network learns
        what the Jacobi step misses (use ``two_level="additive"`` with it)."""
        import torch

        if loss not in ("angle", "additive", "energy", "mse"):
            raise ValueError("loss must be 'angle', 'additive', 'energy' or 'mse'")
        g = torch.Generator().manual_seed(seed)
        nx, ny, nz = self.grid
        m = R.shape[0]
        mask = self.mask.contiguous()
        if loss == "energy":
            # e^T K e of each normalised pair is e . r (r = K e exactly)
            w = (1.0 / (E.double() * R.double()).sum(dim=(1, 2))).cpu().tolist()
        losses = []
        for ep in range(epochs):
            order = torch.randperm(m, generator=g).tolist()
            tot, cnt = 0.0, 0
            for i0 in range(0, m, batch):
                _lib.check(self.lib.jxb_cnn_zero_grad(self.handle, _s()))
                idx = order[i0:i0 + batch]
                for j in idx:
                    inp = self._input(R[j] * self.in_scale)
                    val = ctypes.c_double()
                    if loss in ("energy", "angle", "additive"):
                        angle = {"energy": 0, "angle": 1, "additive": 2}[loss]
                        _lib.check(self.lib.jxb_cnn_accumulate_energy(
                            self.op.handle, self.handle, _s(), _p(inp), _p(E[j].contiguous()),
                            _p(R[j].contiguous()) if angle else None, float(self.out_scale),
                            1.0 if angle else float(w[j]), angle, ctypes.byref(val)))
                    else:
                        tgt = (E[j] / self.out_scale).contiguous()
                        _lib.check(self.lib.jxb_cnn_accumulate(self.handle, _s(), nx, ny, nz, _p(inp), _p(tgt),
                                                               _p(mask), ctypes.byref(val)))
                    tot += val.value
                    cnt += 1
                _lib.check(self.lib.jxb_cnn_adam(self.handle, _s(), float(lr), 1.0 / len(idx)))
            losses.append(tot / max(cnt, 1))
            if log:
                log(f"epoch {ep}: loss {losses[-1]:.4e}")
        self.history += losses
        return losses

    def forward(self, r):
        """z = ||r|| out_scale N(in_scale r / ||r||) for a DOF vector r (the preconditioner map)."""
        import torch

        nx, ny, nz = self.grid
        r = self.op._vec(r)
        rn = float(torch.linalg.norm(r))
        inp = self._input(self._to_grid(r / rn) * self.in_scale)
        out = torch.empty((self.vec, self.ncp), dtype=torch.float32, device=self.dev)
        _lib.check(self.lib.jxb_cnn_forward(self.handle, _s(), nx, ny, nz, _p(inp), _p(out)))
        z = out.double().t().reshape(-1) * rn * self.out_scale
        return (z * torch.as_tensor(~self.op.prescribed_mask, device=self.dev)).contiguous()

    def fit_additive_weight(self, R, E, n_pairs=64):
        """Weight a of the network in the additive two-level map z = a n + D^-1 r,
        for a network trained on its own (``loss="angle"``); one trained on the
        map itself (``loss="additive"``) keeps a = 1.

        For a pair (r, e = K^-1 r) the energy-optimal a minimises
        ||e - a n - D^-1 r||_K: a = (n.r - (K n).(D^-1 r)) / (n^T K n). The pooled
        estimate sums numerator and denominator over up to ``n_pairs`` pairs,
        each normalised by its e.r. One operator apply per pair; sets and
        returns ``additive_weight``.
        """
        import torch

        op = self.op
        inv = op.diag()
        free = torch.as_tensor(~op.prescribed_mask, device=self.dev)
        inv = torch.where(free & (inv.abs() > 0), 1.0 / torch.where(inv.abs() > 0, inv, torch.ones_like(inv)),
                          torch.zeros_like(inv))
        num = den = 0.0
        m = min(int(R.shape[0]), int(n_pairs))
        for j in range(m):
            r = R[j].t().reshape(-1).double().contiguous()
            e = E[j].t().reshape(-1).double().contiguous()
            er = float(e @ r)
            if not er > 0:
                continue
            z = self.forward(r)
            Kz = op.apply(z)
            num += (float(z @ r) - float(Kz @ (inv * r))) / er
            den += float(z @ Kz) / er
        if not den > 0:
            raise ValueError("fit_additive_weight: the network output has no energy on these pairs")
        self.additive_weight = num / den
        return self.additive_weight

    # -- solve -------------------------------------------------------------------
    def solve(self, b, tol=1e-8, maxiter=None, stall=50, depth=4, mixed=False, inner_tol=None, check_every=16,
              use_network=True, two_level=False, refinement="reliable", restarts=3):
        """Flexible CG with this preconditioner (Jacobi fallback); returns (x, stats).

        ``restarts``: when the flexible CG's recursive residual met ``tol`` but
        the true FP64 residual did not, up to this many correction solves on the
        true residual, each to half the remaining target, on a shared iteration
        budget -- the rule of the reference's CPU CG
        (src/jaxiga/solvers/linear.py:261-321). ``stats["restarts"]`` counts them.

        ``mixed``: the flexible CG runs in FP32 with FP64 corrections. With
        ``refinement="reliable"`` the FP32 iterate is folded into the FP64
        solution and the residual recomputed in FP64 each time the residual has
        fallen by ``inner_tol`` (default 1e-2), keeping the stored directions;
        with ``"restart"`` each FP32 solve to ``inner_tol`` (default 1e-4) starts
        afresh inside FP64 iterative refinement.
        ``two_level``: ``True`` (or ``"multiplicative"``) takes the network
        output n as a coarse correction with its own line search, then one
        Jacobi step: z = a n + D^-1 (r - a K n), one more apply per iteration;
        ``"additive"`` uses z = a n + D^-1 r with the fixed weight
        ``additive_weight`` (``fit_additive_weight``) and no extra apply.
        ``use_network=False`` runs the same FCG with Jacobi only (the baseline
        the network is measured against).
        """
        if refinement not in ("reliable", "restart"):
            raise ValueError(f"refinement must be 'reliable' or 'restart', got {refinement!r}")
        if isinstance(restarts, bool) or not isinstance(restarts, (int, np.integer)) or not 0 <= restarts <= 8:
            raise ValueError("restarts must be an integer in 0..8")
        kw = dict(stall=stall, depth=depth, mixed=mixed, inner_tol=inner_tol, check_every=check_every,
                  use_network=use_network, two_level=two_level, refinement=refinement)
        x, out = self._solve_once(b, tol, maxiter, **kw)
        out["restarts"] = 0
        if restarts == 0 or out["converged"] or not out["finite"]:
            return x, out
        import torch

        op = self.op
        keep = torch.as_tensor(~op.prescribed_mask, device=op.device)
        b = torch.where(keep, op._vec(b), 0.0)  # the solve's right-hand side: its free rows
        bn = float(torch.linalg.norm(b))
        budget = (maxiter if maxiter is not None else 10 * int(op.info["n_free"])) - out["iterations"]
        rel = out["relative_residual"]
        for _ in range(restarts):
            if budget <= 0 or rel <= tol:
                break
            r = b - op.apply(x)
            rn = float(torch.linalg.norm(r))
            dx, o = self._solve_once(r, min(0.5, 0.5 * tol * bn / rn), budget, **kw)
            budget -= o["iterations"]
            cand = x + dx
            rc = float(torch.linalg.norm(b - op.apply(cand)))
            out["iterations"] += o["iterations"]
            out["learned_iterations"] += o["learned_iterations"]
            out["seconds"] += o["seconds"]
            out["restarts"] += 1
            if not o["finite"] or rc >= rn:  # the correction did not help: keep x
                break
            x, rel = cand, rc / bn
            out["residual"], out["relative_residual"] = rc, rel
        out["converged"] = int(rel <= tol)
        return x, out

    def _solve_once(self, b, tol, maxiter, stall, depth, mixed, inner_tol, check_every, use_network, two_level,
                    refinement):
        if two_level not in (False, True, "multiplicative", "additive"):
            raise ValueError(f"two_level must be False, True, 'multiplicative' or 'additive', got {two_level!r}")
        additive = two_level == "additive"
        mult = two_level is True or two_level == "multiplicative"
        out_scale = self.out_scale * (self.additive_weight if additive else 1.0)
        if inner_tol is None:
            inner_tol = 1e-2 if refinement == "reliable" else 1e-4
        op = self.op
        b = op._vec(b)
        x = op._empty(op.n_dofs)
        o = op._opts(tol, 0.0, maxiter, "jacobi", check_every, inner_tol, 0)
        st = _lib.Stats()
        feats = self.features
        rc = self.lib.jxb_fcg_learned(op.handle, self.handle if use_network else None, _s(), _p(b), _p(x),
                                      _p(feats) if feats is not None else None, self.n_feat,
                                      float(self.in_scale), float(out_scale), int(stall), int(depth),
                                      (1 if mixed else 0) | (2 if mult else 0) | (8 if additive else 0)
                                      | (4 if refinement == "restart" else 0), ctypes.byref(o), ctypes.byref(st))
        _lib.check_solve(rc)
        out = {k: getattr(st, k) for k, _ in _lib.Stats._fields_}
        out["learned_iterations"] = out.pop("outer")
        return x, out

    # -- checkpoint / resume -------------------------------------------------------
    def save(self, path):
        np.savez(path, params=self.params.cpu().numpy(), in_scale=self.in_scale, out_scale=self.out_scale,
                 channels=np.asarray(self.channels), vec=self.vec, n_feat=self.n_feat,
                 history=np.asarray(self.history), additive_weight=self.additive_weight,
                 pool_input=int(self.pool_input))

    @classmethod
    def from_checkpoint(cls, op, path, features=None, inference_bf16=False):
        """A preconditioner with the network shape, weights and scales stored in
        ``path``; ``inference_bf16`` as :meth:`set_inference_bf16`."""
        d = np.load(path)
        pool = bool(int(d["pool_input"])) if "pool_input" in d.files else False
        lp = cls(op, features=features, channels=tuple(int(c) for c in d["channels"]), pool_input=pool)
        lp.load(path)
        if inference_bf16:
            lp.set_inference_bf16(True)
        return lp

    def load(self, path):
        import torch

        d = np.load(path)
        pool = bool(int(d["pool_input"])) if "pool_input" in d.files else False
        if (tuple(d["channels"]) != self.channels or int(d["vec"]) != self.vec or int(d["n_feat"]) != self.n_feat
                or pool != self.pool_input):
            raise ValueError("checkpoint does not match this network's shape")
        self.params.copy_(torch.as_tensor(d["params"], device=self.dev))
        self.in_scale = float(d["in_scale"])
        self.out_scale = float(d["out_scale"])
        self.additive_weight = float(d["additive_weight"]) if "additive_weight" in d.files else 1.0
        self.history = list(d["history"])


def default_channels(grid):
    """Channels per level for a control-point grid: enough levels that the
    coarsest grid has at most 8 points per direction (2..6 levels), 8 channels
    on the finest level growing to 48."""
    n = max(grid)
    levels = 2
    while levels < 6 and -(-n // 2 ** (levels - 1)) > 8:
        levels += 1
    return (8, 16, 24, 32, 48, 48)[:levels]


def time_network(n=99, channels=None, reps=10, in_ch=2, once=False, pool_input=False, bf16=False):
    """Device time (ms) of the network's forward and backward on an n^3 grid of
    random inputs, CUDA events on the current stream. ``once``: one forward and
    one backward after three warm-up forwards (for a profiler launch list).
    ``bf16``: forwards on the BF16 tensor-core convolutions (inference); the
    backward is then left out."""
    import torch

    lib = _lib.load()
    m = (n + 1) // 2 if pool_input else n
    channels = tuple(channels or default_channels((m, m, m)))
    h = ctypes.c_void_p()
    _lib.check(lib.jxb_cnn_create(in_ch, 1, len(channels), (ctypes.c_int32 * len(channels))(*channels), 1,
                                  ctypes.byref(h)))
    try:
        if pool_input:
            _lib.check(lib.jxb_cnn_set_input_pooling(h, 1))
        if bf16:
            _lib.check(lib.jxb_cnn_set_inference_bf16(h, 1))
        x = torch.randn(in_ch, n, n, n, device="cuda")
        out = torch.empty(1, n, n, n, device="cuda")
        g = torch.randn(1, n, n, n, device="cuda")
        fwd = lambda: _lib.check(lib.jxb_cnn_forward(h, _s(), n, n, n, _p(x), _p(out)))  # noqa: E731
        bwd = lambda: _lib.check(lib.jxb_cnn_backward(h, _s(), n, n, n, _p(x), _p(g)))  # noqa: E731
        for _ in range(3):
            fwd()
        if not once and not bf16:  # the first backward sizes its buffers: keep that out of the timed loop
            bwd()
        if once:
            fwd()
            if not bf16:
                bwd()
            torch.cuda.synchronize()
            return None
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        for _ in range(reps):
            fwd()
        e1.record()
        if not bf16:
            for _ in range(reps):
                fwd()
                bwd()
        e2.record()
        torch.cuda.synchronize()
        f = e0.elapsed_time(e1) / reps
        return {"grid": n, "channels": channels, "pool_input": bool(pool_input), "bf16": bool(bf16),
                "forward_ms": f, "backward_ms": None if bf16 else e1.elapsed_time(e2) / reps - f}
    finally:
        lib.jxb_cnn_destroy(h)


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="time the learned preconditioner's network on an n^3 grid")
    ap.add_argument("--grid", type=int, default=99)
    ap.add_argument("--channels", default=None, help="per-level channels, e.g. 8,16,24,32,48")
    ap.add_argument("--once", action="store_true", help="3 warm-up forwards, then one forward and one backward")
    ap.add_argument("--pool-input", action="store_true", help="run on the pooled input (half resolution)")
    ap.add_argument("--bf16", action="store_true", help="forwards on the BF16 tensor-core convolutions")
    a = ap.parse_args()
    ch = None if a.channels is None else [int(c) for c in a.channels.split(",")]
    print(json.dumps(time_network(a.grid, ch, once=a.once, pool_input=a.pool_input, bf16=a.bf16)))
