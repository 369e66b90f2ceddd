"""A device operator for one linear Galerkin problem, backed by a libjxb plan.

``Operator`` owns a ``jxb_plan`` and exposes its entry points on CUDA torch
tensors (torch supplies device memory and the current stream; all arithmetic
happens in libjxb's kernels). It is what ``jaxiga_b200.solve`` drives, and is
usable directly by hosts that run their own Krylov loop.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _hptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class Operator:
    """K (with the Dirichlet partition) of one problem on one single-patch space.

    Parameters
    ----------
    space : FunctionSpace
    op : {"poisson", "elasticity", "plate", "hyperelastic"}
    coef : sequence of up to 4 floats -- a0 | (E, nu) | (E, nu, t) | (mu, lambda)
        ("hyperelastic": the compressible neo-Hookean tangent at the state set by
        ``state(u)``, u = 0 until then)
    prescribed : optional bool/uint8 array (n_dofs,), True on Dirichlet DOFs
    coef_qp : optional (n_elem, n_q^dim) per-point a0 for Poisson
    want_f32 : keep FP32 copies of the factors for mixed precision
    plane_strain : 2D elasticity flavour
    """

    OPS = {"poisson": _lib.OP_POISSON, "elasticity": _lib.OP_ELASTICITY, "plate": _lib.OP_PLATE,
           "hyperelastic": _lib.OP_HYPERELASTIC}

    def __init__(self, space, op="poisson", coef=(1.0,), prescribed=None, coef_qp=None,
                 want_f32=False, plane_strain=False, vec=None, tile=None):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("the B200 solver needs a CUDA device; none is visible")
        self.lib = _lib.load()
        self.space = space
        self.op = op
        self.vec = space.vec if vec is None else int(vec)
        self.device = torch.device("cuda", torch.cuda.current_device())
        p = space.degree[0]
        nodes, weights = np.polynomial.legendre.leggauss(p + 1)
        self._keep = []  # host arrays referenced by the descriptor
        d = _lib.Desc()
        d.dim = space.dim
        d.vec = self.vec
        d.degree = p
        d.n_quad = p + 1
        for k in range(3):
            d.n_cp[k] = space.n_cp[k] if k < space.dim else 1
            d.n_span[k] = space.n_span[k] if k < space.dim else 1
        for k in range(space.dim):
            first = np.ascontiguousarray(space.first[k], dtype=np.int32)
            lo = np.ascontiguousarray(space.span_lo[k], dtype=np.float64)
            hi = np.ascontiguousarray(space.span_hi[k], dtype=np.float64)
            ext = np.ascontiguousarray(space.ext1d[k], dtype=np.float64)
            self._keep += [first, lo, hi, ext]
            d.first[k] = _hptr(first, ctypes.c_int32)
            d.span_lo[k] = _hptr(lo, ctypes.c_double)
            d.span_hi[k] = _hptr(hi, ctypes.c_double)
            d.extraction[k] = _hptr(ext, ctypes.c_double)
        cpts = np.ascontiguousarray(space.cpts[:, : space.dim], dtype=np.float64)
        wgts = np.ascontiguousarray(space.wgts, dtype=np.float64)
        nodes = np.ascontiguousarray(nodes)
        weights = np.ascontiguousarray(weights)
        self._keep += [cpts, wgts, nodes, weights]
        d.cpts = _hptr(cpts, ctypes.c_double)
        d.wgts = _hptr(wgts, ctypes.c_double)
        d.gauss_nodes = _hptr(nodes, ctypes.c_double)
        d.gauss_weights = _hptr(weights, ctypes.c_double)
        d.op = self.OPS[op]
        coef = list(coef) + [0.0] * (4 - len(coef))
        for k in range(4):
            d.coef[k] = float(coef[k])
        d.plane_strain = 1 if plane_strain else 0
        if coef_qp is not None:
            cq = np.ascontiguousarray(np.asarray(coef_qp, dtype=np.float64).reshape(-1))
            if cq.size != space.n_elems * (p + 1) ** space.dim:
                raise ValueError(f"coef_qp has {cq.size} values, expected {space.n_elems * (p + 1) ** space.dim}")
            self._keep.append(cq)
            d.coef_qp = _hptr(cq, ctypes.c_double)
        if prescribed is not None:
            pm = np.ascontiguousarray(np.asarray(prescribed).astype(np.uint8))
            if pm.size != space.n_scalar_basis * self.vec:
                raise ValueError("prescribed mask must have n_dofs entries")
            self._keep.append(pm)
            d.prescribed = _hptr(pm, ctypes.c_uint8)
        self.prescribed_mask = (np.zeros(space.n_scalar_basis * self.vec, bool) if prescribed is None
                                else np.asarray(prescribed).astype(bool).copy())
        d.want_f32 = 1 if want_f32 else 0
        if tile is not None:
            d.tile[0], d.tile[1] = int(tile[0]), int(tile[1])
        self.tile = tuple(tile) if tile is not None else None
        handle = ctypes.c_void_p()
        _lib.check(self.lib.jxb_plan_create(ctypes.byref(d), ctypes.byref(handle)))
        self._keep = []
        self.handle = handle
        info = _lib.Info()
        _lib.check(self.lib.jxb_plan_info(handle, ctypes.byref(info)))
        self.info = {k: getattr(info, k) for k, _ in _lib.Info._fields_}
        self.n_dofs = info.n_dofs
        self.n_qp = info.n_qp
        self.nqe = (p + 1) ** space.dim
        self.want_f32 = bool(want_f32)

    # -- lifetime ------------------------------------------------------------
    def close(self):
        mg = getattr(self, "_multigrid", None)
        if mg is not None:  # its V-cycle holds this plan as its finest level
            mg.close()
            self._multigrid = None
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.jxb_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- helpers ---------------------------------------------------------------
    def _vec(self, x, dtype=None):
        import torch

        dtype = dtype or torch.float64
        t = torch.as_tensor(x, dtype=dtype, device=self.device).contiguous()
        if t.numel() != self.n_dofs:
            raise ValueError(f"vector has {t.numel()} entries, expected {self.n_dofs}")
        return t

    def _empty(self, n, dtype=None):
        import torch

        return torch.empty(n, dtype=dtype or torch.float64, device=self.device)

    # -- operator --------------------------------------------------------------
    def apply(self, x, masked=True, out=None):
        """y = K x (masked: on free DOFs only, the Krylov operator)."""
        x = self._vec(x)
        y = out if out is not None else self._empty(self.n_dofs)
        _lib.check(self.lib.jxb_apply(self.handle, _stream(), _dptr(x), _dptr(y), 1 if masked else 0))
        return y

    def apply_f32(self, x, out=None):
        import torch

        x = self._vec(x, torch.float32)
        y = out if out is not None else self._empty(self.n_dofs, torch.float32)
        _lib.check(self.lib.jxb_apply_f32(self.handle, _stream(), _dptr(x), _dptr(y)))
        return y

    def diag(self):
        d = self._empty(self.n_dofs)
        _lib.check(self.lib.jxb_diag(self.handle, _stream(), _dptr(d)))
        return d

    def state(self, u, energy=False):
        """Hyperelastic plans: set the state to the displacement ``u`` (all DOFs,
        Dirichlet values included) for the tangent and the residual; with
        ``energy`` return the stored energy sum_q w_q W(F_q) (host float)."""
        if self.op != "hyperelastic":
            raise ValueError("state() belongs to the hyperelastic operator")
        uv = self._vec(u)  # referenced until the launch is queued on the stream
        e = ctypes.c_double()
        _lib.check(self.lib.jxb_hyper_state(self.handle, _stream(), _dptr(uv),
                                            ctypes.byref(e) if energy else None))
        return e.value if energy else None

    def residual(self):
        """Hyperelastic plans: the internal forces int P(F) : grad v at the
        current state, over all DOFs (device tensor)."""
        if self.op != "hyperelastic":
            raise ValueError("residual() belongs to the hyperelastic operator")
        r = self._empty(self.n_dofs)
        _lib.check(self.lib.jxb_hyper_residual(self.handle, _stream(), _dptr(r)))
        return r

    def load(self, f_qp):
        """F = sum_q w f R (full length) for source values at the Gauss points."""
        import torch

        f = torch.as_tensor(f_qp, dtype=torch.float64, device=self.device).contiguous()
        if f.numel() != self.n_qp * self.vec:
            raise ValueError(f"source has {f.numel()} values, expected {self.n_qp * self.vec}")
        F = self._empty(self.n_dofs)
        _lib.check(self.lib.jxb_load(self.handle, _stream(), _dptr(f), _dptr(F)))
        return F

    def qp_coords(self):
        x = self._empty(self.n_qp * self.space.dim)
        _lib.check(self.lib.jxb_qp_coords(self.handle, _stream(), _dptr(x)))
        return x.view(self.space.n_elems, self.nqe, self.space.dim)

    def qp_weights(self):
        w = self._empty(self.n_qp)
        _lib.check(self.lib.jxb_qp_weights(self.handle, _stream(), _dptr(w)))
        return w.view(self.space.n_elems, self.nqe)

    def interpolate(self, coef):
        import torch

        c = torch.as_tensor(coef, dtype=torch.float64, device=self.device).contiguous()
        ncomp = c.numel() // self.space.n_scalar_basis
        if ncomp * self.space.n_scalar_basis != c.numel():
            raise ValueError("coefficient field must have n_scalar_basis * ncomp entries")
        out = self._empty(self.n_qp * ncomp)
        _lib.check(self.lib.jxb_interpolate(self.handle, _stream(), _dptr(c), ncomp, _dptr(out)))
        return out.view(self.space.n_elems, self.nqe, ncomp)

    def interpolate_grad(self, coef):
        """Physical gradients of a control-point field at the Gauss points,
        (n_elem, n_q, ncomp, dim)."""
        import torch

        c = torch.as_tensor(coef, dtype=torch.float64, device=self.device).contiguous()
        ncomp = c.numel() // self.space.n_scalar_basis
        if ncomp * self.space.n_scalar_basis != c.numel():
            raise ValueError("coefficient field must have n_scalar_basis * ncomp entries")
        out = self._empty(self.n_qp * ncomp * self.space.dim)
        _lib.check(self.lib.jxb_interpolate_grad(self.handle, _stream(), _dptr(c), ncomp, _dptr(out)))
        return out.view(self.space.n_elems, self.nqe, ncomp, self.space.dim)

    def eval_points(self, elems, ref, coef=None, val=True, grad=False, x=False, jac=False):
        """Evaluate at arbitrary points: element indices (n,) and reference
        coordinates (n, dim) in [-1, 1]^dim. Returns a dict with the requested
        "val" (n, ncomp), "grad" (n, ncomp, dim) of the control-point field
        ``coef``, physical coordinates "x" (n, dim) and "jac" (n) =
        |det J| prod(h/2)."""
        import torch

        dim = self.space.dim
        e = torch.as_tensor(np.asarray(elems, dtype=np.int64), device=self.device).contiguous()
        r = torch.as_tensor(np.asarray(ref, dtype=np.float64), device=self.device).contiguous()
        n = e.numel()
        if r.numel() != n * dim:
            raise ValueError(f"ref must be ({n}, {dim})")
        c, ncomp = None, 0
        if coef is not None:
            c = torch.as_tensor(coef, dtype=torch.float64, device=self.device).contiguous()
            ncomp = c.numel() // self.space.n_scalar_basis
            if ncomp * self.space.n_scalar_basis != c.numel():
                raise ValueError("coefficient field must have n_scalar_basis * ncomp entries")
        elif val or grad:
            raise ValueError("values and gradients need a coefficient field")
        out = {}
        if val:
            out["val"] = self._empty(max(n * ncomp, 1))
        if grad:
            out["grad"] = self._empty(max(n * ncomp * dim, 1))
        if x:
            out["x"] = self._empty(max(n * dim, 1))
        if jac:
            out["jac"] = self._empty(max(n, 1))
        ptr = lambda k: _dptr(out[k]) if k in out else None  # noqa: E731
        _lib.check(self.lib.jxb_eval_points(self.handle, _stream(), _dptr(c) if c is not None else None, ncomp, n,
                                            _dptr(e), _dptr(r), ptr("val"), ptr("grad"), ptr("x"), ptr("jac")))
        shapes = {"val": (n, ncomp), "grad": (n, ncomp, dim), "x": (n, dim), "jac": (n,)}
        return {k: v[: int(np.prod(shapes[k]))].view(*shapes[k]) for k, v in out.items()}

    def profile_apply(self, x, reps=20, f32=False):
        """Average device ms of one brick launch and one combine launch (CUDA events)."""
        import torch

        dt = torch.float32 if f32 else torch.float64
        x = self._vec(x, dt)
        y = self._empty(self.n_dofs, dt)
        ms = (ctypes.c_double * 2)()
        _lib.check(self.lib.jxb_profile_apply(self.handle, _stream(), _dptr(x), _dptr(y), int(reps),
                                              1 if f32 else 0, ms))
        return ms[0], ms[1]

    def dot(self, a, b):
        r = ctypes.c_double()
        a, b = self._vec(a), self._vec(b)  # referenced until the call returns (it synchronises)
        _lib.check(self.lib.jxb_dot(self.handle, _stream(), _dptr(a), _dptr(b), ctypes.byref(r)))
        return r.value

    # -- solves ---------------------------------------------------------------
    def _opts(self, tol, atol, maxiter, preconditioner, check_every, inner_tol, max_outer, restarts=0):
        o = _lib.SolveOpts()
        o.tol = float(tol)
        o.atol = float(atol)
        o.maxiter = int(maxiter or 0)
        o.preconditioner = 1 if preconditioner in ("jacobi", 1, True) else 0
        o.check_every = int(check_every)
        o.inner_tol = float(inner_tol)
        o.max_outer = int(max_outer)
        o.restarts = int(restarts)
        return o

    def pcg(self, b, tol=1e-12, atol=0.0, maxiter=None, preconditioner="jacobi", check_every=16, restarts=0,
            raise_on_nonfinite=False):
        """Jacobi-PCG from x = 0 (jax CG semantics); returns (x, stats dict).

        ``restarts`` > 0: when the FP64 true residual misses the tolerance after
        CG stopped, restart CG on it (at most that many times, sharing
        ``maxiter``), as the reference's CPU CG does; stats["outer"] counts them.
        """
        b = self._vec(b)
        x = self._empty(self.n_dofs)
        st = _lib.Stats()
        o = self._opts(tol, atol, maxiter, preconditioner, check_every, 0.0, 0, restarts)
        rc = self.lib.jxb_pcg(self.handle, _stream(), _dptr(b), _dptr(x), ctypes.byref(o), ctypes.byref(st))
        _lib.check_solve(rc, raise_on_nonfinite)
        return x, {k: getattr(st, k) for k, _ in _lib.Stats._fields_}

    def bicgstab(self, b, tol=1e-12, atol=0.0, maxiter=None, preconditioner="jacobi", check_every=16):
        """BiCGSTAB from x = 0 (jax semantics, Jacobi right preconditioning); returns (x, stats dict)."""
        b = self._vec(b)
        x = self._empty(self.n_dofs)
        st = _lib.Stats()
        o = self._opts(tol, atol, maxiter, preconditioner, check_every, 0.0, 0)
        rc = self.lib.jxb_bicgstab(self.handle, _stream(), _dptr(b), _dptr(x), ctypes.byref(o), ctypes.byref(st))
        _lib.check_solve(rc)
        return x, {k: getattr(st, k) for k, _ in _lib.Stats._fields_}

    def refine_solve(self, b, tol=1e-8, inner_tol=1e-4, maxiter=None, max_outer=40, check_every=16):
        """FP64 iterative refinement around FP32 Jacobi-PCG inner solves."""
        if not self.want_f32:
            raise ValueError("create the Operator with want_f32=True for mixed precision")
        b = self._vec(b)
        x = self._empty(self.n_dofs)
        st = _lib.Stats()
        o = self._opts(tol, 0.0, maxiter, "jacobi", check_every, inner_tol, max_outer)
        rc = self.lib.jxb_refine_solve(self.handle, _stream(), _dptr(b), _dptr(x), ctypes.byref(o), ctypes.byref(st))
        _lib.check_solve(rc)
        return x, {k: getattr(st, k) for k, _ in _lib.Stats._fields_}

    def mixed_pcg(self, b, tol=1e-8, delta=1e-2, maxiter=None, max_updates=1000, check_every=16):
        """FP32 Jacobi-PCG with reliable FP64 updates every ``delta`` of residual decrease."""
        if not self.want_f32:
            raise ValueError("create the Operator with want_f32=True for mixed precision")
        if not (0 < delta < 1):
            raise ValueError("delta must lie in (0, 1)")
        b = self._vec(b)
        x = self._empty(self.n_dofs)
        st = _lib.Stats()
        o = self._opts(tol, 0.0, maxiter, "jacobi", check_every, delta, max_updates)
        rc = self.lib.jxb_mixed_pcg(self.handle, _stream(), _dptr(b), _dptr(x), ctypes.byref(o), ctypes.byref(st))
        _lib.check_solve(rc)
        return x, {k: getattr(st, k) for k, _ in _lib.Stats._fields_}
