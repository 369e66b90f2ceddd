"""Device Jacobi-PCG on assembled CSR matrices: the B200 ``DeviceCG``.

The reference's staggered phase-field solver solves its two subproblems by
Jacobi-PCG on assembled CSR matrices, kept on the device so that no sweep
moves the matrix across the bus (``DeviceCG``,
src/jaxiga/solvers/phase_field.py:305-390). This class keeps its interface --
``solve(data, b)`` warm-started from the previous solution, ``relative_residual``,
``calls``/``iterations``/``failures``, ``report`` and ``release`` -- with the
pattern uploaded once and the solve in ``jxb_csr_pcg``. Unlike jax's CG it
knows its iteration count, so ``iterations`` is filled in.
"""

from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _lib


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@dataclasses.dataclass(frozen=True)
class CSRPattern:
    """Row pointers and column indices of a square sparse matrix (solvers/linear.py:38-68)."""

    indptr: np.ndarray
    column_indices: np.ndarray
    shape: tuple

    @classmethod
    def from_scipy(cls, A):
        A = A.tocsr()
        A.sort_indices()
        return cls(np.asarray(A.indptr, np.int64), np.asarray(A.indices, np.int32), tuple(A.shape))


class DeviceCG:
    """Jacobi-PCG on a fixed CSR pattern, warm-started across calls."""

    on_device = True

    def __init__(self, pattern, tol=1e-9, maxiter=5000, check_every=16):
        import torch

        self.lib = _lib.load()
        n = int(pattern.shape[0])
        if pattern.shape[0] != pattern.shape[1]:
            raise ValueError("DeviceCG needs a square matrix")
        indptr = np.ascontiguousarray(pattern.indptr, dtype=np.int64)
        cols = np.ascontiguousarray(pattern.column_indices, dtype=np.int32)
        h = ctypes.c_void_p()
        _lib.check(self.lib.jxb_csr_create(n, indptr.ctypes.data_as(_lib.c_int64_p),
                                           cols.ctypes.data_as(_lib.c_int32_p), ctypes.byref(h)))
        self.handle, self.n, self.nnz = h, n, int(indptr[-1])
        self.shape, self.tol, self.maxiter, self.check_every = (n, n), float(tol), int(maxiter), int(check_every)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.x0 = None
        self.calls, self.iterations, self.failures = 0, 0, 0
        self.last_stats = None

    def _dev(self, a, n):
        import torch

        t = torch.as_tensor(np.asarray(a) if not isinstance(a, torch.Tensor) else a, dtype=torch.float64,
                            device=self.device).contiguous()
        if t.numel() != n:
            raise ValueError(f"expected {n} values, got {t.numel()}")
        return t

    def solve(self, data, b):
        """x with A x = b from the previous solution (0 the first time)."""
        import torch

        self.calls += 1
        data, b = self._dev(data, self.nnz), self._dev(b, self.n)
        x = self.x0.clone() if self.x0 is not None else torch.zeros(self.n, dtype=torch.float64, device=self.device)
        o = _lib.SolveOpts()
        o.tol, o.atol, o.maxiter, o.preconditioner, o.check_every = self.tol, 0.0, self.maxiter, 1, self.check_every
        st = _lib.Stats()
        rc = self.lib.jxb_csr_pcg(self.handle, _stream(), _dptr(data), _dptr(b), _dptr(x), ctypes.byref(o),
                                  ctypes.byref(st))
        _lib.check_solve(rc)
        self.last_stats = {k: getattr(st, k) for k, _ in _lib.Stats._fields_}
        self.iterations += int(st.iterations)
        if not st.converged:  # reported, not fatal: the best iterate comes back
            self.failures += 1
        self.x0 = x
        return x

    def matvec(self, data, x):
        import torch

        y = torch.empty(self.n, dtype=torch.float64, device=self.device)
        # the device copies must stay referenced until the kernel has run: a
        # temporary freed after _dptr would hand its memory to the next one
        d, xv = self._dev(data, self.nnz), self._dev(x, self.n)
        _lib.check(self.lib.jxb_csr_matvec(self.handle, _stream(), _dptr(d), _dptr(xv), _dptr(y)))
        return y

    def relative_residual(self, data, b, x):
        """|A x - b| / |b|, computed on the device."""
        import torch

        b = self._dev(b, self.n)
        r = self.matvec(data, x) - b
        nb = float(torch.linalg.norm(b))
        return float(torch.linalg.norm(r)) / (nb if nb > 0 else 1.0)

    def report(self):
        return (f"{self.calls} device CG solves, {self.iterations} iterations "
                f"({self.iterations / max(self.calls, 1):.0f} per solve)"
                + (f", {self.failures} did not converge" if self.failures else ""))

    def release(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.jxb_csr_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
