"""CPU restatement of the multigrid V-cycle preconditioner (test infrastructure).

TEST INFRASTRUCTURE ONLY: the tests use it to check the device V-cycle
(csrc/mg.cu, jaxiga_b200/multigrid.py) on the same inputs. Nothing in the
product package imports it.

The reference has no multigrid (its preconditioner is Jacobi,
src/jaxiga/solvers/linear.py:419-431). This module restates the device
algorithm with the oracle's assembled operators (iga_oracle.Assembled, the
restatement of the reference's element tangents and CSR scatter):

* levels: the hierarchy's spaces, each operator assembled on its free DOFs;
* transfers: the tensor product of the 1D knot-insertion matrices, with the
  NURBS weights around it (diag(1/w_f) P diag(w_c)), restricted to free rows
  and columns; the restriction is its transpose;
* smoothing: Chebyshev acceleration of Jacobi of a given degree on
  [1.1 lmax / range, 1.1 lmax], before and after the coarse correction;
* coarsest level: the exact inverse of its free block.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import iga_oracle as O


def transfer_matrix(Ps, w_fine, w_coarse, vec):
    P = sp.csr_matrix(Ps[0])
    for d in range(1, len(Ps)):
        P = sp.kron(sp.csr_matrix(Ps[d]), P)
    P = sp.diags(1.0 / w_fine) @ P @ sp.diags(w_coarse)
    return (sp.kron(P, sp.eye(vec)) if vec > 1 else P).tocsr()


class VCycle:
    """levels: list of (space, op, params, prescribed) finest first; transfers[l]: 1D
    matrices from level l+1 to l; lmax[l]: lmax of D^-1 K per level."""

    def __init__(self, levels, transfers, lmax, degree, smooth_range):
        self.A, self.P = [], []
        for S, op, params, pres in levels:
            self.A.append(O.Assembled(S, op, params, pres, np.zeros(len(pres)), need_full=False))
        for l, Ps in enumerate(transfers):
            Sf, Sc = levels[l][0], levels[l + 1][0]
            P = transfer_matrix(Ps, Sf.wgts, Sc.wgts, Sf.vec)
            self.P.append(P[self.A[l].free][:, self.A[l + 1].free].tocsr())
        self.lmax, self.degree, self.range = lmax, degree, smooth_range
        self.Kinv = np.linalg.inv(self.A[-1].K.toarray())

    def smooth(self, l, r):
        K, inv = self.A[l].K, O.jacobi_inverse(self.A[l].diag)
        lmax = 1.1 * self.lmax[l]
        lmin = lmax / self.range
        theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
        sigma = theta / delta
        rho = 1.0 / sigma
        e = inv * r / theta
        d = e.copy()
        for _ in range(1, self.degree):
            rho_new = 1.0 / (2.0 * sigma - rho)
            d = rho_new * rho * d + 2.0 * rho_new / delta * inv * (r - K @ e)
            e = e + d
            rho = rho_new
        return e

    def __call__(self, r, l=0):
        if l == len(self.A) - 1:
            return self.Kinv @ r
        K = self.A[l].K
        z = self.smooth(l, r)
        z = z + self.P[l] @ self(self.P[l].T @ (r - K @ z), l + 1)
        return z + self.smooth(l, r - K @ z)
