"""CPU oracle for the nonlinear Galerkin path: compressible neo-Hookean solid.

TEST INFRASTRUCTURE ONLY. The tests call it to produce the answers the CUDA
path must reproduce; nothing in the product package imports it.

The reference defines the solid by its stored energy density
(src/jaxiga/forms/library.py:206-225)

    W(F) = mu/2 (tr F^T F - d) - mu ln J + lambda/2 (ln J)^2,  F = I + grad u,

with (lambda, mu) from E and nu by forms/materials.py:75-79, and obtains the
residual (the energy's gradient, methods/_common.py:280-309 under jax.grad) and
the tangent (its Hessian, methods/galerkin.py:207-237) by differentiation. The
restatement writes both out,

    P(F)  = mu (F - F^-T) + lambda ln J F^-T
    dP    = mu dF + (mu - lambda ln J) F^-T dF^T F^-T + lambda (F^-T : dF) F^-T,

assembled element by element on the interior Gauss rule (basis evaluation of
iga_oracle.evaluate). Since jax's autodiff is not available here, the
restatement is pinned by finite differences: the residual against the energy
and the tangent against the residual (tests/test_hyper_oracle.py). Newton's
method with halving line search restates solvers/newton.py:27-135.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import iga_oracle as O


def lame(E, nu):
    """(lambda, mu), forms/materials.py:75-79."""
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


class NeoHookean:
    """Energy, residual and tangent of a neo-Hookean solid on one space."""

    def __init__(self, space, mu, lam):
        self.space, self.mu, self.lam = space, float(mu), float(lam)
        self.basis = O.evaluate(space, np.arange(space.n_elems))
        self.gd = space.expand(space.elem_dofs)  # (n_e, n_loc * d) interleaved

    def _F(self, u):
        d = self.space.dim
        ue = u[self.gd].reshape(self.gd.shape[0], -1, d)  # (e, n, c)
        G = np.einsum("enc,eqkn->eqck", ue, self.basis["dR"])  # du_c / dx_k
        return np.eye(d) + G

    def energy(self, u):
        F = self._F(u)
        d = F.shape[-1]
        J = np.linalg.det(F)
        lnJ = np.log(J)
        W = self.mu / 2 * (np.einsum("eqij,eqij->eq", F, F) - d) - self.mu * lnJ + self.lam / 2 * lnJ**2
        return float(np.sum(self.basis["w"] * W))

    def residual(self, u):
        """int P(F) : grad v over all DOFs."""
        F = self._F(u)
        FiT = np.linalg.inv(F).transpose(0, 1, 3, 2)
        lnJ = np.log(np.linalg.det(F))
        P = self.mu * (F - FiT) + self.lam * lnJ[..., None, None] * FiT
        re = np.einsum("eq,eqck,eqkn->enc", self.basis["w"], P, self.basis["dR"]).reshape(len(self.gd), -1)
        r = np.zeros(self.space.n_dofs)
        np.add.at(r, self.gd.ravel(), re.ravel())
        return r

    def tangent(self, u):
        """K(u) (CSR, all DOFs): the derivative of ``residual``."""
        F = self._F(u)
        d = F.shape[-1]
        FiT = np.linalg.inv(F).transpose(0, 1, 3, 2)
        lnJ = np.log(np.linalg.det(F))
        c = self.mu - self.lam * lnJ
        I = np.eye(d)
        # A[c,k,d,l] = dP_ck / dF_dl
        A = (self.mu * np.einsum("cd,kl->ckdl", I, I)[None, None]
             + c[..., None, None, None, None] * np.einsum("eqcl,eqdk->eqckdl", FiT, FiT)
             + self.lam * np.einsum("eqck,eqdl->eqckdl", FiT, FiT))
        dR, w = self.basis["dR"], self.basis["w"]
        Ke = np.einsum("eq,eqkn,eqckdl,eqlm->encmd", w, dR, A, dR)
        ne, nl = Ke.shape[0], Ke.shape[1] * d
        Ke = Ke.reshape(ne, nl, nl)
        rows = np.repeat(self.gd, nl, axis=1).ravel()
        cols = np.tile(self.gd, (1, nl)).ravel()
        K = sp.coo_matrix((Ke.ravel(), (rows, cols)), shape=(self.space.n_dofs,) * 2).tocsr()
        K.sum_duplicates()
        return K


def newton(model, prescribed, values, f_ext, tol=1e-8, max_steps=25, line_search=True):
    """solvers/newton.py:27-135 on the free DOFs, SuperLU tangent solves."""
    n = model.space.n_dofs
    free = np.setdiff1d(np.arange(n), prescribed)
    u = np.zeros(n)
    u[prescribed] = values

    def res(uu):
        return (model.residual(uu) - f_ext)[free]

    def norm_of(uu):
        return float(np.linalg.norm(res(uu)))

    r_norm = norm_of(u)
    hist = [r_norm]
    step, alpha = 0, 1.0
    while np.isfinite(r_norm) and r_norm > tol and step < max_steps and alpha > 0:
        r = res(u)
        K = model.tangent(u)[free][:, free].tocsc()
        du = np.zeros(n)
        du[free] = spla.spsolve(K, -r)
        alpha = 1.0
        trial = norm_of(u + du)
        k = 0
        while line_search and (not np.isfinite(trial) or trial >= r_norm) and k < 20:
            alpha *= 0.5
            trial = norm_of(u + alpha * du)
            k += 1
        if not (np.isfinite(trial) and trial < r_norm):
            alpha = 0.0
        if alpha > 0:
            u = u + alpha * du
            r_norm = trial
        step += 1
        hist.append(r_norm)
    return u, {"iterations": step, "residual": norm_of(u), "history": hist, "converged": norm_of(u) <= tol}
