"""Device operator of Poisson and linear-elasticity problems on truncated
hierarchical spaces.

A ``HierarchicalSpace`` (hierarchical.py) has elements with different numbers
of basis functions, so the tensor-product brick kernels do not apply. Its plan
(``jxb_thb_create``, csrc/thb.cu) runs K.u element by element through each
element's extraction operator, and hooks into the same entry points, so
``apply``, ``diag``, ``load``, ``dot`` and ``pcg`` are the single-patch
``Operator``'s.

The per-point data the device reads is made here once per operator: for every
leaf element the Bernstein form of the geometry (the element's homogeneous
control points pushed through its extraction operator), the Jacobian, its
determinant and inverse at the Gauss points of [-1, 1]^dim, the rational
weight function W and its gradient, and from them the metric M = a w L^T L of
the channels (numerator value, reference gradient) with L = J^-T (1/W)
[-grad W / W | I] -- the quotient rule of src/jaxiga/space/evaluation.py:95-172
folded into the operator, as the tensor kernels do. For elasticity the device
takes J^-1, w |J|, 1/W and grad W / W per point and forms the isotropic stress
(src/jaxiga/forms/library.py:174-181, materials.py:53-112) itself.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .hierarchical import HierarchicalSpace
from .space import bernstein_basis, gauss_1d


def _bernstein_deriv(u, p):
    """d/du of the Bernstein polynomials on [-1, 1]: (p/2)(B^{p-1}_{k-1} - B^{p-1}_k)."""
    if p == 0:
        return np.zeros((len(u), 1))
    lo = bernstein_basis(u, p - 1)
    d = np.zeros((len(u), p + 1))
    d[:, 1:] += lo
    d[:, :-1] -= lo
    return 0.5 * p * d


def reference_tables(dim, p):
    """Gauss points and weights of [-1, 1]^dim ((p+1)^dim, first direction
    fastest) and the (dim + 1, nq, nb) table of the Bernstein polynomials and
    their reference derivatives there (tensor order first direction fastest)."""
    u, w1 = gauss_1d(p + 1)
    B1, D1 = bernstein_basis(u, p), _bernstein_deriv(u, p)
    n1 = p + 1

    def tensor(fs):  # fs[d]: (n1 points, n1 functions) -> (n1^dim, n1^dim)
        out = fs[0]
        for d in range(1, dim):
            out = np.einsum("qa,rb->rqba", out.reshape(-1, n1 ** d), fs[d]).reshape(n1 ** (d + 1), n1 ** (d + 1))
        return out

    T = [tensor([B1] * dim)]
    for k in range(dim):
        T.append(tensor([D1 if d == k else B1 for d in range(dim)]))
    wq = w1
    for d in range(1, dim):
        wq = np.einsum("q,r->rq", wq, w1).ravel()
    return np.stack(T), wq


def _bernstein_deriv2(u, p):
    """d^2/du^2 of the Bernstein polynomials on [-1, 1]: (p/2)(dB^{p-1}_{k-1} - dB^{p-1}_k)."""
    if p < 2:
        return np.zeros((len(u), p + 1))
    lo = _bernstein_deriv(u, p - 1)
    d = np.zeros((len(u), p + 1))
    d[:, 1:] += lo
    d[:, :-1] -= lo
    return 0.5 * p * d


def gauss_points(dim, p):
    """The (p+1)^dim Gauss points of [-1, 1]^dim, first direction fastest, and their weights."""
    u, _ = gauss_1d(p + 1)
    pts = np.stack([g.ravel(order="F") for g in np.meshgrid(*([u] * dim), indexing="ij")], -1)
    return pts, reference_tables(dim, p)[1]


def tables_at(pts, p, order=1):
    """(dim + 1, n_pts, nb) table of the tensor Bernstein polynomials of degree
    ``p`` and their reference derivatives at points ``pts`` (n_pts, dim) of
    [-1, 1]^dim, functions first direction fastest (the order of
    ``reference_tables``); ``order=2`` appends the second derivatives of the
    pairs (a, b), a <= b, in row order (11, 12, 22 in 2D)."""
    pts = np.asarray(pts, dtype=float)
    dim = pts.shape[1]
    B1 = [bernstein_basis(pts[:, d], p) for d in range(dim)]
    D1 = [_bernstein_deriv(pts[:, d], p) for d in range(dim)]

    def tensor(fs):
        out = fs[0]
        for d in range(1, dim):
            out = np.einsum("qa,qb->qba", out, fs[d]).reshape(len(pts), -1)
        return out

    T = [tensor(B1)] + [tensor([D1[d] if d == k else B1[d] for d in range(dim)]) for k in range(dim)]
    if order >= 2:
        D2 = [_bernstein_deriv2(pts[:, d], p) for d in range(dim)]
        for a in range(dim):
            for b in range(a, dim):
                T.append(tensor([(D2[d] if a == b else D1[d]) if d in (a, b) else B1[d] for d in range(dim)]))
    return np.stack(T)


def _bernstein_geometry(space, elems, T):
    """Geometry of the elements ``elems`` at the points of table ``T``: x
    (e, q, dim), J (e, q, i, a) = d x_i / d xi_a in reference coordinates, the
    weight function W (e, q) and its reference gradient (e, q, a), from the
    Bernstein form of the homogeneous control net (each element's extraction
    rows applied to its functions' (w P, w))."""
    dim = space.dim
    hom = np.concatenate([space.cpts * space.wgts[:, None], space.wgts[:, None]], 1)
    hom = np.concatenate([hom, np.zeros((1, dim + 1))])  # the padding index reads zeros
    Pb = np.einsum("eia,eik->eak", space.extraction[elems], hom[space.elem_dofs[elems]])
    val = np.einsum("qa,eak->eqk", T[0], Pb)
    grd = np.einsum("cqa,eak->ecqk", T[1:], Pb)  # (e, dir, q, k)
    W = val[..., -1]
    x = val[..., :-1] / W[..., None]
    dW = grd[..., -1]  # (e, dir, q)
    dx = (grd[..., :-1] - x[:, None] * dW[..., None]) / W[:, None, :, None]  # (e, dir a, q, i) = d x_i / d xi_a
    return x, np.moveaxis(dx, 1, -1), W, np.moveaxis(dW, 1, -1)


def point_data(space: HierarchicalSpace, a0=1.0, chunk=4096, op="poisson"):
    """(factors (n_e, nq, nf), w / W (n_e, nq), x (n_e, nq, dim), w (n_e, nq))
    of every leaf element's Gauss points; ``a0`` scalar or (n_e, nq).

    Poisson factors: the channel metric a w L^T L, packed upper triangle row by
    row (nf = (dim+1)(dim+2)/2). Elasticity factors: J^-1 in reference
    coordinates ([a][k] = d xi_a / d x_k), w |J|, 1/W, grad W / W
    (nf = dim^2 + 2 + dim)."""
    dim, p = space.dim, space.degree[0]
    if space.dim_phys != dim:
        raise NotImplementedError("hierarchical operators need the physical and parametric dimensions equal")
    T, gw = reference_tables(dim, p)
    ne, nq = space.n_elems, len(gw)
    el = op == "elasticity"
    nf = dim * dim + 2 + dim if el else (dim + 1) * (dim + 2) // 2
    fac = np.zeros((ne, nq, nf))
    wqW = np.zeros((ne, nq))
    X = np.zeros((ne, nq, dim))
    W8 = np.zeros((ne, nq))
    iu = np.triu_indices(dim + 1)
    for lo in range(0, ne, chunk):
        sl = slice(lo, min(lo + chunk, ne))
        x, J, W, dWq = _bernstein_geometry(space, sl, T)
        det = np.linalg.det(J)
        Ji = np.linalg.inv(J)       # (e, q, a, k) = (J^-1)[a][k]
        w = gw[None, :] * np.abs(det)
        a = a0 if np.ndim(a0) == 0 else np.asarray(a0, dtype=float).reshape(ne, nq)[sl]
        L = np.zeros(J.shape[:2] + (dim, dim + 1))
        iW = 1.0 / W
        for k in range(dim):
            L[..., k, 0] = -np.einsum("eqa,eqa->eq", Ji[..., :, k], dWq) * iW * iW
            for c in range(dim):
                L[..., k, 1 + c] = Ji[..., c, k] * iW
        if el:
            fac[sl] = np.concatenate([Ji.reshape(Ji.shape[:2] + (dim * dim,)), w[..., None], iW[..., None],
                                      dWq * iW[..., None]], axis=-1)
        else:
            M = (a * w)[..., None, None] * np.einsum("eqkr,eqks->eqrs", L, L)
            fac[sl] = M[..., iu[0], iu[1]]
        wqW[sl] = w * iW
        X[sl] = x
        W8[sl] = w
    return fac, wqW, X, W8


def _create_plan(lib, space, elems, T, fac, wq, op, lam=0.0, mu=0.0, prescribed=None):
    """``jxb_thb_create`` over the elements ``elems`` of ``space`` with the point
    table ``T`` ((dim + 1, (p+1)^dim, nb)), per-point factors and weights w / W."""
    keep = [np.ascontiguousarray(space.elem_dofs[elems], dtype=np.int64),
            np.ascontiguousarray(space.extraction[elems], dtype=np.float64),
            np.ascontiguousarray(space.wgts, dtype=np.float64), np.ascontiguousarray(T, dtype=np.float64),
            np.ascontiguousarray(fac, dtype=np.float64), np.ascontiguousarray(wq, dtype=np.float64)]
    d = _lib.ThbDesc()
    d.dim, d.degree, d.n_local_max = space.dim, space.degree[0], space.n_local_max
    d.n_elem, d.n_scalar = len(keep[0]), space.n_scalar_basis
    d.op = {"poisson": _lib.OP_POISSON, "elasticity": _lib.OP_ELASTICITY, "plate": _lib.OP_PLATE}[op]
    d.lam, d.mu = lam, mu
    d.elem_dofs, d.extraction, d.wgts, d.tables, d.factors, d.wq = [k.ctypes.data for k in keep]
    pm = None
    if prescribed is not None:
        pm = np.ascontiguousarray(np.asarray(prescribed).astype(np.uint8))
        d.prescribed = pm.ctypes.data
    h = ctypes.c_void_p()
    _lib.check(lib.jxb_thb_create(ctypes.byref(d), ctypes.byref(h)))
    return h


def plate_point_data(space: HierarchicalSpace, E, nu, t, chunk=4096):
    """(factors (n_e, nq, 21), w / W, x, w) of the Kirchhoff plate
    (library.py:68-143) at every leaf element's Gauss points: per point the
    metric w L^T D L of the six channels g = (n, n_1, n_2, n_11, n_12, n_22) of
    the rational numerator n = sum_i w_i u_i N_i in reference coordinates, L
    the linear map from g to the curvatures -(R_xx, R_yy, 2 R_xy), D the
    bending stiffness E t^3 / (12 (1 - nu^2)) [[1, nu, 0], [nu, 1, 0], [0, 0,
    (1 - nu) / 2]]. L is the second-order quotient rule of R = n / W followed
    by the push-forward of second derivatives through the geometry's first
    and second derivatives (evaluation.py:95-172)."""
    if space.dim != 2 or space.vec != 1 or space.dim_phys != 2:
        raise NotImplementedError("the Kirchhoff plate runs on 2D scalar spaces")
    p = space.degree[0]
    pts, gw = gauss_points(2, p)
    T = tables_at(pts, p, order=2)  # (6, nq, nb)
    D = E * t**3 / (12.0 * (1.0 - nu**2)) * np.array([[1.0, nu, 0.0], [nu, 1.0, 0.0], [0.0, 0.0, (1.0 - nu) / 2.0]])
    pairs = [(0, 0), (0, 1), (1, 1)]
    hom = np.concatenate([space.cpts * space.wgts[:, None], space.wgts[:, None]], 1)
    hom = np.concatenate([hom, np.zeros((1, 3))])
    ne, nq = space.n_elems, len(gw)
    fac = np.zeros((ne, nq, 21))
    wqW, X, W8 = np.zeros((ne, nq)), np.zeros((ne, nq, 2)), np.zeros((ne, nq))
    iu = np.triu_indices(6)
    for lo in range(0, ne, chunk):
        sl = slice(lo, min(lo + chunk, ne))
        Pb = np.einsum("eia,eik->eak", space.extraction[sl], hom[space.elem_dofs[sl]])
        ch = np.einsum("cqa,eak->eqck", T, Pb)     # (e, q, channel, (wx, wy, w))
        W = ch[:, :, 0, 2]
        x = ch[:, :, 0, :2] / W[..., None]
        Wa = ch[:, :, 1:3, 2]                       # (e, q, a)
        xa = (ch[:, :, 1:3, :2] - Wa[..., None] * x[:, :, None]) / W[..., None, None]  # (e, q, a, i)
        xab = np.stack([(ch[:, :, 3 + k, :2] - xa[:, :, a] * Wa[..., b, None] - xa[:, :, b] * Wa[..., a, None]
                         - x * ch[:, :, 3 + k, 2, None]) / W[..., None] for k, (a, b) in enumerate(pairs)], 2)
        e_, q_ = W.shape
        iW = 1.0 / W
        dR = np.zeros((e_, q_, 2, 6))   # reference first derivatives of R in the channels
        d2R = np.zeros((e_, q_, 3, 6))  # reference second derivatives
        for a in range(2):
            dR[..., a, 0] = -Wa[..., a] * iW**2
            dR[..., a, 1 + a] = iW
        for k, (a, b) in enumerate(pairs):
            d2R[..., k, 3 + k] = iW
            d2R[..., k, 1 + a] -= Wa[..., b] * iW**2
            d2R[..., k, 1 + b] -= Wa[..., a] * iW**2
            d2R[..., k, 0] = -ch[:, :, 3 + k, 2] * iW**2 + 2.0 * Wa[..., a] * Wa[..., b] * iW**3
        J = xa                                      # [a][i] = d x_i / d xi_a
        dRx = np.linalg.solve(J, dR)                # physical gradient channels
        Tm = np.zeros((e_, q_, 3, 3))
        for r, (a, b) in enumerate(pairs):
            for c, (i, j) in enumerate(pairs):
                Tm[..., r, c] = J[..., a, i] * J[..., b, j] + (J[..., a, j] * J[..., b, i] if i != j else 0.0)
        d2Rx = np.linalg.solve(Tm, d2R - np.einsum("eqki,eqin->eqkn", xab, dRx))  # (xx, xy, yy)
        L = -np.stack([d2Rx[..., 0, :], d2Rx[..., 2, :], 2.0 * d2Rx[..., 1, :]], axis=2)
        w = gw[None, :] * np.abs(np.linalg.det(J))
        M = w[..., None, None] * np.einsum("eqsc,st,eqtd->eqcd", L, D, L)
        fac[sl] = M[..., iu[0], iu[1]]
        wqW[sl], X[sl], W8[sl] = w * iW, x, w
    return fac, wqW, X, W8, T


class ThbOperator:
    """Device Poisson (coef (a0,)) or linear-elasticity (coef (E, nu), vec = dim)
    operator on a HierarchicalSpace (``jxb_thb_create``): apply, diagonal,
    load, dot and Jacobi-PCG on the hierarchical DOFs."""

    def __init__(self, space, op="poisson", coef=(1.0,), prescribed=None, coef_qp=None, want_f32=False,
                 plane_strain=False):
        import torch

        if not ((op == "poisson" and space.vec == 1) or (op == "elasticity" and space.vec == space.dim)
                or (op == "plate" and space.vec == 1 and space.dim == 2)):
            raise NotImplementedError("hierarchical spaces run the Poisson (vec = 1), linear elasticity "
                                      "(vec = dim) and 2D Kirchhoff plate operators")
        if op == "plate" and coef_qp is not None:
            raise NotImplementedError("the plate on hierarchical spaces takes constant E, nu and t")
        if op == "elasticity" and coef_qp is not None:
            raise NotImplementedError("elasticity on hierarchical spaces takes constant E and nu")
        if want_f32:
            raise NotImplementedError("hierarchical operators run in FP64")
        if not torch.cuda.is_available():
            raise RuntimeError("the B200 solver needs a CUDA device; none is visible")
        self.lib = _lib.load()
        self.space, self.op, self.vec = space, op, space.vec
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.want_f32, self.tile = False, None
        if op == "plate":
            fac, wqW, X, W, T = plate_point_data(space, float(coef[0]), float(coef[1]), float(coef[2]))
        else:
            a0 = float(coef[0]) if coef_qp is None else np.asarray(coef_qp, dtype=float)
            fac, wqW, X, W = point_data(space, a0, op=op)
            T, _ = reference_tables(space.dim, space.degree[0])
        self.qp_x, self.qp_w = X, W
        self.prescribed_mask = (np.zeros(space.n_dofs, bool) if prescribed is None
                                else np.asarray(prescribed).astype(bool).copy())
        lam = mu = 0.0
        if op == "elasticity":  # the tensor plan's Lame pair (plane stress unless plane strain)
            E, nu = float(coef[0]), float(coef[1])
            mu = E / (2.0 * (1.0 + nu))
            lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)) if space.dim == 3 or plane_strain else E * nu / (1.0 - nu * nu)
        h = _create_plan(self.lib, space, slice(None), T, fac, wqW, op, lam, mu, self.prescribed_mask)
        self.handle = h
        info = _lib.Info()
        _lib.check(self.lib.jxb_plan_info(h, ctypes.byref(info)))
        self.info = {k: getattr(info, k) for k, _ in _lib.Info._fields_}
        self.n_dofs = info.n_dofs
        self.n_qp = info.n_qp
        self.nqe = len(T[0])

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.jxb_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ThbGeometry:
    """Gauss-point coordinates, weights and field interpolation on a
    HierarchicalSpace (the read-back of src/jaxiga/post/solution.py:39-50 at
    the interior Gauss set), from the host point data."""

    def __init__(self, space):
        import torch

        self.space = space
        _, _, self.x, self.w = point_data(space)
        T, _ = reference_tables(space.dim, space.degree[0])
        self.B = T[0]
        self.device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else None

    def qp_coords(self):
        import torch

        return torch.as_tensor(self.x)

    def qp_weights(self):
        import torch

        return torch.as_tensor(self.w)

    def interpolate(self, coef):
        """u(x_q) = sum_i u_i R_i(x_q) per element, (n_e, nq, ncomp)."""
        import torch

        s = self.space
        c = np.asarray(coef.cpu().numpy() if hasattr(coef, "cpu") else coef, dtype=float).reshape(s.n_scalar_basis, -1)
        c = np.concatenate([c, np.zeros((1, c.shape[1]))])
        w = np.concatenate([s.wgts, np.zeros(1)])
        N = np.einsum("eia,qa->eqi", s.extraction, self.B)  # B-spline values of each element's functions
        M = N * w[s.elem_dofs][:, None, :]
        Wq = M.sum(-1)
        return torch.as_tensor(np.einsum("eqi,eic->eqc", M, c[s.elem_dofs]) / Wq[..., None])

    def interpolate_grad(self, coef):
        """Physical gradients of a control-point field at the Gauss points,
        (n_e, nq, ncomp, dim): the quotient rule of R_i = w_i N_i / W, mapped by
        J^-T (evaluation.py:95-152)."""
        import torch

        s = self.space
        dim = s.dim
        c = np.asarray(coef.cpu().numpy() if hasattr(coef, "cpu") else coef, dtype=float).reshape(s.n_scalar_basis, -1)
        c = np.concatenate([c, np.zeros((1, c.shape[1]))])
        w = np.concatenate([s.wgts, np.zeros(1)])
        T, _ = reference_tables(dim, s.degree[0])
        wl = w[s.elem_dofs]                                               # (e, i)
        M = np.einsum("eia,qa->eqi", s.extraction, T[0]) * wl[:, None]    # w_i N_i
        dM = np.einsum("eia,dqa->edqi", s.extraction, T[1:]) * wl[:, None, None]
        W = M.sum(-1)
        dW = dM.sum(-1)                                                   # (e, d, q)
        cl = c[s.elem_dofs]                                               # (e, i, ncomp)
        num = np.einsum("eqi,eic->eqc", M, cl)
        dnum = np.einsum("edqi,eic->edqc", dM, cl)
        gref = (dnum - num[:, None] * (dW / W[:, None])[..., None]) / W[:, None, :, None]  # (e, d, q, c)
        hom = np.concatenate([s.cpts * s.wgts[:, None], s.wgts[:, None]], 1)
        hom = np.concatenate([hom, np.zeros((1, dim + 1))])
        Pb = np.einsum("eia,eik->eak", s.extraction, hom[s.elem_dofs])
        val = np.einsum("qa,eak->eqk", T[0], Pb)
        grd = np.einsum("cqa,eak->ecqk", T[1:], Pb)
        x = val[..., :-1] / val[..., -1:]
        J = np.moveaxis((grd[..., :-1] - x[:, None] * grd[..., -1:]) / val[:, None, :, -1:], 1, -1)  # (e, q, i, a)
        Ji = np.linalg.inv(J)                                             # (e, q, a, k)
        # grad_x u_c[k] = sum_a Ji[a][k] d u_c / d xi_a
        return torch.as_tensor(np.einsum("eqak,eaqc->eqck", Ji, gref))

    def eval_points(self, elems, ref, coef=None, val=True, grad=False, x=False, jac=False):
        """Values, physical gradients of a control-point field, coordinates and
        |det J| (reference coordinates) at points given by element indices (n,)
        and reference coordinates (n, dim) in [-1, 1]^dim; the interface of the
        tensor ``Operator.eval_points`` (evaluation.py:305-467)."""
        import torch

        s = self.space
        dim = s.dim
        e = np.asarray(elems, dtype=np.int64).reshape(-1)
        r = np.asarray(ref, dtype=float).reshape(len(e), dim)
        if coef is None and (val or grad):
            raise ValueError("values and gradients need a coefficient field")
        T = tables_at(r, s.degree[0])                                      # (dim + 1, n, nb): row k is point k
        hom = np.concatenate([s.cpts * s.wgts[:, None], s.wgts[:, None]], 1)
        hom = np.concatenate([hom, np.zeros((1, dim + 1))])
        C, d = s.extraction[e], s.elem_dofs[e]
        geo = np.einsum("cka,kia,kij->kcj", T, C, hom[d])                  # (n, channel, (w x, w))
        W, Wa = geo[:, 0, dim], geo[:, 1:, dim]
        xp = geo[:, 0, :dim] / W[:, None]
        J = (geo[:, 1:, :dim] - Wa[..., None] * xp[:, None]) / W[:, None, None]  # [a][i]
        out = {}
        if coef is not None:
            c = np.asarray(coef.cpu().numpy() if hasattr(coef, "cpu") else coef, dtype=float)
            c = c.reshape(s.n_scalar_basis, -1)
            cw = np.concatenate([c * s.wgts[:, None], np.zeros((1, c.shape[1]))])
            num = np.einsum("cka,kia,kij->kcj", T, C, cw[d])                # (n, channel, ncomp)
            f = num[:, 0] / W[:, None]
            if val:
                out["val"] = torch.as_tensor(f)
            if grad:
                fa = (num[:, 1:] - Wa[..., None] * f[:, None]) / W[:, None, None]  # (n, a, ncomp)
                out["grad"] = torch.as_tensor(np.moveaxis(np.linalg.solve(J, fa), 1, 2))
        if x:
            out["x"] = torch.as_tensor(xp)
        if jac:
            out["jac"] = torch.as_tensor(np.abs(np.linalg.det(J)))
        return out

    def close(self):
        pass


def side_points(space, elems, code, pts, wref):
    """Boundary data of side ``code`` (2 direction + end) of the elements
    ``elems`` at reference points ``pts`` (nq, dim) with weights ``wref``: x
    (e, q, dim), the outward unit normal grad xi_d / |grad xi_d| signed by the
    end, the surface weight wref |tangent| (2D) or wref |t1 x t2| (3D) in
    reference coordinates, W, and the point table
    (src/jaxiga/space/evaluation.py:174-193, 432-455)."""
    dim = space.dim
    T = tables_at(pts, space.degree[0])
    x, J, W, _ = _bernstein_geometry(space, np.asarray(elems), T)
    direction, end = divmod(int(code), 2)
    nrm = np.linalg.inv(J)[:, :, direction, :]
    nrm = nrm / np.linalg.norm(nrm, axis=-1, keepdims=True) * (1.0 if end == 1 else -1.0)
    tang = [a for a in range(dim) if a != direction]
    if dim == 2:
        sj = np.linalg.norm(J[..., tang[0]], axis=-1)
    else:
        sj = np.linalg.norm(np.cross(J[..., tang[0]], J[..., tang[1]]), axis=-1)
    return x, nrm, np.asarray(wref, dtype=float)[None, :] * sj, W, T


def side_centres(space, elems, sides):
    """Physical centre of the side each leaf element presents (problem.py:364-381)."""
    elems, sides = np.asarray(elems, dtype=np.int64), np.asarray(sides, dtype=np.int64)
    out = np.zeros((len(elems), space.dim))
    for code in np.unique(sides):
        sel = np.flatnonzero(sides == code)
        direction, end = divmod(int(code), 2)
        ref = np.zeros((1, space.dim))
        ref[0, direction] = -1.0 if end == 0 else 1.0
        out[sel] = _bernstein_geometry(space, elems[sel], tables_at(ref, space.degree[0]))[0][:, 0]
    return out


def neumann_load(op, problem, params, F):
    """F plus the loads F_i,c = sum_q w t_c(x, n) R_i of every Neumann condition
    of ``problem`` on a HierarchicalSpace (methods/_common.py:312-318).

    The faces of one side code share their reference points, so each code's
    faces become a plan of their own whose points are the face Gauss points
    (zero-padded to the plan's (p+1)^dim rows: padded points have zero table
    rows and zero weight): ``jxb_load`` integrates and the plan's fixed-order
    combine scatters them, as it does the volume load."""
    import torch

    from .neumann import _call_traction, resolve_set
    from .pointset import boundary_gauss

    space = problem.space
    dim, vec, p = space.dim, space.vec, space.degree[0]
    nb = (p + 1) ** dim
    kind = "elasticity" if vec > 1 else "poisson"
    nf = dim * dim + 2 + dim if vec > 1 else (dim + 1) * (dim + 2) // 2
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for bc in problem.neumann:
        ps = boundary_gauss(space, resolve_set(space, bc.where), problem.quadrature)
        sides = np.asarray(ps.sides, dtype=np.int64)
        for code in np.unique(sides):
            sel = np.flatnonzero(sides == code)
            elems = np.asarray(ps.elems, dtype=np.int64)[sel]
            x, nrm, w, W, T = side_points(space, elems, code, ps.ref[sel[0]], ps.weights[sel[0]])
            ne, nq = w.shape
            if nq > nb:
                raise NotImplementedError("boundary rules of more than (p+1)^(dim-1) points on hierarchical spaces")
            t = _call_traction(bc.value, x.reshape(-1, dim), nrm.reshape(-1, dim), params, vec)
            Tp = np.zeros((dim + 1, nb, nb))
            Tp[:, :nq] = T
            wq = np.zeros((ne, nb))
            wq[:, :nq] = w / W
            fq = np.zeros((ne, nb, vec))
            fq[:, :nq] = t.reshape(ne, nq, vec)
            h = _create_plan(op.lib, space, elems, Tp, np.zeros((ne, nb, nf)), wq, kind)
            try:
                f_dev = torch.as_tensor(fq.reshape(-1), device=op.device)
                Fs = torch.empty(space.n_dofs, dtype=torch.float64, device=op.device)
                _lib.check(op.lib.jxb_load(h, stream, ctypes.c_void_p(f_dev.data_ptr()),
                                           ctypes.c_void_p(Fs.data_ptr())))
                F += Fs
                torch.cuda.current_stream().synchronize()
            finally:
                op.lib.jxb_plan_destroy(h)
    return F


def _bind_operator_methods():
    from .operator import Operator

    for name in ("_vec", "_empty", "apply", "diag", "load", "dot", "_opts", "pcg"):
        setattr(ThbOperator, name, getattr(Operator, name))


_bind_operator_methods()
