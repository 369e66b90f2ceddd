"""CPU oracle of the learned-preconditioner network (NumPy, FP64).

TEST INFRASTRUCTURE ONLY: the GPU network (libjxb's cnn kernels) is checked
against this restatement -- forward output and parameter gradients for a
given output gradient (masked mean-squared error, or any other loss). The
reference has no learned preconditioner (its only preconditioner is Jacobi,
src/jaxiga/solvers/linear.py:419-431), so this oracle restates the network
the way libjxb defines it: a U-Net with L levels and channels c[0..L-1],

    encoder, l = 0..L-2:  x -> c[l] relu; c[l] -> c[l] relu = s_l; x = pool(s_l)
    bottom (level L-1):   x -> c[L-1] relu; two more c[L-1] -> c[L-1] relu
    decoder, l = L-2..0:  y = up(y); m_l = 1x1 c[l+1] -> c[l] (y) + s_l;
                          y = c[l] -> c[l] relu (m_l)
    output:               c[0] -> 4 (linear; the first out_ch channels are used)

With input pooling the input is pooled once, the U-Net runs on the pooled
grid and its output is interpolated to the input grid: trilinear, fine point
X = 2c taking coarse c and odd X the mean of (X - 1) / 2 and (X + 1) / 2 (the
lower one alone past the end).

3x3x3 convolutions use zero padding, tap index k = dx + 3 dy + 9 dz; pooling
averages the existing children of a coarse voxel (odd sizes round up);
upsampling copies a coarse voxel to its children. Parameters are one flat
vector: per layer (in the order above) the weights [co][ci][k] then the
biases [co].
"""

from __future__ import annotations

import numpy as np

def layer_shapes(in_ch, channels):
    """(ci, co, k, relu) of every layer, in parameter order."""
    c = [int(v) for v in channels]
    n = len(c)
    out, prev = [], in_ch
    for lv in range(n - 1):
        out += [(prev, c[lv], 3, True), (c[lv], c[lv], 3, True)]
        prev = c[lv]
    out += [(prev, c[-1], 3, True), (c[-1], c[-1], 3, True), (c[-1], c[-1], 3, True)]
    for lv in range(n - 2, -1, -1):
        out += [(c[lv + 1], c[lv], 1, False), (c[lv], c[lv], 3, True)]
    out.append((c[0], 4, 3, False))
    return out


def unpack(params, in_ch, channels):
    out, off = [], 0
    for ci, co, k, relu in layer_shapes(in_ch, channels):
        nw = co * ci * k**3
        w = params[off: off + nw].reshape(co, ci, k, k, k)  # [co][ci][dz][dy][dx]
        off += nw
        b = params[off: off + co]
        off += co
        out.append((w, b, k, relu))
    assert off == len(params)
    return out


def conv(x, w, b):
    """x [ci, nz, ny, nx] -> [co, nz, ny, nx]."""
    co, ci, K = w.shape[0], w.shape[1], w.shape[2]
    R = K // 2
    xp = np.pad(x, ((0, 0), (R, R), (R, R), (R, R)))
    nz, ny, nx = x.shape[1:]
    y = np.broadcast_to(b[:, None, None, None], (co, nz, ny, nx)).astype(np.float64).copy()
    for dz in range(K):
        for dy in range(K):
            for dx in range(K):
                patch = xp[:, dz: dz + nz, dy: dy + ny, dx: dx + nx]
                y += np.einsum("oc,czyx->ozyx", w[:, :, dz, dy, dx], patch)
    return y


def conv_grads(x, w, g):
    """Gradients of sum(g * conv(x, w, b)) w.r.t. x, w, b."""
    co, ci, K = w.shape[0], w.shape[1], w.shape[2]
    R = K // 2
    xp = np.pad(x, ((0, 0), (R, R), (R, R), (R, R)))
    nz, ny, nx = x.shape[1:]
    gw = np.zeros_like(w)
    gxp = np.zeros_like(xp)
    for dz in range(K):
        for dy in range(K):
            for dx in range(K):
                patch = xp[:, dz: dz + nz, dy: dy + ny, dx: dx + nx]
                gw[:, :, dz, dy, dx] = np.einsum("ozyx,czyx->oc", g, patch)
                gxp[:, dz: dz + nz, dy: dy + ny, dx: dx + nx] += np.einsum("oc,ozyx->czyx", w[:, :, dz, dy, dx], g)
    gx = gxp[:, R: R + nz, R: R + ny, R: R + nx]
    return gx, gw, g.sum(axis=(1, 2, 3))


def half(shape):
    return tuple((n + 1) // 2 for n in shape)


def pool(x):
    c = x.shape[0]
    nz, ny, nx = x.shape[1:]
    cz, cy, cx = half((nz, ny, nx))
    s = np.zeros((c, cz, cy, cx))
    n = np.zeros((cz, cy, cx))
    for dz in range(2):
        for dy in range(2):
            for dx in range(2):
                sub = x[:, dz::2, dy::2, dx::2]
                s[:, : sub.shape[1], : sub.shape[2], : sub.shape[3]] += sub
                n[: sub.shape[1], : sub.shape[2], : sub.shape[3]] += 1
    return s / n


def pool_grad(gc, fine_shape):
    nz, ny, nx = fine_shape
    cz, cy, cx = gc.shape[1:]
    n = np.zeros((cz, cy, cx))
    for dz in range(2):
        for dy in range(2):
            for dx in range(2):
                n[: len(range(dz, nz, 2)), : len(range(dy, ny, 2)), : len(range(dx, nx, 2))] += 1
    g = gc / n
    return up(g, fine_shape)


def up(x, fine_shape):
    nz, ny, nx = fine_shape
    return x.repeat(2, 1).repeat(2, 2).repeat(2, 3)[:, :nz, :ny, :nx]


def up_grad(gf, coarse_shape):
    c = gf.shape[0]
    out = np.zeros((c,) + tuple(coarse_shape))
    for dz in range(2):
        for dy in range(2):
            for dx in range(2):
                sub = gf[:, dz::2, dy::2, dx::2]
                out[:, : sub.shape[1], : sub.shape[2], : sub.shape[3]] += sub
    return out


def lin_matrix(nf, nc):
    """Linear prolongation along one direction, (nf, nc)."""
    P = np.zeros((nf, nc))
    for X in range(nf):
        lo = X // 2
        if X % 2 == 0 or lo + 1 >= nc:
            P[X, lo] = 1.0
        else:
            P[X, lo] = P[X, lo + 1] = 0.5
    return P


def up_lin(x, fine_shape):
    Pz, Py, Px = (lin_matrix(f, c) for f, c in zip(fine_shape, x.shape[1:]))
    return np.einsum("Zz,Yy,Xx,czyx->cZYX", Pz, Py, Px, x)


def up_lin_grad(gf, coarse_shape):
    Pz, Py, Px = (lin_matrix(f, c) for f, c in zip(gf.shape[1:], coarse_shape))
    return np.einsum("Zz,Yy,Xx,cZYX->czyx", Pz, Py, Px, gf)


def forward(params, x, in_ch, channels, pool_input=False):
    """Returns (output [4, ...], cache)."""
    if pool_input:
        out, cache = forward(params, pool(x), in_ch, channels)
        return up_lin(out, x.shape[1:]), cache
    L = unpack(np.asarray(params, dtype=np.float64), in_ch, channels)
    n = len(channels)
    relu = lambda v: np.maximum(v, 0.0)  # noqa: E731
    a = {"in": x, "enc_in": [], "A": [], "S": [], "D": [None] * (n - 1)}
    i = 0
    h = x
    for lv in range(n - 1):
        a["enc_in"].append(h)
        a["A"].append(relu(conv(h, *L[i][:2])))
        a["S"].append(relu(conv(a["A"][-1], *L[i + 1][:2])))
        h = pool(a["S"][-1])
        i += 2
    a["bot_in"] = h
    a["B0"] = relu(conv(h, *L[i][:2]))
    a["B1"] = relu(conv(a["B0"], *L[i + 1][:2]))
    a["B2"] = relu(conv(a["B1"], *L[i + 2][:2]))
    i += 3
    y = a["B2"]
    a["U"] = [None] * (n - 1)
    a["M"] = [None] * (n - 1)
    for lv in range(n - 2, -1, -1):
        a["U"][lv] = up(y, a["S"][lv].shape[1:])
        a["M"][lv] = conv(a["U"][lv], *L[i][:2]) + a["S"][lv]
        a["D"][lv] = relu(conv(a["M"][lv], *L[i + 1][:2]))
        y = a["D"][lv]
        i += 2
    out = conv(y, *L[i][:2])
    return out, (L, a)


def backward(params, x, gout, in_ch, channels, pool_input=False):
    """Flat parameter gradient of sum(gout * forward(x)[:gout.shape[0]])."""
    if pool_input:
        xc = pool(x)
        return backward(params, xc, up_lin_grad(gout, xc.shape[1:]), in_ch, channels)
    out, (L, a) = forward(params, x, in_ch, channels)
    n = len(channels)
    g = np.zeros_like(out)
    g[: gout.shape[0]] = gout
    grads = [None] * len(L)
    mask_relu = lambda gg, act: gg * (act > 0)  # noqa: E731
    i = len(L) - 1
    gx, gw, gb = conv_grads(a["D"][0], L[i][0], g)
    grads[i] = (gw, gb)
    gskip = [None] * (n - 1)
    i -= 2  # the level-0 decoder 1x1 layer; its 3x3 partner is i + 1
    for lv in range(n - 1):
        gx = mask_relu(gx, a["D"][lv])
        gx, gw, gb = conv_grads(a["M"][lv], L[i + 1][0], gx)
        grads[i + 1] = (gw, gb)
        gskip[lv] = gx.copy()
        gx, gw, gb = conv_grads(a["U"][lv], L[i][0], gx)
        grads[i] = (gw, gb)
        coarse = a["D"][lv + 1] if lv + 1 < n - 1 else a["B2"]
        gx = up_grad(gx, coarse.shape[1:])
        i -= 2
    ib = 2 * (n - 1)  # first bottom layer
    gx = mask_relu(gx, a["B2"])
    gx, gw, gb = conv_grads(a["B1"], L[ib + 2][0], gx)
    grads[ib + 2] = (gw, gb)
    gx = mask_relu(gx, a["B1"])
    gx, gw, gb = conv_grads(a["B0"], L[ib + 1][0], gx)
    grads[ib + 1] = (gw, gb)
    gx = mask_relu(gx, a["B0"])
    gx, gw, gb = conv_grads(a["bot_in"], L[ib][0], gx)
    grads[ib] = (gw, gb)
    for lv in range(n - 2, -1, -1):
        gs = mask_relu(gskip[lv] + pool_grad(gx, a["S"][lv].shape[1:]), a["S"][lv])
        gx, gw, gb = conv_grads(a["A"][lv], L[2 * lv + 1][0], gs)
        grads[2 * lv + 1] = (gw, gb)
        gx = mask_relu(gx, a["A"][lv])
        gx, gw, gb = conv_grads(a["enc_in"][lv], L[2 * lv][0], gx)
        grads[2 * lv] = (gw, gb)
    return np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in grads])


def loss_and_grads(params, x, target, mask, in_ch, out_ch, channels, pool_input=False):
    """Masked MSE over the first out_ch outputs and its parameter gradient (flat)."""
    out, _ = forward(params, x, in_ch, channels, pool_input)
    m = np.ones(x.shape[1:]) if mask is None else mask
    diff = out[:out_ch] - target
    denom = m.sum() * out_ch
    loss = float((m * diff**2).sum() / denom)
    g = 2 * m * diff / denom
    return loss, out, backward(params, x, g, in_ch, channels, pool_input)
