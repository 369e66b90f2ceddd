"""CPU oracle of the learned-preconditioner network (NumPy, FP64).

TEST INFRASTRUCTURE ONLY: the GPU network (libjxb's cnn kernels) is checked
against this restatement -- forward output and parameter gradients of the
masked mean-squared-error loss. The reference has no learned preconditioner
(its only preconditioner is Jacobi, src/jaxiga/solvers/linear.py:419-431), so
this oracle restates the network the way libjxb defines it:

    level 0: in -> c0 relu; c0 -> c0 relu = s0
    level 1: pool(s0) -> c1 relu; c1 -> c1 relu = s1
    level 2: pool(s1) -> c2 relu; c2 -> c2 relu; c2 -> c2 relu
    level 1: up -> 1x1 c2 -> c1 (+ s1); c1 -> c1 relu
    level 0: up -> 1x1 c1 -> c0 (+ s0); c0 -> c0 relu; c0 -> 4 (linear; first out_ch used)

3x3x3 convolutions use zero padding, tap index k = dx + 3 dy + 9 dz; pooling
averages the existing children of a coarse voxel (odd sizes round up);
upsampling copies a coarse voxel to its children. Parameters are one flat
vector: per layer the weights [co][ci][k] then the biases [co].
"""

from __future__ import annotations

import numpy as np

SPECS = ["L0A", "L0B", "L1A", "L1B", "L2A", "L2B", "L2C", "L1C", "L1D", "L0C", "L0D", "L0E"]


def layer_shapes(in_ch, channels):
    c0, c1, c2 = channels
    return [(in_ch, c0, 3, True), (c0, c0, 3, True), (c0, c1, 3, True), (c1, c1, 3, True), (c1, c2, 3, True),
            (c2, c2, 3, True), (c2, c2, 3, True), (c2, c1, 1, False), (c1, c1, 3, True), (c1, c0, 1, False),
            (c0, c0, 3, True), (c0, 4, 3, False)]


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


def forward(params, x, in_ch, channels):
    """Returns (output [4, ...], cache)."""
    L = unpack(np.asarray(params, dtype=np.float64), in_ch, channels)
    relu = lambda v: np.maximum(v, 0.0)  # noqa: E731
    a = {}
    a["in"] = x
    a["A0A"] = relu(conv(x, *L[0][:2]))
    a["S0"] = relu(conv(a["A0A"], *L[1][:2]))
    a["P1"] = pool(a["S0"])
    a["A1A"] = relu(conv(a["P1"], *L[2][:2]))
    a["S1"] = relu(conv(a["A1A"], *L[3][:2]))
    a["P2"] = pool(a["S1"])
    a["A2A"] = relu(conv(a["P2"], *L[4][:2]))
    a["A2B"] = relu(conv(a["A2A"], *L[5][:2]))
    a["A2C"] = relu(conv(a["A2B"], *L[6][:2]))
    a["U1"] = up(a["A2C"], a["S1"].shape[1:])
    a["M1"] = conv(a["U1"], *L[7][:2]) + a["S1"]
    a["A1D"] = relu(conv(a["M1"], *L[8][:2]))
    a["U0"] = up(a["A1D"], a["S0"].shape[1:])
    a["M0"] = conv(a["U0"], *L[9][:2]) + a["S0"]
    a["A0D"] = relu(conv(a["M0"], *L[10][:2]))
    out = conv(a["A0D"], *L[11][:2])
    return out, (L, a)


def loss_and_grads(params, x, target, mask, in_ch, out_ch, channels):
    """Masked MSE over the first out_ch outputs and its parameter gradient (flat)."""
    out, (L, a) = forward(params, x, in_ch, channels)
    m = np.ones(x.shape[1:]) if mask is None else mask
    diff = out[:out_ch] - target
    denom = m.sum() * out_ch
    loss = float((m * diff**2).sum() / denom)
    g = np.zeros_like(out)
    g[:out_ch] = 2 * m * diff / denom
    grads = [None] * len(L)
    mask_relu = lambda gg, act: gg * (act > 0)  # noqa: E731
    gx, gw, gb = conv_grads(a["A0D"], L[11][0], g)
    grads[11] = (gw, gb)
    gx = mask_relu(gx, a["A0D"])
    gx, gw, gb = conv_grads(a["M0"], L[10][0], gx)
    grads[10] = (gw, gb)
    gS0 = gx.copy()
    gx, gw, gb = conv_grads(a["U0"], L[9][0], gx)
    grads[9] = (gw, gb)
    gx = mask_relu(up_grad(gx, a["A1D"].shape[1:]), a["A1D"])
    gx, gw, gb = conv_grads(a["M1"], L[8][0], gx)
    grads[8] = (gw, gb)
    gS1 = gx.copy()
    gx, gw, gb = conv_grads(a["U1"], L[7][0], gx)
    grads[7] = (gw, gb)
    gx = mask_relu(up_grad(gx, a["A2C"].shape[1:]), a["A2C"])
    gx, gw, gb = conv_grads(a["A2B"], L[6][0], gx)
    grads[6] = (gw, gb)
    gx = mask_relu(gx, a["A2B"])
    gx, gw, gb = conv_grads(a["A2A"], L[5][0], gx)
    grads[5] = (gw, gb)
    gx = mask_relu(gx, a["A2A"])
    gx, gw, gb = conv_grads(a["P2"], L[4][0], gx)
    grads[4] = (gw, gb)
    gS1 = mask_relu(gS1 + pool_grad(gx, a["S1"].shape[1:]), a["S1"])
    gx, gw, gb = conv_grads(a["A1A"], L[3][0], gS1)
    grads[3] = (gw, gb)
    gx = mask_relu(gx, a["A1A"])
    gx, gw, gb = conv_grads(a["P1"], L[2][0], gx)
    grads[2] = (gw, gb)
    gS0 = mask_relu(gS0 + pool_grad(gx, a["S0"].shape[1:]), a["S0"])
    gx, gw, gb = conv_grads(a["A0A"], L[1][0], gS0)
    grads[1] = (gw, gb)
    gx = mask_relu(gx, a["A0A"])
    gx, gw, gb = conv_grads(x, L[0][0], gx)
    grads[0] = (gw, gb)
    flat = np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in grads])
    return loss, out, flat
