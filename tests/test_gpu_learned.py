"""The learned preconditioner on the GPU: network forward and gradients against
the NumPy oracle (FP32 kernels vs FP64 oracle: 2e-4 relative on outputs, 2e-3
relative to the largest entry on gradients) for 2-4 level U-Nets, the
energy-norm training step against the oracle network plus the assembled
oracle operator, and truncated flexible CG with the trained network against
plain Jacobi-PCG (same tolerance, same answer, fewer iterations)."""

import ctypes

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200 import _lib
from jaxiga_b200.learned import LearnedPreconditioner, _DeviceArray
from jaxiga_b200.space import expand_dofs
from oracle import cnn_oracle

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _s():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _make_net(lib, in_ch, out_ch, channels, seed, rng, pool=False):
    import torch

    h = ctypes.c_void_p()
    _lib.check(lib.jxb_cnn_create(in_ch, out_ch, len(channels), (ctypes.c_int32 * len(channels))(*channels), seed,
                                  ctypes.byref(h)))
    if pool:
        _lib.check(lib.jxb_cnn_set_input_pooling(h, 1))
    ptr, n = ctypes.c_void_p(), ctypes.c_int64()
    _lib.check(lib.jxb_cnn_params(h, ctypes.byref(ptr), ctypes.byref(n)))
    params = torch.as_tensor(_DeviceArray(ptr.value, n.value), device="cuda")
    params.copy_(torch.as_tensor(rng.uniform(-0.3, 0.3, n.value), dtype=torch.float32))
    return h, params.cpu().numpy().astype(np.float64)


def _grads(lib, h):
    import torch

    gp, gn = ctypes.c_void_p(), ctypes.c_int64()
    _lib.check(lib.jxb_cnn_grads(h, ctypes.byref(gp), ctypes.byref(gn)))
    return torch.as_tensor(_DeviceArray(gp.value, gn.value), device="cuda").cpu().numpy()


@pytest.mark.parametrize("grid,in_ch,out_ch,channels,pool", [
    ((9, 7, 5), 2, 1, (4, 8, 12), False),
    ((6, 6, 1), 3, 3, (8, 8, 16), False),
    ((19, 18, 17), 2, 1, (8, 16, 24, 32), False),
    ((11, 9, 7), 4, 3, (12, 24), False),
    ((21, 5, 3), 1, 1, (16, 32, 48), False),
    ((66, 64, 40), 2, 1, (8, 16), False),  # level 0 with wide channel blocks, level 1 with narrow ones
    ((19, 18, 17), 2, 1, (8, 16, 24), True),  # input pooling: odd sizes round up
    ((13, 10, 6), 4, 3, (8, 16), True),
])
def test_network_forward_and_gradient_match_oracle(grid, in_ch, out_ch, channels, pool):
    import torch

    lib = _lib.load()
    rng = np.random.default_rng(3)
    h, p32 = _make_net(lib, in_ch, out_ch, channels, 5, rng, pool)
    nx, ny, nz = grid
    x = rng.standard_normal((in_ch, nz, ny, nx))
    t = rng.standard_normal((out_ch, nz, ny, nx))
    mask = (rng.random((nz, ny, nx)) > 0.2).astype(np.float64)
    xd = torch.as_tensor(x, dtype=torch.float32, device="cuda").contiguous()
    out = torch.empty((out_ch, nz, ny, nx), dtype=torch.float32, device="cuda")
    _lib.check(lib.jxb_cnn_forward(h, _s(), nx, ny, nz, _p(xd), _p(out)))
    x32 = x.astype(np.float32).astype(np.float64)
    loss_ref, out_ref, g_ref = cnn_oracle.loss_and_grads(p32, x32, t.astype(np.float32).astype(np.float64), mask,
                                                         in_ch, out_ch, channels, pool)
    o = out.cpu().numpy()
    assert np.abs(o - out_ref[:out_ch]).max() <= 2e-4 * np.abs(out_ref[:out_ch]).max()
    _lib.check(lib.jxb_cnn_zero_grad(h, _s()))
    loss = ctypes.c_double()
    td = torch.as_tensor(t, dtype=torch.float32, device="cuda").contiguous()
    md = torch.as_tensor(mask, dtype=torch.float32, device="cuda").contiguous()
    _lib.check(lib.jxb_cnn_accumulate(h, _s(), nx, ny, nz, _p(xd), _p(td), _p(md), ctypes.byref(loss)))
    g = _grads(lib, h)
    assert abs(loss.value - loss_ref) <= 1e-4 * abs(loss_ref)
    assert np.abs(g - g_ref).max() <= 2e-3 * np.abs(g_ref).max()
    # backward from an arbitrary output gradient
    gout = rng.standard_normal((out_ch, nz, ny, nx))
    god = torch.as_tensor(gout, dtype=torch.float32, device="cuda").contiguous()
    _lib.check(lib.jxb_cnn_zero_grad(h, _s()))
    _lib.check(lib.jxb_cnn_forward(h, _s(), nx, ny, nz, _p(xd), _p(out)))
    _lib.check(lib.jxb_cnn_backward(h, _s(), nx, ny, nz, _p(xd), _p(god)))
    g2 = _grads(lib, h)
    g2_ref = cnn_oracle.backward(p32, x32, gout.astype(np.float32).astype(np.float64), in_ch, channels, pool)
    assert np.abs(g2 - g2_ref).max() <= 2e-3 * np.abs(g2_ref).max()
    lib.jxb_cnn_destroy(h)


@pytest.mark.parametrize("op_name,angle,pool", [("poisson", 0, False), ("elasticity", 0, False), ("poisson", 1, False),
                                               ("elasticity", 1, False), ("poisson", 1, True), ("poisson", 2, True),
                                               ("elasticity", 2, False)])
def test_energy_loss_gradient_matches_oracle(op_name, angle, pool):
    """Energy-norm losses against the oracle network and the assembled K:
    w d^T K d with d = P_f (e - s N(in)), and w (1 - (z.r)^2 / ((z^T K z)(e.r)))
    with z = P_f s N(in), r = K e."""
    import torch

    from oracle import iga_oracle as O

    lib = _lib.load()
    rng = np.random.default_rng(11)
    kn = np.linspace(0, 1, 4)[1:-1]
    vec = 3 if op_name == "elasticity" else 1
    V = jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kn), vec=vec)
    pres = np.unique(expand_dofs(V.side_indices("u0"), vec))
    mask = np.zeros(V.n_dofs, bool)
    mask[pres] = True
    coef = (1.0, 0.3) if vec == 3 else (1.0,)
    op = jx.Operator(V, op_name, coef, prescribed=mask)
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, vec)
    params = {"E": 1.0, "nu": 0.3} if vec == 3 else {"a0": 1.0}
    A = O.Assembled(S, op_name, params, pres, np.zeros(len(pres)), need_full=False)
    nx, ny, nz = V.n_cp
    ncp = V.n_scalar_basis
    in_ch = vec + 1
    h, p32 = _make_net(lib, in_ch, vec, (4, 8, 12), 7, rng, pool)
    x = rng.standard_normal((in_ch, nz, ny, nx))
    e = rng.standard_normal((vec, nz, ny, nx)).astype(np.float32).astype(np.float64)
    s, w = 0.7, 0.3
    to_dof = lambda v: v.reshape(vec, ncp).T.reshape(-1)  # noqa: E731  grid [c][cp] -> DOF vec*cp + c
    to_grid = lambda v: v.reshape(ncp, vec).T.reshape(vec, nz, ny, nx)  # noqa: E731

    def K(v):
        out = np.zeros(V.n_dofs)
        out[A.free] = A.K @ v[A.free]
        return out

    ed_ = to_dof(e)
    ed_[mask] = 0.0
    r = to_grid(K(ed_)).astype(np.float32).astype(np.float64)  # the pair's residual r = K e
    xd = torch.as_tensor(x, dtype=torch.float32, device="cuda").contiguous()
    ed = torch.as_tensor(e, dtype=torch.float32, device="cuda").contiguous()
    rd = torch.as_tensor(r, dtype=torch.float32, device="cuda").contiguous()
    _lib.check(lib.jxb_cnn_zero_grad(h, _s()))
    loss = ctypes.c_double()
    _lib.check(lib.jxb_cnn_accumulate_energy(op.handle, h, _s(), _p(xd), _p(ed), _p(rd), s, w, angle,
                                             ctypes.byref(loss)))
    g = _grads(lib, h)
    x32 = x.astype(np.float32).astype(np.float64)
    out, _ = cnn_oracle.forward(p32, x32, in_ch, (4, 8, 12), pool)
    if not angle:
        d = to_dof(e - s * out[:vec])
        d[mask] = 0.0
        Kd = K(d)
        loss_ref = w * float(d @ Kd)
        gout = to_grid(-2.0 * w * s * Kd)
    else:
        z = to_dof(s * out[:vec])
        z[mask] = 0.0
        rdof = to_dof(r)
        rdof[mask] = 0.0
        if angle == 2:  # additive two-level map z = s N + D^-1 r
            inv = np.zeros(V.n_dofs)
            inv[A.free] = O.jacobi_inverse(A.diag)
            z = z + inv * rdof
        Kz = K(z)
        a, bq, c = float(z @ rdof), float(z @ Kz), float(ed_ @ rdof)
        loss_ref = w * (1.0 - a * a / (bq * c))
        gz = w * 2.0 * a / (bq * c) * (a / bq * Kz - rdof)
        gz[mask] = 0.0
        gout = to_grid(s * gz)
    g_ref = cnn_oracle.backward(p32, x32, gout, in_ch, (4, 8, 12), pool)
    assert abs(loss.value - loss_ref) <= 1e-4 * abs(loss_ref)
    assert np.abs(g - g_ref).max() <= 2e-3 * np.abs(g_ref).max()
    lib.jxb_cnn_destroy(h)
    op.close()


def _darcy(n=16, seed=4):
    from jaxiga_b200 import workloads

    kn = np.linspace(0, 1, n + 1)[1:-1]
    V = jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kn))
    nx, ny, nz = V.n_cp
    axes = [V.cpts[:nx, 0], V.cpts[: nx * ny: nx, 1], V.cpts[:: nx * ny, 2]]
    loga = workloads.grf_on_grid(axes, 0.1, 1.0, np.random.default_rng(seed))
    geo = jx.Operator(V, "poisson", (1.0,))
    a = np.exp(geo.interpolate(loga).cpu().numpy()[..., 0])
    geo.close()
    mask = np.zeros(V.n_dofs, bool)
    mask[np.unique(np.concatenate([V.side_indices(s) for s in ("u0", "u1", "v0", "v1", "w0", "w1")]))] = True
    op = jx.Operator(V, "poisson", (1.0,), prescribed=mask, coef_qp=a, want_f32=True)
    feat = ((loga - loga.mean()) / loga.std())[None, :]
    return V, op, feat


def test_learned_fcg_solves_and_beats_jacobi_pcg(tmp_path):
    import torch

    V, op, feat = _darcy(16)
    b = op.load(torch.ones(V.n_elems * 64, dtype=torch.float64, device="cuda"))
    lp = LearnedPreconditioner(op, features=feat, seed=1)
    R, E, st = lp.pairs_from_solve(b, n_pairs=150, every=1, tol=1e-12)
    assert st["converged"] and R.shape[0] > 50
    R2, E2 = lp.pairs_random(250, tol=1e-10, seed=3)
    R, E = torch.cat([R, R2]), torch.cat([E, E2])
    # long enough that the gain does not hinge on rounding: measured on a B200,
    # 4 + 12 epochs left the network alone at 106-109 iterations against
    # Jacobi's 105, 10 + 50 epochs at 57-72 (loss 0.05)
    losses = lp.train(R, E, epochs=10, lr=3e-3, batch=4)
    losses += lp.train(R, E, epochs=50, lr=1e-3, batch=4, seed=1)
    assert losses[-1] < 0.5 * losses[0]
    x_ref, st_ref = op.pcg(b, tol=1e-8, preconditioner="jacobi")
    x, st_l = lp.solve(b, tol=1e-8)
    assert st_l["converged"] and st_ref["converged"]
    rel = float(torch.linalg.norm(x - x_ref) / torch.linalg.norm(x_ref))
    assert rel < 1e-6
    # the trained network takes fewer Krylov iterations than Jacobi-PCG, and
    # the same flexible CG without the network matches Jacobi-PCG
    _, st_j = lp.solve(b, tol=1e-8, use_network=False)
    assert st_j["converged"] and abs(st_j["iterations"] - st_ref["iterations"]) <= 2, (st_j, st_ref)
    assert st_l["learned_iterations"] == st_l["iterations"], st_l
    assert st_l["iterations"] < st_ref["iterations"], (st_l, st_ref)
    # two-level: the network as a line-searched coarse correction plus one Jacobi step
    x_t, st_t = lp.solve(b, tol=1e-8, two_level=True)
    assert st_t["converged"] and st_t["iterations"] < st_ref["iterations"], (st_t, st_ref)
    assert float(torch.linalg.norm(x_t - x_ref) / torch.linalg.norm(x_ref)) < 1e-6
    # mixed precision: FP32 flexible CG with reliable FP64 updates (the stored
    # directions kept), and restarted FP32 solves inside FP64 refinement
    x_m, st_m = lp.solve(b, tol=1e-8, mixed=True)
    assert st_m["converged"], st_m
    assert float(torch.linalg.norm(x_m - x_ref) / torch.linalg.norm(x_ref)) < 1e-6
    x_r, st_r = lp.solve(b, tol=1e-8, mixed=True, refinement="restart")
    assert st_r["converged"], st_r
    assert float(torch.linalg.norm(x_r - x_ref) / torch.linalg.norm(x_ref)) < 1e-6
    # keeping the directions costs fewer iterations than restarting (Jacobi FCG)
    _, st_jm = lp.solve(b, tol=1e-8, mixed=True, use_network=False)
    _, st_jr = lp.solve(b, tol=1e-8, mixed=True, use_network=False, refinement="restart")
    assert st_jm["converged"] and st_jr["converged"]
    assert st_jm["iterations"] <= 1.15 * st_j["iterations"] + 10, (st_jm, st_j)
    assert st_jm["iterations"] < st_jr["iterations"], (st_jm, st_jr)
    # additive two-level map with the fitted weight: one apply per iteration
    a = lp.fit_additive_weight(R, E, n_pairs=32)
    assert np.isfinite(a) and a > 0
    x_a, st_a = lp.solve(b, tol=1e-8, two_level="additive")
    assert st_a["converged"] and st_a["iterations"] < st_ref["iterations"], (st_a, st_ref)
    assert float(torch.linalg.norm(x_a - x_ref) / torch.linalg.norm(x_ref)) < 1e-6
    _, st_am = lp.solve(b, tol=1e-8, two_level="additive", mixed=True)
    assert st_am["converged"], st_am
    # the network's inference on the BF16 tensor cores: same answer, about as many iterations
    lp.set_inference_bf16(True)
    x_b, st_b = lp.solve(b, tol=1e-8, two_level="additive", mixed=True)
    assert st_b["converged"] and st_b["iterations"] <= 1.2 * st_am["iterations"] + 3, (st_b, st_am)
    assert float(torch.linalg.norm(x_b - x_ref) / torch.linalg.norm(x_ref)) < 1e-6
    lp.set_inference_bf16(False)
    # a network on the pooled residual (half resolution) in the additive map
    lpp = LearnedPreconditioner(op, features=feat, seed=2, pool_input=True)
    lpp.in_scale, lpp.out_scale = lp.in_scale, lp.out_scale
    lpp.train(R, E, epochs=6, lr=3e-3, batch=4, loss="additive")
    lpp.fit_additive_weight(R, E, n_pairs=32)
    x_p, st_p = lpp.solve(b, tol=1e-8, two_level="additive", mixed=True)
    assert st_p["converged"], st_p
    assert float(torch.linalg.norm(x_p - x_ref) / torch.linalg.norm(x_ref)) < 1e-6
    lpp.save(tmp_path / "pool.npz")
    lpq = LearnedPreconditioner.from_checkpoint(op, tmp_path / "pool.npz", features=feat)
    assert lpq.pool_input and lpq.channels == lpp.channels
    lpq.close()
    lpp.close()
    # checkpoint / resume reproduces the preconditioner
    path = tmp_path / "pc.npz"
    lp.save(path)
    lp2 = LearnedPreconditioner(op, features=feat, seed=9)
    lp2.load(path)
    r = torch.randn(V.n_dofs, dtype=torch.float64, device="cuda") * torch.as_tensor(~op.prescribed_mask, device="cuda")
    assert torch.equal(lp.forward(r), lp2.forward(r))
    assert lp2.additive_weight == lp.additive_weight
    lp.close()
    lp2.close()
    op.close()


@pytest.mark.parametrize("grid,in_ch,channels", [((35, 33, 31), 2, (8, 16, 24, 32)), ((20, 19, 1), 1, (8, 16, 24))])
def test_bf16_inference_forward_tracks_the_fp32_network(grid, in_ch, channels):
    """The BF16 tensor-core convolutions (BF16 operands, FP32 accumulation) on the
    layers of <= 32 channels against the FP32 kernels and the FP64 oracle: a
    BF16 tolerance of 2e-2 relative (8-bit mantissas through a dozen layers)."""
    import torch

    lib = _lib.load()
    rng = np.random.default_rng(11)
    h, p64 = _make_net(lib, in_ch, 1, channels, 3, rng)
    nx, ny, nz = grid
    x = rng.standard_normal((in_ch, nz, ny, nx)).astype(np.float32)
    xd = torch.as_tensor(x, device="cuda").contiguous()
    out32 = torch.empty((1, nz, ny, nx), device="cuda")
    out16 = torch.empty_like(out32)
    _lib.check(lib.jxb_cnn_forward(h, _s(), nx, ny, nz, _p(xd), _p(out32)))
    _lib.check(lib.jxb_cnn_set_inference_bf16(h, 1))
    _lib.check(lib.jxb_cnn_forward(h, _s(), nx, ny, nz, _p(xd), _p(out16)))
    a, b = out16.cpu().numpy().astype(np.float64), out32.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(a - b) < 2e-2 * np.linalg.norm(b)
    ref, _ = cnn_oracle.forward(p64, x.astype(np.float64), in_ch, channels, False)
    assert np.linalg.norm(a.reshape(-1) - ref[0].reshape(-1)) < 2e-2 * np.linalg.norm(ref[0])
    # a backward after a BF16 forward is refused; the FP32 forward makes it valid again
    g = torch.ones_like(out32)
    assert lib.jxb_cnn_backward(h, _s(), nx, ny, nz, _p(xd), _p(g)) == 1
    _lib.check(lib.jxb_cnn_set_inference_bf16(h, 0))
    _lib.check(lib.jxb_cnn_forward(h, _s(), nx, ny, nz, _p(xd), _p(out32)))
    _lib.check(lib.jxb_cnn_backward(h, _s(), nx, ny, nz, _p(xd), _p(g)))
    lib.jxb_cnn_destroy(h)
