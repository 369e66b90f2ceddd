"""The learned preconditioner on the GPU: network forward and gradients against
the NumPy oracle (FP32 kernels vs FP64 oracle: 2e-4 relative on outputs, 2e-3
relative to the largest entry on gradients), and flexible CG with the trained
network against plain Jacobi-PCG (same tolerance, same answer, fewer iterations)."""

import ctypes

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200 import _lib
from jaxiga_b200.learned import LearnedPreconditioner, _DeviceArray
from oracle import cnn_oracle

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _s():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("grid,in_ch,out_ch,channels", [((9, 7, 5), 2, 1, (4, 8, 12)), ((6, 6, 1), 3, 3, (8, 8, 16))])
def test_network_forward_and_gradient_match_oracle(grid, in_ch, out_ch, channels):
    import torch

    lib = _lib.load()
    h = ctypes.c_void_p()
    _lib.check(lib.jxb_cnn_create(in_ch, out_ch, (ctypes.c_int32 * 3)(*channels), 5, ctypes.byref(h)))
    ptr, n = ctypes.c_void_p(), ctypes.c_int64()
    _lib.check(lib.jxb_cnn_params(h, ctypes.byref(ptr), ctypes.byref(n)))
    params = torch.as_tensor(_DeviceArray(ptr.value, n.value), device="cuda")
    rng = np.random.default_rng(3)
    p = rng.uniform(-0.3, 0.3, n.value)
    params.copy_(torch.as_tensor(p, dtype=torch.float32))
    p32 = params.cpu().numpy().astype(np.float64)
    nx, ny, nz = grid
    x = rng.standard_normal((in_ch, nz, ny, nx))
    t = rng.standard_normal((out_ch, nz, ny, nx))
    mask = (rng.random((nz, ny, nx)) > 0.2).astype(np.float64)
    xd = torch.as_tensor(x, dtype=torch.float32, device="cuda").contiguous()
    out = torch.empty((out_ch, nz, ny, nx), dtype=torch.float32, device="cuda")
    _lib.check(lib.jxb_cnn_forward(h, _s(), nx, ny, nz, _p(xd), _p(out)))
    loss_ref, out_ref, g_ref = cnn_oracle.loss_and_grads(p32, x.astype(np.float32).astype(np.float64),
                                                         t.astype(np.float32).astype(np.float64), mask, in_ch,
                                                         out_ch, channels)
    o = out.cpu().numpy()
    assert np.abs(o - out_ref[:out_ch]).max() <= 2e-4 * np.abs(out_ref[:out_ch]).max()
    _lib.check(lib.jxb_cnn_zero_grad(h, _s()))
    loss = ctypes.c_double()
    td = torch.as_tensor(t, dtype=torch.float32, device="cuda").contiguous()
    md = torch.as_tensor(mask, dtype=torch.float32, device="cuda").contiguous()
    _lib.check(lib.jxb_cnn_accumulate(h, _s(), nx, ny, nz, _p(xd), _p(td), _p(md), ctypes.byref(loss)))
    gp, gn = ctypes.c_void_p(), ctypes.c_int64()
    _lib.check(lib.jxb_cnn_grads(h, ctypes.byref(gp), ctypes.byref(gn)))
    g = torch.as_tensor(_DeviceArray(gp.value, gn.value), device="cuda").cpu().numpy()
    assert abs(loss.value - loss_ref) <= 1e-4 * abs(loss_ref)
    assert np.abs(g - g_ref).max() <= 2e-3 * np.abs(g_ref).max()
    lib.jxb_cnn_destroy(h)


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
    op = jx.Operator(V, "poisson", (1.0,), prescribed=mask, coef_qp=a)
    feat = ((loga - loga.mean()) / loga.std())[None, :]
    return V, op, feat


def test_learned_fcg_solves_and_beats_jacobi_pcg(tmp_path):
    import torch

    V, op, feat = _darcy(16)
    b = op.load(torch.ones(V.n_elems * 64, dtype=torch.float64, device="cuda"))
    lp = LearnedPreconditioner(op, features=feat, channels=(8, 16, 32), seed=1)
    R, E, st = lp.pairs_from_solve(b, n_pairs=400, every=1, tol=1e-12)
    assert st["converged"] and R.shape[0] > 50
    losses = lp.train(R, E, epochs=6, lr=3e-3, batch=4)
    assert losses[-1] < losses[0]
    x_ref, st_ref = op.pcg(b, tol=1e-8, preconditioner="jacobi")
    x, st_l = lp.solve(b, tol=1e-8)
    assert st_l["converged"] and st_ref["converged"]
    rel = float(torch.linalg.norm(x - x_ref) / torch.linalg.norm(x_ref))
    assert rel < 1e-6
    # the trained network takes fewer Krylov iterations than Jacobi
    assert st_l["iterations"] < st_ref["iterations"], (st_l, st_ref)
    # checkpoint / resume reproduces the preconditioner
    path = tmp_path / "pc.npz"
    lp.save(path)
    lp2 = LearnedPreconditioner(op, features=feat, channels=(8, 16, 32), seed=9)
    lp2.load(path)
    r = torch.randn(V.n_dofs, dtype=torch.float64, device="cuda") * torch.as_tensor(~op.prescribed_mask, device="cuda")
    assert torch.equal(lp.forward(r), lp2.forward(r))
    lp.close()
    lp2.close()
    op.close()
