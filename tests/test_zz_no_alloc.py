"""jxb_apply_static -- the operator application that allocates nothing.

Some callers cannot allocate device memory at the point where they apply the
operator (a handler inside a framework that owns all device allocations, a
loop that must not pay an allocation's implicit synchronisation). For them
jxb_apply_static keeps the brick partial sums in a fixed 16 MiB device array
instead of the plan's scratch buffer. These tests call it through the C ABI,
twice in a row, and compare with jxb_apply at the tolerance the operator
tests use (1e-12 relative); they also check that a plan whose scratch does
not fit is refused with a clear message.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest

import jaxiga_b200 as jx
from jaxiga_b200 import _lib

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _elasticity(n):
    kn = np.linspace(0, 1, n + 1)[1:-1]
    V = jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 1, 1.3]).elevate(3).insert_knots(kn, kn, kn), vec=3)
    mask = np.zeros(V.n_dofs, bool)
    mask[jx.expand_dofs(V.side_indices("u0")[:, None], 3).ravel()] = True
    return V, jx.Operator(V, "elasticity", (1.0, 0.3), prescribed=mask)


def _poisson2d_rational():
    kn = np.linspace(0, 1, 41)[1:-1] ** 1.3
    V = jx.FunctionSpace(jx.primitives.quarter_annulus(1.0, 2.0).elevate(3).insert_knots(kn, kn))
    mask = np.zeros(V.n_dofs, bool)
    mask[V.side_indices("u0")] = True
    return V, jx.Operator(V, "poisson", (1.7,), prescribed=mask)


@pytest.mark.parametrize("make", [lambda: _elasticity(12), _poisson2d_rational])
@pytest.mark.parametrize("masked", [1, 0])
def test_static_apply_matches_apply_on_two_calls(make, masked):
    import torch

    V, op = make()
    lib = _lib.load()
    rng = np.random.default_rng(11)
    for call in range(2):
        x = torch.as_tensor(rng.standard_normal(V.n_dofs), device="cuda")
        y_ref = torch.empty_like(x)
        y = torch.full_like(x, float("nan"))
        _lib.check(lib.jxb_apply(op.handle, _stream(), _ptr(x), _ptr(y_ref), masked))
        _lib.check(lib.jxb_apply_static(op.handle, _stream(), _ptr(x), _ptr(y), masked))
        torch.cuda.synchronize()
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        assert np.all(np.isfinite(a)), f"call {call}"
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), f"call {call}"
    op.close()


def test_static_apply_refuses_a_plan_that_does_not_fit():
    import torch

    V, op = _elasticity(64)  # 26 MB of brick scratch > 16 MiB
    assert op.info["scratch_bytes"] > 16 << 20
    lib = _lib.load()
    x = torch.zeros(V.n_dofs, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    rc = lib.jxb_apply_static(op.handle, _stream(), _ptr(x), _ptr(y), 1)
    assert rc == 1
    assert b"jxb_apply" in lib.jxb_last_error() and b"bytes" in lib.jxb_last_error()
    op.close()
