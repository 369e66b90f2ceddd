"""The degree-3 3D apply exists as an FP64 tensor-core kernel (the default) and
as the FMA kernel (JXB_BRICK3_MMA=0, read once per process). Both must give the
same K.v: the FMA result is computed in a child process and compared with the
tensor-core result of this process to 1e-13 relative (the two sum in different
orders)."""

import os
import subprocess
import sys

import numpy as np
import pytest

import jaxiga_b200 as jx

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys, numpy as np
sys.path.insert(0, {root!r})
import jaxiga_b200 as jx
from tests.test_gpu_kernel_variants import case
V, op, x = case({kind!r})
np.save({out!r}, op.apply(x).cpu().numpy())
"""


def case(kind):
    kn = np.linspace(0, 1, 7)[1:-1]  # 6 spans per direction: one full brick column and a partial one
    kz = np.linspace(0, 1, 11)[1:-1]  # 10 layers: a full brick of 8 and a partial one
    vec = 3 if kind == "elasticity" else 1
    V = jx.FunctionSpace(jx.primitives.cuboid([0, 0, 0], [1, 1, 1]).elevate(3).insert_knots(kn, kn, kz), vec=vec)
    mask = np.zeros(V.n_dofs, bool)
    mask[np.unique(jx.expand_dofs(V.side_indices("u0"), vec))] = True
    rng = np.random.default_rng(7)
    if kind == "elasticity":
        op = jx.Operator(V, "elasticity", (1.0, 0.3), prescribed=mask)
    else:
        a = np.exp(rng.standard_normal((V.n_elems, 64)) * 0.5)
        op = jx.Operator(V, "poisson", (1.0,), prescribed=mask, coef_qp=a)
    x = rng.standard_normal(V.n_dofs)
    return V, op, x


@pytest.mark.parametrize("kind", ["poisson", "elasticity"])
def test_tensor_core_and_fma_kernels_agree(kind, tmp_path):
    V, op, x = case(kind)
    y_mma = op.apply(x).cpu().numpy()
    out = str(tmp_path / "y.npy")
    env = dict(os.environ, JXB_BRICK3_MMA="0")
    subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, kind=kind, out=out)], env=env, check=True,
                   cwd=ROOT, timeout=600)
    y_fma = np.load(out)
    assert np.abs(y_mma - y_fma).max() <= 1e-13 * np.abs(y_fma).max()
    assert not np.array_equal(y_mma, np.zeros_like(y_mma))
    op.close()
