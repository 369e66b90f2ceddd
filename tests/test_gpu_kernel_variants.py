"""The degree-3 3D apply exists in several kernels, selected by JXB_BRICK3_MMA
(read once per process): 0 = the FMA kernel, 2 = the FP64 tensor-core kernel
with stage hand-offs through shared memory, 4 = the register-fragment
tensor-core kernel reading the factor tiles from L2, 5 = the same with the tiles
copied into shared memory by the bulk-copy engine (the default is 4 for the
scalar operator, 5 for elasticity). All must give the same K.v: each variant's
result is computed in a child process and compared with the default kernel's
result of this process to 1e-13 relative (they sum in different orders)."""

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


@pytest.mark.parametrize("variant", ["0", "2", "4", "5"])
@pytest.mark.parametrize("kind", ["poisson", "elasticity"])
def test_kernel_variants_agree(kind, variant, tmp_path):
    V, op, x = case(kind)
    y_mma = op.apply(x).cpu().numpy()
    out = str(tmp_path / "y.npy")
    env = dict(os.environ, JXB_BRICK3_MMA=variant)
    subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, kind=kind, out=out)], env=env, check=True,
                   cwd=ROOT, timeout=600)
    y_var = np.load(out)
    assert np.abs(y_mma - y_var).max() <= 1e-13 * np.abs(y_var).max()
    assert not np.array_equal(y_mma, np.zeros_like(y_mma))
    op.close()
