"""bench.py's reference arm runs on the CPU (the reference's SciPy CSR matvec on
whole rows of the 64^3 elasticity operator, and its Jacobi-CG on the assembled
16^3 and 24^3 workloads): its JSON line carries the keys the benchmark contract
names, the headline workload's config and the CPU time to solution."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "3", "--warmup", "1"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600, check=True).stdout
    lines = [line for line in out.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 3
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["host"]["cpu_count"] >= 1
    assert d["config"]["workload"] == "elasticity3d_p3_64^3" and d["config"]["n_dofs"] == 902289
    assert d["cpu_baseline"]["rows"] > 0 and d["cpu_baseline"]["cores"] == d["cpu_baseline"]["host"]["threads_used"]
    for tts in d["time_to_solution"]["scipy_jacobi_cg_true_residual_restarts"].values():
        assert tts["converged"] and tts["relative_residual"] <= 1e-8 and tts["iterations"] > 0


def test_row_sample_rows_are_the_assembled_operators_rows():
    """The K.u sample of the CPU baseline is made of whole rows of the assembled
    free-free operator: on an 8^3 mesh, the rows built from an 8 x 6 x 4 element
    box equal the same rows of the oracle's full assembly, and the threaded
    product equals SciPy's."""
    import numpy as np

    sys.path.insert(0, ROOT)
    import bench
    from jaxiga_b200 import workloads
    from oracle import iga_oracle as O

    V, K, rows, _ = bench.cpu_row_sample(span=8, box=(8, 6, 4))
    assert K.shape[0] == len(rows) > 0
    Vf, problem, params = workloads.config2(n=8)
    pres, vals = problem.resolve_dirichlet(params)
    S = O.Space(Vf.knots, Vf.degree, Vf.cpts, Vf.wgts, 3)
    A = O.Assembled(S, "elasticity", {"E": 1.0, "nu": 0.3}, pres, vals, need_full=False)
    free_pos = np.searchsorted(A.free, rows)
    assert np.array_equal(A.free[free_pos], rows)
    ref = A.K[free_pos]
    diff = abs(ref - K).max()
    assert diff <= 1e-13 * abs(ref).max(), diff
    op = bench.ThreadedCSR(K, 3)
    x = np.random.default_rng(1).standard_normal(K.shape[1])
    assert np.allclose(op @ x, K @ x, rtol=1e-14, atol=1e-14)
    op.close()
