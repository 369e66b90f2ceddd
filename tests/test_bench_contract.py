"""bench.py's reference arm runs on the CPU (the reference's SciPy CSR matvec and
Jacobi-CG on an assembled 16^3 sample of the elasticity workload): its JSON line
carries the keys the benchmark contract names and the CPU time to solution."""

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
    tts = d["time_to_solution"]["scipy_jacobi_cg_true_residual_restarts"]
    assert tts["converged"] and tts["relative_residual"] <= 1e-8 and tts["iterations"] > 0
