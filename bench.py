#!/usr/bin/env python
"""Benchmark of the Galerkin linear-solve path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one matrix-free stiffness application K.u (FP64, masked to the
free DOFs) of the 3D linear-elasticity workload: unit cube, cubic NURBS,
64^3 elements, 902,289 DOFs, 16.8M Gauss points. The per-point factors
(1.34 GB) exceed the 126 MB L2, so consecutive steps stream them from HBM.
``value`` is whole-job DOF/s (N_dof x steps x n_gpus / max-over-ranks time,
CUDA events, barrier + synchronize on both sides). ``e2e`` is the same metric
through the C ABI with host buffers: every step copies u from pinned host
memory to the device, applies K and copies y back to pinned host memory, the
copies on their own streams overlapping the neighbouring steps' applies.
``time_to_solution`` gives the solves to a 1e-8 true relative residual: plain
FP64 Jacobi-PCG (with the reference CPU CG's true-residual restarts), the two
mixed-precision schemes, multigrid-preconditioned CG and, when
jaxiga_b200/checkpoints holds a trained network for the workload
(``python -m jaxiga_b200.train_pc``), flexible CG with the learned
preconditioner in every map.

On one GPU the same line also carries, under ``workloads``, the other
benchmark configurations measured the same way (apply DOF/s, roofline and
time to solution): Darcy 96^3 with a lognormal random coefficient, the
clamped Kirchhoff plate 256^2, and 256 uneven quarter-annulus Poisson
instances solved as one batch.

``cpu_baseline`` times the reference's CPU path on the host cores, all of
them: SciPy's CSR K.u on whole rows of the 64^3 elasticity operator (its
assembled matrix restricted to the control points of an element box, built
from that box's element tangents; the full assembly is infeasible on a CPU,
77 GB of element matrices), and its Jacobi-CG with true-residual restarts
(src/jaxiga/solvers/linear.py:261-321, restated in the oracle) on the same
workload at 16^3 elements, next to the GPU's time to solution at that size.

``--impl reference`` times that CPU path alone for the headline metric, on
the same config: each step one threaded SciPy CSR product of the 64^3 row
sample (caches flushed before each); the line adds the CPU time to solution
at 16^3 and 24^3.

With ``--gpus N > 1`` (torchrun) every rank runs an independent replica of
the headline workload (weak scaling; the single-patch apply does not
exchange data).
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-1e-8 residual & K·u DOF/s: mixed+learned vs plain FP64 PCG, 1 B200"
UNIT = "DOF/s"
N_SPAN = 64
CPU_SAMPLE_SPAN = 16
CPU_SAMPLE_SPAN_LARGE = 24  # the reference arm also times the CPU solve here (about 80 s of assembly and CG)
TOL = 1e-8
# Chebyshev smoother (degree, range) of the multigrid rows, per workload: the
# fastest of degrees {2, 3, 4} x ranges {10, 20, 40} in a sweep of
# `python -m jaxiga_b200.multigrid` on a B200 (elasticity 64^3: 0.221 s at
# (3, 40) against 0.238 s at the library default (3, 20); Darcy 96^3: 0.085 s
# at (2, 20) against 0.092 s)
MG_SMOOTHER = {"elasticity": (3, 40.0), "darcy": (2, 20.0), "plate": (3, 20.0)}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-solve", action="store_true", help="skip the time-to-solution runs")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-extra", action="store_true", help="skip the Darcy / plate / batch rows")
    ap.add_argument("--span", type=int, default=None, help="elements per direction (default 64, Darcy 96)")
    ap.add_argument("--workload", default="elasticity", choices=["elasticity", "darcy", "plate", "batch"],
                    help="elasticity: 3D elasticity 64^3 (the headline); darcy: 3D Darcy 96^3; plate: Kirchhoff "
                         "plate 256^2; batch: 256 uneven quarter-annulus Poisson instances in one graph")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region (NVML reads only)
# ---------------------------------------------------------------------------
REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
           0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
           0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}


def nvml_handle(pynvml, device):
    """NVML handle of CUDA device ``device`` (an index into the visible
    devices), found by PCI bus id: NVML numbers every GPU of the machine and
    its order need not follow CUDA's or CUDA_VISIBLE_DEVICES."""
    import torch

    p = torch.cuda.get_device_properties(device)
    bus = "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
    try:
        return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
    except Exception:
        return pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())


class ClockSampler:
    """SM clock and clock-event reasons of one GPU, sampled in a thread; no
    samples (and clocks reported as unknown) when NVML cannot find the GPU."""

    def __init__(self, device, period=0.005):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.period = period
        self.stop_ev = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = nvml_handle(pynvml, device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nvml = None
        self.t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self.stop_ev.is_set():
            try:
                self.samples.append(self.nvml.nvmlDeviceGetClockInfo(self.h, self.nvml.NVML_CLOCK_SM))
                mask = self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in REASONS.items():
                    if mask & bit and bit != 0x1:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.nvml:
            self.t.start()
        return self

    def __exit__(self, *a):
        self.stop_ev.set()
        if self.nvml:
            self.t.join()

    def summary(self):
        med = float(np.median(self.samples)) if self.samples else None
        return {"sm_mhz": med, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profile_traffic(workload, span):
    """DRAM bytes per launch of the workload's brick kernel from the committed ncu
    summary (profiles/apply_dram.json), scaled from the captured size by the
    element count when the capture was smaller; None when there is none."""
    try:
        with open(os.path.join(ROOT, "profiles", "apply_dram.json")) as f:
            d = json.load(f)[workload]
        scale = (span / d["span"]) ** (2 if workload == "plate" else 3)
        return {"dram_bytes_per_launch": d["dram_bytes_per_launch"] * scale, "captured_span": d["span"]}
    except Exception:
        return None


# ---------------------------------------------------------------------------
# CPU baseline: the reference's CPU path (SciPy CSR K.u and Jacobi-CG with
# true-residual restarts) on the host cores. K.u is timed on a bounded sample
# of the 64^3 elasticity operator itself (whole rows of its assembled matrix);
# the solves run at the sizes whose full assembly a CPU can hold.
# ---------------------------------------------------------------------------
INFEASIBLE = ("64^3 elements assembled on a CPU is infeasible: 262,144 element matrices of 192 x 192 "
              "(77 GB), a 38.7 GB int32 scatter map and ~1 h of CSR-pattern construction")
CPU_ROW_BOX = (64, 32, 4)  # elements per direction of the element box whose rows K.u is timed on
CPU_FLUSH_BYTES = 512 << 20  # read between timed CPU steps so the sample starts outside the caches


def cpu_threads():
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return max(1, os.cpu_count() or 1)


def host_info(threads):
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_count": os.cpu_count(), "cpu_model": model, "threads_used": threads,
            "threads_env": {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS",
                                                           "MKL_NUM_THREADS")},
            "note": "SciPy's CSR matvec runs on row blocks in a thread pool (it releases the GIL); "
                    "the CG's vector updates and BLAS dots run on one thread"}


class ThreadedCSR:
    """A SciPy CSR matrix whose K.u runs as row blocks of about equal nonzero
    count on a thread pool. It offers what the reference's CPU CG uses of its
    operator (shape, dtype, diagonal(), the product), so the SciPy solver runs
    on it unchanged."""

    def __init__(self, K, threads):
        import scipy.sparse.linalg as spla
        from concurrent.futures import ThreadPoolExecutor

        self.K = K
        self.shape, self.dtype = K.shape, K.dtype
        self.threads = threads
        cuts = np.searchsorted(K.indptr, np.linspace(0, K.nnz, threads + 1)).clip(0, K.shape[0])
        cuts[0], cuts[-1] = 0, K.shape[0]
        self.blocks = [(int(a), int(b), K[int(a):int(b)]) for a, b in zip(cuts[:-1], cuts[1:]) if b > a]
        self.pool = ThreadPoolExecutor(threads)
        self.op = spla.LinearOperator(K.shape, matvec=self.matvec, dtype=K.dtype)
        self.op.diagonal = K.diagonal

    def matvec(self, x):
        x = np.asarray(x).ravel()
        y = np.empty(self.shape[0])

        def run(blk):
            a, b, B = blk
            y[a:b] = B @ x

        list(self.pool.map(run, self.blocks))
        return y

    def __matmul__(self, x):
        return self.matvec(x)

    def flush(self, buf):
        """Read ``buf`` across the pool (evicts the sample from the caches)."""
        parts = np.array_split(buf, self.threads)
        list(self.pool.map(np.sum, parts))

    def close(self):
        self.pool.shutdown()


def cpu_row_sample(span=N_SPAN, box=CPU_ROW_BOX):
    """Whole rows of the elasticity workload's free-free operator K_ff at
    ``span``^3 elements, for the free DOFs of every control point whose support
    lies inside an element box of ``box`` elements (the full width in x, centred
    in y and z). Only the box's element tangents are formed (oracle restatement of
    src/jaxiga/forms/library.py:174-181) and scattered into those rows
    (src/jaxiga/methods/galerkin.py:122-148), so each row is exactly the full
    operator's row; columns index the free DOFs.

    Returns (space, CSR rows (n_rows x n_free), row DOFs, set-up seconds)."""
    import scipy.sparse as sps

    from jaxiga_b200 import workloads
    from oracle import iga_oracle as O

    t0 = time.perf_counter()
    V, problem, params = workloads.config2(n=span)
    pres, _ = problem.resolve_dirichlet(params)
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 3)
    n_dofs, ncp = S.n_dofs, S.n_cp
    free_index = np.full(n_dofs, -1, dtype=np.int64)
    free = np.setdiff1d(np.arange(n_dofs), pres)
    free_index[free] = np.arange(len(free))
    lo = [(S.n_span[d] - box[d]) // 2 for d in range(3)]
    hi = [lo[d] + box[d] for d in range(3)]
    inside = np.all([(S.elem_idx[d] >= lo[d]) & (S.elem_idx[d] < hi[d]) for d in range(3)], axis=0)
    elems = np.nonzero(inside)[0]
    # control points whose support (elements first..first+p per direction) is inside the box
    cp_ok = []
    for d in range(3):
        first = S.spans[d][2]
        ok = np.zeros(ncp[d], bool)
        for i in range(ncp[d]):
            sup = np.nonzero((first <= i) & (first + S.degree[d] >= i))[0]
            ok[i] = len(sup) > 0 and sup.min() >= lo[d] and sup.max() < hi[d]
        cp_ok.append(ok)
    idx = np.arange(S.n_scalar)
    ijk = (idx % ncp[0], (idx // ncp[0]) % ncp[1], idx // (ncp[0] * ncp[1]))
    cp_sel = cp_ok[0][ijk[0]] & cp_ok[1][ijk[1]] & cp_ok[2][ijk[2]]
    row_dofs = np.nonzero(np.repeat(cp_sel, 3) & (free_index >= 0))[0]
    row_index = np.full(n_dofs, -1, dtype=np.int64)
    row_index[row_dofs] = np.arange(len(row_dofs))
    gd_all = S.expand(S.elem_dofs)
    K = None
    for c0 in range(0, len(elems), 2048):
        el = elems[c0:c0 + 2048]
        Ke = O.element_tangents("elasticity", O.evaluate(S, el), {"E": 1.0, "nu": 0.3}, 3)
        gd = gd_all[el]
        e_i, r_i = np.nonzero(row_index[gd] >= 0)
        cols = free_index[gd[e_i]]
        vals = Ke[e_i, r_i]
        keep = cols >= 0
        rows = np.broadcast_to(row_index[gd[e_i, r_i]][:, None], cols.shape)
        part = sps.csr_matrix((vals[keep], (rows[keep], cols[keep])), shape=(len(row_dofs), len(free)))
        K = part if K is None else K + part
    K.sum_duplicates()
    K.sort_indices()
    return V, K, row_dofs, time.perf_counter() - t0


def time_cpu_rows(K, threads, steps, warmup=1):
    """Seconds of each of ``steps`` threaded K.u products of the row sample, the
    caches flushed (a 512 MB read) before each; the flush is outside the timing."""
    from threadpoolctl import threadpool_limits

    op = ThreadedCSR(K, threads)
    x = np.random.default_rng(0).standard_normal(K.shape[1])
    buf = np.ones(CPU_FLUSH_BYTES // 8)
    times = []
    with threadpool_limits(1):  # idle BLAS threads would spin against the pool's
        for _ in range(max(warmup, 1)):
            op @ x
        for _ in range(steps):
            op.flush(buf)
            t0 = time.perf_counter()
            op @ x
            times.append(time.perf_counter() - t0)
    op.close()
    return np.asarray(times)


def cpu_sample(span):
    """The elasticity workload at ``span``^3 assembled by the oracle, with its
    load vector (body force plus the interpolated random field)."""
    from jaxiga_b200 import workloads
    from oracle import iga_oracle as O

    t0 = time.perf_counter()
    V, problem, params = workloads.config2(n=span)
    pres, vals = problem.resolve_dirichlet(params)
    S = O.Space(V.knots, V.degree, V.cpts, V.wgts, 3)
    fq = O.interpolate_qp(S, params["eta"]) + np.array([0.0, 0.0, -1.0])
    A = O.Assembled(S, "elasticity", {"E": 1.0, "nu": 0.3}, pres, vals, source_qp=fq, need_full=False)
    return V, A, time.perf_counter() - t0


def cpu_time_to_solution(A, threads, runs=3):
    """Warm median of ``runs`` SciPy Jacobi-CG solves to TOL (the reference's
    restart logic, src/jaxiga/solvers/linear.py:261-321, restated in the oracle)
    on the threaded operator, with the true relative residual of the last."""
    from threadpoolctl import threadpool_limits

    from oracle import iga_oracle as O

    op = ThreadedCSR(A.K, threads)
    times = []
    with threadpool_limits(1):  # the CG's BLAS dots stay on one thread, so its threads do not spin
        for _ in range(runs):
            t0 = time.perf_counter()
            u, it = O.scipy_cg(op.op, A.b, TOL)
            times.append(time.perf_counter() - t0)
    rel = float(np.linalg.norm(A.b - A.K @ u) / np.linalg.norm(A.b))
    op.close()
    return {"seconds": float(np.median(times)), "runs": runs, "iterations": int(it), "relative_residual": rel,
            "converged": rel <= TOL, "threads": threads}


def cpu_solves(threads, spans=(CPU_SAMPLE_SPAN,), runs=3):
    out = {}
    for s in spans:
        V, A, setup = cpu_sample(s)
        out[f"elasticity3d_p3_{s}^3"] = dict(cpu_time_to_solution(A, threads, runs=runs if s == spans[0] else 1),
                                            span=s, n_dofs=V.n_dofs, nnz=int(A.K.nnz), assembly_seconds=setup)
        del A
    return out


def cpu_kv_record(steps, warmup):
    """The K.u row sample of the 64^3 workload timed on the host's threads."""
    threads = cpu_threads()
    V, K, rows, setup = cpu_row_sample()
    t = time_cpu_rows(K, threads, steps, warmup)
    value = len(rows) / float(np.mean(t))
    sample = (f"{len(rows)} whole rows ({K.nnz} nonzeros, {K.data.nbytes + K.indices.nbytes >> 20} MB) of the "
              f"64^3 elasticity operator K_ff, assembled by the oracle from the element tangents of a "
              f"{CPU_ROW_BOX[0]} x {CPU_ROW_BOX[1]} x {CPU_ROW_BOX[2]} element box (set-up {setup:.1f} s, "
              f"excluded); one step = one SciPy CSR product of those rows on {threads} threads, caches "
              f"flushed before each; DOF/s = rows per second; {INFEASIBLE}")
    return {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
            "rows": len(rows), "nnz": int(K.nnz), "setup_seconds": setup, "steps": len(t),
            "ms_per_step": float(np.mean(t)) * 1e3, "host": host_info(threads)}


def cpu_baseline(steps=20):
    rec = cpu_kv_record(steps, 1)
    rec["time_to_solution"] = cpu_solves(rec["cores"])
    return rec


def headline_config(name, span, V, n_qp, ngeo, world):
    return {"workload": workload_tag(name, span), "n_dofs": V.n_dofs, "elements": V.n_elems,
            "gauss_points": n_qp,
            "l2": "inputs larger than L2 (per-point factors %.2f GB per step)" % (8 * n_qp * ngeo / 1e9),
            "parallelism": f"replicas x{world}"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from jaxiga_b200 import workloads

    rec = cpu_kv_record(args.steps, args.warmup)
    value = rec["value"]
    V, _, _ = workloads.config2(n=N_SPAN)
    solves = cpu_solves(rec["cores"], spans=(CPU_SAMPLE_SPAN, CPU_SAMPLE_SPAN_LARGE))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": rec["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config("elasticity", N_SPAN, V, V.n_elems * 64, 10, world),
        "operator": "assembled CSR rows (SciPy), the reference's CPU path",
        "cpu_baseline": rec,
        "time_to_solution": {"tol": TOL, "scipy_jacobi_cg_true_residual_restarts": solves,
                             "full_size": INFEASIBLE},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def build_workload(name, span, dev):
    """(space, operator, load vector, learned-network features, points per element,
    (problem, parameters) for the multigrid hierarchy)."""
    import torch

    import jaxiga_b200 as jx
    from jaxiga_b200 import workloads
    from jaxiga_b200.solve import geometry_operator

    if name == "plate":
        V, problem, params = workloads.config5(n=span)
        pres, _ = problem.resolve_dirichlet(params)
        mask = np.zeros(V.n_dofs, bool)
        mask[pres] = True
        op = jx.Operator(V, "plate", problem.operator_coefficients(params)[0], prescribed=mask, want_f32=True)
        nqe = 25
        F = op.load(torch.ones(V.n_elems * nqe, dtype=torch.float64, device=dev))
        return V, op, F, None, nqe, (problem, params)
    if name == "darcy":
        V, problem, params = workloads.config4(n=span)
        a_qp = torch.exp(geometry_operator(V).interpolate(params["loga"])[..., 0]).cpu().numpy()
        pres, _ = problem.resolve_dirichlet(params)
        mask = np.zeros(V.n_dofs, bool)
        mask[pres] = True
        op = jx.Operator(V, "poisson", (1.0,), prescribed=mask, coef_qp=a_qp, want_f32=True)
        F = op.load(torch.ones(V.n_elems * 64, dtype=torch.float64, device=dev))
        loga = params["loga"]
        return V, op, F, ((loga - loga.mean()) / loga.std())[None, :], 64, (problem, {"a0": jx.PointField(a_qp)})
    V, problem, params = workloads.config2(n=span)
    pres, _ = problem.resolve_dirichlet(params)
    mask = np.zeros(V.n_dofs, bool)
    mask[pres] = True
    op = jx.Operator(V, "elasticity", (1.0, 0.3), prescribed=mask, want_f32=True)
    fq = geometry_operator(V).interpolate(params["eta"])
    fq[..., 2] -= 1.0
    F = op.load(fq)
    return V, op, F, None, 64, (problem, params)


def workload_tag(name, span):
    return f"plate2d_p4_{span}^2" if name == "plate" else f"{'darcy3d' if name == 'darcy' else 'elasticity3d'}_p3_{span}^3"


_FP64_PEAK = {}


def fp64_peak_tflops():
    """FP64 dense throughput of this GPU, measured once per run: the best of 5
    cuBLAS DGEMMs of 8192^3 (torch.matmul in float64; 2 n^3 flops), CUDA events.
    MEASURED_PEAKS.json carries HBM and BF16 peaks only; the FP64-bound brick
    kernels are compared with this."""
    if "tflops" not in _FP64_PEAK:
        import torch

        n = 8192
        a = torch.randn(n, n, dtype=torch.float64, device="cuda")
        b = torch.randn(n, n, dtype=torch.float64, device="cuda")
        c = a @ b
        best = float("inf")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(5):
            e0.record()
            torch.matmul(a, b, out=c)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        _FP64_PEAK["tflops"] = 2 * n**3 / (best * 1e-3) / 1e12
        del a, b, c
        torch.cuda.empty_cache()
    return _FP64_PEAK["tflops"]


def roofline_of(op, name, V, n_qp, x, peaks, peak_kind, span):
    """Per-kernel device times (CUDA events on the launching stream) and the
    HBM roofline of the brick kernel: algorithmic bytes = u and y once plus the
    per-point factors, 8 (2 N_dof + N_qp n_geo)."""
    n = V.n_dofs
    ms_bricks, ms_combine = op.profile_apply(x, reps=50)
    ms_b32, _ = op.profile_apply(x.float(), reps=50, f32=True)
    ngeo = op.info["ngeo"]
    alg_bytes = 8 * 2 * n + 8 * n_qp * ngeo
    alg_bytes32 = 4 * 2 * n + 4 * n_qp * ngeo
    # n_e vec 2*2*d^2 (p+1)^(d+1) + N_qp c_pt, c_pt = 2 d^4 (elasticity) or 2 d^2 (scalar)
    if name == "plate":  # 2D, p = 4: x 2.5 for the Hessian channels, 2 * 15 per point
        flops = int(V.n_elems * 2 * 2 * 4 * 5**3 * 2.5 + n_qp * 2 * 15)
    else:
        flops = V.n_elems * V.vec * (2 * 2 * 9 * 4**3 * 4) + n_qp * (2 * 81 if V.vec == 3 else 2 * 9)
    achieved = alg_bytes / (ms_bricks * 1e-3) / 1e9
    traffic = profile_traffic(name, span)
    variant = os.environ.get("JXB_BRICK3_MMA", "")
    opn = "poisson" if name == "darcy" else "elasticity"
    if name == "plate":
        kernel = "k_brick2<double,4,5,plate> (brick apply)"
    elif variant == "0":
        kernel = "k_brick3<double,3,4,%s> (FMA brick apply)" % opn
    elif variant in ("1", "2"):
        kernel = "k_brick3_mma (FP64 mma.sync brick apply, stages through shared memory, %s p=3)" % opn
    else:
        kernel = ("k_brick3_rf (FP64 mma.sync brick apply, register fragments%s, %s p=3)"
                  % (", factor tiles by bulk copy" if variant == "5" or (not variant and opn == "elasticity") else "", opn))
    return {
        "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
        "frac": achieved / peaks["hbm_gbs"], "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)",
        "traffic": None if traffic is None else traffic.get("dram_bytes_per_launch"), "kernel": kernel,
        "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": ms_bricks, "combine_ms": ms_combine,
        "fp64_tflops_achieved": flops / (ms_bricks * 1e-3) / 1e12, "flops_per_launch": flops,
        "fp64_peak_tflops": fp64_peak_tflops(), "fp64_peak_source": "measured here: cuBLAS DGEMM 8192^3",
        "fp64_frac": flops / (ms_bricks * 1e-3) / 1e12 / fp64_peak_tflops(),
        "f32_kernel_ms": ms_b32, "f32_achieved_gbs": alg_bytes32 / (ms_b32 * 1e-3) / 1e9,
    }


def _row(st, ref_x=None, x=None):
    import torch

    r = {"seconds": st["seconds"], "iterations": int(st["iterations"]),
         "relative_residual": st["relative_residual"], "converged": bool(st["converged"])}
    if ref_x is not None and x is not None:
        r["relative_difference_to_plain"] = float(torch.linalg.norm(x - ref_x) / torch.linalg.norm(ref_x))
    return r


def time_network_of(lp, reps=10):
    """Device ms of one forward of a preconditioner's network in BF16 inference
    and in FP32, on a random residual (CUDA events on the current stream)."""
    import torch

    r = torch.randn(lp.op.n_dofs, dtype=torch.float64, device=lp.dev)
    out = {}
    for mode in (True, False):
        lp.set_inference_bf16(mode)
        for _ in range(3):
            lp.forward(r)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            lp.forward(r)
        e1.record()
        torch.cuda.synchronize()
        out["bf16" if mode else "fp32"] = e0.elapsed_time(e1) / reps
    lp.set_inference_bf16(True)
    return out


def time_to_solution(name, span, op, F, feats, problem_params=None):
    """Solves to TOL, each run twice and the second reported (the first
    captures its CUDA graphs); speed-ups only for solves that converged. Set-up
    (the multigrid hierarchy, a network's weights) is not in the timed solve."""
    tts = {"tol": TOL}
    for _ in range(2):
        x_p, st_p = op.pcg(F, tol=TOL, preconditioner="jacobi", check_every=32, maxiter=80000, restarts=3)
    tts["plain_fp64_jacobi_pcg"] = dict(_row(st_p), restarts=int(st_p["outer"]))
    t_plain = st_p["seconds"] if st_p["converged"] else None
    rows = {}
    if name == "plate":
        rows["mixed"] = {"not_run": "the FP32 operator cannot resolve the biharmonic plate (condition number "
                                    "times FP32 rounding > 1): its mixed form keeps the FP64 operator and puts "
                                    "FP32 only in the preconditioner (the learned rows)"}
    else:
        for _ in range(2):
            x_m, st_m = op.refine_solve(F, tol=TOL, inner_tol=1e-3, check_every=32, maxiter=80000)
        rows["mixed_fp32_inner_fp64_refinement"] = dict(_row(st_m, x_p, x_m), outer=int(st_m["outer"]))
        for _ in range(2):
            x_r, st_r = op.mixed_pcg(F, tol=TOL, delta=1e-2, check_every=32, maxiter=80000)
        rows["mixed_fp32_pcg_reliable_fp64_updates"] = dict(_row(st_r, x_p, x_r), updates=int(st_r["outer"]))
    if problem_params is not None:
        from jaxiga_b200.multigrid import Multigrid

        deg, rng = MG_SMOOTHER.get(name, (3, 20.0))
        t0 = time.perf_counter()
        mg = Multigrid(*problem_params, degree=deg, smooth_range=rng, fine_op=op)
        mg_setup = time.perf_counter() - t0
        for _ in range(2):
            x_g, st_g = mg.solve(F, tol=TOL, maxiter=20000)
        rows["multigrid_fp64_pcg"] = dict(_row(st_g, x_p, x_g), levels=mg.levels, setup_seconds=mg_setup,
                                          smoother=f"Chebyshev-Jacobi, degree {deg}, range {rng:g}, before and after")
        mg.close()
    tts.update(rows)
    tts["learned_preconditioner"] = None
    ckpt = os.path.join(ROOT, "jaxiga_b200", "checkpoints", f"{name}{span}.npz")
    if os.path.exists(ckpt):
        from jaxiga_b200.learned import LearnedPreconditioner

        # the network's inference runs its <= 32-channel convolutions on the BF16 tensor cores
        lp = LearnedPreconditioner.from_checkpoint(op, ckpt, features=feats, inference_bf16=True)
        lrows = {}
        # FP32 operator rows only where the FP32 operator resolves the problem
        variants = [("learned_fcg_fp64", False, False), ("learned_two_level_fp64", False, True),
                    ("learned_additive_fp64", False, "additive")]
        if name != "plate":
            variants += [("mixed_learned_fcg", True, False), ("mixed_learned_two_level", True, True),
                         ("mixed_learned_additive", True, "additive")]
        for key, mixed, two in variants:
            lp.solve(F, tol=TOL, mixed=mixed, two_level=two)
            x_l, st_l = lp.solve(F, tol=TOL, mixed=mixed, two_level=two)
            lrows[key] = dict(_row(st_l, x_p, x_l), learned_iterations=int(st_l["learned_iterations"]))
        # the same additive map with the FP32 network, for comparison
        lp.set_inference_bf16(False)
        mixed_add = name != "plate"
        lp.solve(F, tol=TOL, mixed=mixed_add, two_level="additive")
        x_l, st_l = lp.solve(F, tol=TOL, mixed=mixed_add, two_level="additive")
        lrows["learned_additive_fp32_network"] = dict(_row(st_l, x_p, x_l), mixed=mixed_add,
                                                      learned_iterations=int(st_l["learned_iterations"]))
        lp.set_inference_bf16(True)
        try:
            lrows["network_forward_ms"] = dict(time_network_of(lp, reps=10), grid=list(lp.grid))
        except Exception as exc:  # timing is informative only
            lrows["network_forward_ms"] = {"error": str(exc)}
        tts["learned_preconditioner"] = {
            "checkpoint": os.path.relpath(ckpt, ROOT), "channels": list(lp.channels), "params": lp.n_params,
            "inference": "BF16 tensor-core convolutions (mma.sync m16n8k16, FP32 accumulation) on layers of <= 32 "
                         "channels, FP32 elsewhere",
            "pool_input": lp.pool_input, "additive_weight": lp.additive_weight,
            "training": "offline, python -m jaxiga_b200.train_pc (not in the timed solve)", **lrows}
        rows.update(lrows)
        lp.close()
    for k, v in rows.items():
        if isinstance(v, dict) and "seconds" in v:
            tts[f"speedup_{k}_vs_plain"] = (t_plain / v["seconds"] if t_plain and v["converged"] else None)
    best = [(k, v) for k, v in rows.items() if isinstance(v, dict) and v.get("converged")]
    if best and t_plain:
        k, v = min(best, key=lambda kv: kv[1]["seconds"])
        tts["best"] = {"form": k, "seconds": v["seconds"], "speedup_vs_plain": t_plain / v["seconds"],
                       "target_speedup": 10.0}
    return tts


def measure_workload(name, span, dev, steps, peaks, peak_kind, solve=True):
    """Apply DOF/s, roofline and time to solution of one extra workload."""
    import torch

    t0 = time.perf_counter()
    V, op, F, feats, nqe, pp = build_workload(name, span, dev)
    setup = time.perf_counter() - t0
    n_qp = V.n_elems * nqe
    x = torch.randn(V.n_dofs, dtype=torch.float64, device=dev, generator=torch.Generator(device=dev).manual_seed(7))
    y = torch.empty_like(x)
    for _ in range(3):
        op.apply(x, out=y)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        op.apply(x, out=y)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    rec = {"workload": workload_tag(name, span), "n_dofs": V.n_dofs, "elements": V.n_elems, "gauss_points": n_qp,
           "value": V.n_dofs / (ms * 1e-3), "unit": UNIT, "ms_per_apply": ms, "setup_seconds": setup,
           "roofline": roofline_of(op, name, V, n_qp, x, peaks, peak_kind, span)}
    if solve:
        rec["time_to_solution"] = time_to_solution(name, span, op, F, feats, pp)
    op.close()
    del F, x, y
    torch.cuda.empty_cache()
    return rec


def matched_gpu_solve(dev, span=CPU_SAMPLE_SPAN):
    """GPU time to solution of the CPU baseline's workload (elasticity span^3)."""
    V, op, F, _, _, _ = build_workload("elasticity", span, dev)
    for _ in range(2):
        _, st = op.pcg(F, tol=TOL, preconditioner="jacobi", check_every=32, restarts=3)
    for _ in range(2):
        _, st_r = op.mixed_pcg(F, tol=TOL, delta=1e-2, check_every=32)
    op.close()
    return {"span": span, "n_dofs": V.n_dofs, "plain_fp64_jacobi_pcg": _row(st),
            "mixed_fp32_pcg_reliable_fp64_updates": _row(st_r)}


def time_e2e(op, x, n, steps, stream, barrier, world, dev):
    """DOF/s of K.u with host input and output (see run_ours), max over ranks."""
    import torch
    import torch.distributed as dist

    xh = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    yh = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    for h in xh:
        h.copy_(x.cpu())
    xd = [torch.empty_like(x) for _ in range(2)]
    yd = [torch.empty_like(x) for _ in range(2)]
    s_in, s_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    ev_in = [torch.cuda.Event() for _ in range(2)]     # input j on the device
    ev_used = [torch.cuda.Event() for _ in range(2)]   # apply j has read xd[j] and written yd[j]
    ev_out = [torch.cuda.Event() for _ in range(2)]    # result j back on the host
    k_e2e = max(10, steps // 5)

    def step(k):
        j = k % 2
        with torch.cuda.stream(s_in):
            if k >= 2:
                s_in.wait_event(ev_used[j])
            xd[j].copy_(xh[j], non_blocking=True)
            ev_in[j].record(s_in)
        stream.wait_event(ev_in[j])
        if k >= 2:
            stream.wait_event(ev_out[j])
        op.apply(xd[j], out=yd[j])
        ev_used[j].record(stream)
        with torch.cuda.stream(s_out):
            s_out.wait_event(ev_used[j])
            yh[j].copy_(yd[j], non_blocking=True)
            ev_out[j].record(s_out)

    for k in range(4):
        step(k)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s_in.wait_event(e0)
    for k in range(k_e2e):
        step(k)
    stream.wait_event(ev_out[(k_e2e - 1) % 2])
    stream.wait_event(ev_out[k_e2e % 2])
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return world * n * k_e2e / (float(t.item()) * 1e-3), k_e2e


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    name = args.workload
    span = args.span or {"darcy": 96, "plate": 256}.get(name, N_SPAN)
    t_setup = time.perf_counter()
    V, op, F, feats, nqe, pp = build_workload(name, span, dev)
    setup_s = time.perf_counter() - t_setup
    n = V.n_dofs
    n_qp = V.n_elems * nqe
    gen = torch.Generator(device=dev).manual_seed(1234 + rank)
    x = torch.randn(n, dtype=torch.float64, device=dev, generator=gen)
    y = torch.empty_like(x)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(max(args.warmup, 3)):
        op.apply(x, out=y)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            op.apply(x, out=y)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * n * args.steps / (ms_max * 1e-3)
    peaks, peak_kind = measured_peaks()
    roofline = roofline_of(op, name, V, n_qp, x, peaks, peak_kind, span)

    # e2e through the C ABI with host buffers: every step copies its input from
    # pinned host memory to the device, applies K and copies the result back to
    # pinned host memory. The copies run on their own streams, two buffers each
    # way, so step k's input copy and step k-1's result copy overlap step k-1's
    # and step k's applies (stream order keeps every buffer's copy, apply and
    # read-back in sequence).
    e2e_value, k_e2e = time_e2e(op, x, n, args.steps, stream, barrier, world, dev)
    tts = None if args.no_solve else time_to_solution(name, span, op, F, feats, pp)
    ngeo = op.info["ngeo"]
    op.close()
    del F, x, y
    torch.cuda.empty_cache()

    extra = None
    if world == 1 and not args.no_extra and args.span is None and name == "elasticity":
        extra = {}
        for w in ("darcy", "plate"):
            extra[w] = measure_workload(w, {"darcy": 96, "plate": 256}[w], dev, max(args.steps, 20), peaks,
                                        peak_kind, solve=not args.no_solve)
        extra["batch"] = batch_record(max(args.steps, 20), rank, world, peaks, peak_kind, solve=not args.no_solve)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline()
        cpu["gpu_same_size"] = matched_gpu_solve(dev)
        cpu["gpu_same_size_24"] = matched_gpu_solve(dev, CPU_SAMPLE_SPAN_LARGE)
        g = cpu["gpu_same_size"]["plain_fp64_jacobi_pcg"]
        c = cpu["time_to_solution"][f"elasticity3d_p3_{CPU_SAMPLE_SPAN}^3"]
        cpu["time_to_solution_ratio_cpu_over_gpu"] = (c["seconds"] / g["seconds"]
                                                      if g["converged"] and c["converged"] else None)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(name, span, V, n_qp, ngeo, world),
            "operator": "matrix-free sum-factorised K.u, FP64, masked",
            "setup_seconds": setup_s,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                    "steps": k_e2e, "copies": "pinned host buffers, copy streams overlapping the applies "
                                              "(two buffers each way)"},
            "gpu_launches": 2 * args.steps,
            "roofline": roofline,
            "clocks": clocks.summary(),
            "time_to_solution": tts,
            "workloads": extra,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)


def batch_record(steps, rank, world, peaks, peak_kind, solve=True):
    """256 uneven 2D Poisson instances (quarter annuli, p in {2,3,4}, 8-128 spans per
    direction), sharded over the ranks by cost: one batched K.u over all instances
    per step, then the time to TOL of the batched PCG (one captured graph) against
    the instances solved one after another (the reference loops over its solves)."""
    import torch

    from jaxiga_b200 import _lib, workloads
    from jaxiga_b200.batch import BatchSolver
    from jaxiga_b200.dist import max_over_ranks, partition_by_cost
    from jaxiga_b200.solve import geometry_operator

    t0 = time.perf_counter()
    problems, params = workloads.config3(
        interpolate=lambda V, c: geometry_operator(V).interpolate(c).cpu().numpy())
    n_all = sum(pr.space.n_dofs for pr in problems)
    costs = [pr.space.n_elems * (pr.space.degree[0] + 1) ** 2 for pr in problems]  # Gauss points
    elems_all = sum(pr.space.n_elems for pr in problems)
    mine = partition_by_cost(costs, world)[rank]
    problems = [problems[i] for i in mine]
    params = [params[i] for i in mine]
    bs = BatchSolver(problems, params)  # 16 x 8 bricks, one launch per degree group
    setup_s = time.perf_counter() - t0
    b = bs.batch
    n = b.total
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=torch.Generator(device="cuda").manual_seed(1234 + rank))
    y = torch.empty_like(x)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def time_apply(bb, k):
        run = lambda: _lib.check(bb.lib.jxb_batch_apply(bb.handle, torch.cuda.current_stream().cuda_stream,  # noqa: E731
                                                        x.data_ptr(), y.data_ptr()))
        for _ in range(3):
            run()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(k):
            run()
        e1.record()
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), device="cuda")

    apply = lambda xx, yy: _lib.check(b.lib.jxb_batch_apply(b.handle, torch.cuda.current_stream().cuda_stream,  # noqa: E731
                                                            xx.data_ptr(), yy.data_ptr()))
    ms = time_apply(b, steps)
    # the persistent launch over every degree (32 x 8 bricks), for comparison
    os.environ["JXB_BATCH_PERSIST"] = "1"
    try:
        bs_t = BatchSolver(problems, params, tiles={p: (32, 8) for p in (1, 2, 3, 4, 5)})
    finally:
        os.environ.pop("JXB_BATCH_PERSIST", None)
    ms_groups = time_apply(bs_t.batch, steps) / steps
    groups = {"tiles": "32 x 8", "brick_launches": bs_t.batch.brick_launches,
              "persistent": bs_t.batch.persistent, "ms_per_apply": ms_groups}
    bs_t.close()
    value = n_all * steps / (ms * 1e-3)
    # algorithmic bytes: u and y once, 6 factors per point (rational 2D scalar metric)
    n_qp = sum(pr.space.n_elems * (pr.space.degree[0] + 1) ** 2 for pr in problems)
    alg = 8 * 2 * n + 8 * 6 * n_qp
    achieved = alg / (ms / steps * 1e-3) / 1e9
    # end to end: pinned host x -> device, batched apply, device y -> pinned host
    xh = torch.empty(n, dtype=torch.float64).pin_memory()
    yh = torch.empty(n, dtype=torch.float64).pin_memory()
    xh.copy_(x.cpu())
    k_e2e = max(10, steps // 5)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(k_e2e):
        x.copy_(xh, non_blocking=True)
        apply(x, y)
        yh.copy_(y, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e = n_all * k_e2e / (max_over_ranks(e0.elapsed_time(e1), device="cuda") * 1e-3)
    tts = None
    if solve:
        bs.solve(tol=TOL)  # captures the graph
        xs, sts, secs = bs.solve(tol=TOL)
        secs = max_over_ranks(secs, device="cuda")
        seq_s, seq_it = 0.0, 0
        for op, bb in zip(bs.ops, torch.split(bs.b, [op.n_dofs for op in bs.ops])):
            _, st = op.pcg(bb.contiguous(), tol=TOL, preconditioner="jacobi")
            seq_s += st["seconds"]
            seq_it += st["iterations"]
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for op, bb in zip(bs.ops, torch.split(bs.b, [op.n_dofs for op in bs.ops])):
            op.pcg(bb.contiguous(), tol=TOL, preconditioner="jacobi")
        torch.cuda.synchronize()
        seq_wall = max_over_ranks(time.perf_counter() - t1, device="cuda")
        seq_s = max_over_ranks(seq_s, device="cuda")
        tts = {"tol": TOL, "batched_pcg_one_graph": {"seconds": secs, "converged": int(sum(s["converged"] for s in sts)),
                                                      "max_iterations": int(max(s["iterations"] for s in sts))},
               "sequential_pcg_loop": {"device_seconds": seq_s, "wall_seconds": seq_wall, "iterations": seq_it},
               "speedup_batched_vs_sequential_wall": seq_wall / secs if secs > 0 else None}
    rec = {"workload": "batched_quarter_annuli_256", "instances": len(costs), "n_dofs": n_all,
           "instances_on_rank0": len(problems), "elements": elems_all, "gauss_points": sum(costs),
           "degrees": sorted({pr.space.degree[0] for pr in problems}),
           "tiles": "16 x 8 elements per brick for every degree",
           "operator": "batched matrix-free K.u, FP64, masked, " + (
               "one persistent launch over the bricks of every degree" if b.persistent else
               "%d launches (one per degree group)" % b.brick_launches),
           "persistent_launch_over_every_degree": groups,
           "parallelism": "instances sharded over %d GPU(s) by cost, no collective" % world,
           "setup_seconds": setup_s, "value": value, "unit": UNIT, "ms_per_apply": ms / steps,
           "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                   "steps": k_e2e},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": achieved / peaks["hbm_gbs"],
                        "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)", "traffic": None,
                        "kernel": ("k_brick2_persist (persistent batched 2D brick apply)" if b.persistent else
                                   "k_brick2_batch (batched 2D brick apply)") + " + k_combine_batch",
                        "algorithmic_bytes_per_launch": alg},
           "time_to_solution": tts}
    bs.close()
    torch.cuda.empty_cache()
    return rec


def run_batch(args, rank, world, local_rank):
    """The batched workload as the line's own measurement (``--workload batch``)."""
    import torch

    torch.cuda.set_device(local_rank)
    with ClockSampler(local_rank) as clk:
        rec = batch_record(args.steps, rank, world, *measured_peaks(), solve=not args.no_solve)
    if rank == 0:
        line = {
            "metric": METRIC, "value": rec["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": rec["ms_per_apply"], "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {k: rec[k] for k in ("workload", "instances", "n_dofs", "instances_on_rank0", "elements",
                                           "gauss_points", "degrees", "tiles", "operator", "parallelism",
                                           "setup_seconds")},
            "e2e": rec["e2e"], "gpu_launches": 3 * args.steps, "roofline": rec["roofline"],
            "clocks": clk.summary(), "time_to_solution": rec["time_to_solution"], "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload == "batch":
            run_batch(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
