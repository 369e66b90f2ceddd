"""Train the learned preconditioner for a benchmark workload on the GPU.

    python -m jaxiga_b200.train_pc --workload elasticity --out pc.npz [--pairs 2000] [--seconds 600]

Pairs come from plain FP64 Jacobi-PCG solves of the workload itself (the load
vector first, then seeded random right-hand sides), one (residual, error)
pair per iteration; training runs the network's own forward/backward kernels
and Adam until the time budget is spent; the checkpoint (weights, scales,
loss history) is written to ``--out``. A JSON line with the training record
is printed.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np


def build(workload, span=None):
    import torch

    import jaxiga_b200 as jx
    from jaxiga_b200 import workloads
    from jaxiga_b200.solve import geometry_operator

    if workload == "elasticity":
        V, problem, params = workloads.config2(n=span or 64)
        pres, _ = problem.resolve_dirichlet(params)
        mask = np.zeros(V.n_dofs, bool)
        mask[pres] = True
        op = jx.Operator(V, "elasticity", (1.0, 0.3), prescribed=mask, want_f32=True)
        fq = geometry_operator(V).interpolate(params["eta"])
        fq[..., 2] -= 1.0
        F = op.load(fq)
        features = None
    else:
        V, problem, params = workloads.config4(n=span or 96)
        a = torch.exp(geometry_operator(V).interpolate(params["loga"])[..., 0]).cpu().numpy()
        pres, _ = problem.resolve_dirichlet(params)
        mask = np.zeros(V.n_dofs, bool)
        mask[pres] = True
        op = jx.Operator(V, "poisson", (1.0,), prescribed=mask, coef_qp=a, want_f32=True)
        F = op.load(torch.ones(V.n_elems * 64, dtype=torch.float64, device=op.device))
        loga = params["loga"]
        features = ((loga - loga.mean()) / loga.std())[None, :]
    return V, op, F, features


def main():
    import torch

    from jaxiga_b200.learned import LearnedPreconditioner

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["elasticity", "darcy"], default="elasticity")
    ap.add_argument("--span", type=int, default=None)
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--seconds", type=float, default=600.0)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--channels", default="8,16,48")
    ap.add_argument("--out", required=True)
    ap.add_argument("--seed", type=int, default=20260901)
    args = ap.parse_args()
    t0 = time.time()
    V, op, F, features = build(args.workload, args.span)
    lp = LearnedPreconditioner(op, features=features, channels=tuple(int(c) for c in args.channels.split(",")),
                               seed=args.seed)
    gen = torch.Generator(device=op.device).manual_seed(args.seed)
    Rs, Es, solves = [], [], []
    have = 0
    k = 0
    while have < args.pairs:
        b = F if k == 0 else torch.randn(V.n_dofs, dtype=torch.float64, device=op.device, generator=gen)
        R, E, st = lp.pairs_from_solve(b, n_pairs=args.pairs - have, every=1, tol=1e-10)
        Rs.append(R)
        Es.append(E)
        have += R.shape[0]
        solves.append({"iterations": st["iterations"], "pairs": int(R.shape[0])})
        k += 1
    R = torch.cat(Rs)
    E = torch.cat(Es)
    # one global output scale over all solves
    free = int(op.info["n_free"])
    lp.out_scale = float(torch.sqrt((E.double() ** 2).sum() / (R.shape[0] * free)))
    t_data = time.time() - t0
    t1 = time.time()
    ep = 0
    while time.time() - t1 < args.seconds:
        lr = args.lr if ep < 4 else args.lr / 3
        lp.train(R, E, epochs=1, lr=lr, batch=4, seed=ep)
        ep += 1
    lp.save(args.out)
    print(json.dumps({"workload": args.workload, "n_dofs": V.n_dofs, "pairs": int(R.shape[0]), "solves": solves,
                      "data_seconds": t_data, "train_seconds": time.time() - t1, "epochs": ep,
                      "loss_first": lp.history[0], "loss_last": lp.history[-1], "params": lp.n_params,
                      "checkpoint": args.out}))


if __name__ == "__main__":
    main()
