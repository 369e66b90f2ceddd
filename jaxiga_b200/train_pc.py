"""Train the learned preconditioner for a benchmark workload on the GPU.

    python -m jaxiga_b200.train_pc --workload darcy --out pc.npz [--pairs 2000] [--seconds 600]

Pairs come from plain FP64 Jacobi-PCG solves of the workload itself (the load
vector first, then seeded random right-hand sides), one (residual, error)
pair per iteration, plus ``--random`` pairs (r ~ N(0, I), e = K^-1 r); training minimises the energy norm of the
preconditioner's error with the network's own forward/backward kernels and
Adam until the time budget is spent; the checkpoint (weights, scales, loss
history, the fitted weight of the additive two-level map) is written to
``--out``. ``--pool-input`` trains a network that runs on the pooled
(half-resolution) residual. Then the workload is solved to 1e-8 by plain
FP64 Jacobi-PCG, by flexible CG with the network alone, with the
multiplicative and the additive two-level maps (FP64 and mixed precision),
and by the flexible CG without the network, and one JSON line with the
training record and the solves is printed.
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
    elif workload == "plate":
        V, problem, params = workloads.config5(n=span or 256)
        pres, _ = problem.resolve_dirichlet(params)
        mask = np.zeros(V.n_dofs, bool)
        mask[pres] = True
        op = jx.Operator(V, "plate", problem.operator_coefficients(params)[0], prescribed=mask, want_f32=True)
        F = op.load(torch.ones(V.n_elems * 25, dtype=torch.float64, device=op.device))
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
    ap.add_argument("--workload", choices=["elasticity", "darcy", "plate"], default="elasticity")
    ap.add_argument("--span", type=int, default=None)
    ap.add_argument("--pairs", type=int, default=2000, help="pairs from the iterates of Jacobi-PCG solves")
    ap.add_argument("--random", type=int, default=0, help="extra pairs (r ~ N(0, I), K^-1 r)")
    ap.add_argument("--seconds", type=float, default=600.0)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--channels", default=None, help="per-level channels, e.g. 8,16,24,32,48 (default: by grid)")
    ap.add_argument("--epochs", type=int, default=1000)
    ap.add_argument("--depth", type=int, default=4)
    ap.add_argument("--out", required=True)
    ap.add_argument("--pool-input", action="store_true", help="network on the pooled (half-resolution) residual")
    ap.add_argument("--loss", choices=["angle", "additive"], default="angle",
                    help="energy angle of the network's output, or of the additive two-level map n + D^-1 r")
    ap.add_argument("--seed", type=int, default=20260901)
    args = ap.parse_args()
    t0 = time.time()
    V, op, F, features = build(args.workload, args.span)
    channels = None if args.channels is None else tuple(int(c) for c in args.channels.split(","))
    lp = LearnedPreconditioner(op, features=features, channels=channels, seed=args.seed, pool_input=args.pool_input)
    gen = torch.Generator(device=op.device).manual_seed(args.seed)
    Rs, Es, solves_data = [], [], []
    have = 0
    k = 0
    while have < args.pairs:
        b = F if k == 0 else torch.randn(V.n_dofs, dtype=torch.float64, device=op.device, generator=gen)
        R, E, st = lp.pairs_from_solve(b, n_pairs=args.pairs - have, every=1, tol=1e-10)
        Rs.append(R)
        Es.append(E)
        have += R.shape[0]
        solves_data.append({"iterations": st["iterations"], "pairs": int(R.shape[0])})
        k += 1
    if args.random > 0:  # white-noise residuals r ~ N(0, I), e = K^-1 r
        R2, E2 = lp.pairs_random(args.random, tol=1e-10, seed=args.seed)
        Rs.append(R2)
        Es.append(E2)
        have += R2.shape[0]
    R = torch.cat(Rs)
    E = torch.cat(Es)
    # one global output scale over all solves
    free = int(op.info["n_free"])
    lp.out_scale = float(torch.sqrt((E.double() ** 2).sum() / (R.shape[0] * free)))
    t_data = time.time() - t0
    t1 = time.time()
    ep = 0
    while time.time() - t1 < args.seconds and ep < args.epochs:
        lr = args.lr if ep < 4 else args.lr / 3
        lp.train(R, E, epochs=1, lr=lr, batch=4, seed=ep, loss=args.loss)
        ep += 1
    t_train = time.time() - t1
    if args.loss == "additive":
        lp.additive_weight = 1.0  # trained as n + D^-1 r: the combination is the one learned
    else:  # trained alone (n ~ e up to scale): the energy-optimal weight of n beside D^-1 r
        idx = torch.linspace(0, R.shape[0] - 1, min(64, R.shape[0]), device=R.device).long()
        lp.fit_additive_weight(R[idx], E[idx], n_pairs=64)
    lp.save(args.out)
    del R, E
    solves = {}
    x_ref, st = op.pcg(F, tol=1e-8, preconditioner="jacobi")
    solves["plain_fp64_jacobi_pcg"] = st
    _, st = lp.solve(F, tol=1e-8, depth=args.depth)
    solves["learned_fcg_fp64"] = st
    x_m, st = lp.solve(F, tol=1e-8, depth=args.depth, mixed=True)
    st["relative_difference_to_plain"] = float(torch.linalg.norm(x_m - x_ref) / torch.linalg.norm(x_ref))
    solves["learned_fcg_mixed"] = st
    _, st = lp.solve(F, tol=1e-8, depth=args.depth, two_level=True)
    solves["learned_fcg_two_level"] = st
    _, st = lp.solve(F, tol=1e-8, depth=args.depth, two_level=True, mixed=True)
    solves["learned_fcg_two_level_mixed"] = st
    _, st = lp.solve(F, tol=1e-8, depth=args.depth, two_level="additive")
    solves["learned_fcg_additive"] = st
    _, st = lp.solve(F, tol=1e-8, depth=args.depth, two_level="additive", mixed=True)
    solves["learned_fcg_additive_mixed"] = st
    _, st = lp.solve(F, tol=1e-8, depth=args.depth, use_network=False)
    solves["fcg_jacobi_only"] = st
    # network inference time on its own
    r = torch.randn(V.n_dofs, dtype=torch.float64, device=op.device)
    for _ in range(3):
        lp.forward(r)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        lp.forward(r)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"workload": args.workload, "n_dofs": V.n_dofs, "pairs": int(have), "channels": lp.channels,
                      "solves_for_pairs": solves_data, "data_seconds": t_data, "train_seconds": t_train,
                      "epochs": ep, "loss_first": lp.history[0], "loss_last": lp.history[-1],
                      "pool_input": lp.pool_input, "additive_weight": lp.additive_weight, "loss": args.loss,
                      "params": lp.n_params, "forward_ms": e0.elapsed_time(e1) / 10, "solves": solves,
                      "checkpoint": args.out}))


if __name__ == "__main__":
    main()
