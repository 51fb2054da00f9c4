"""Train the warm-start U-Net on the GPU from solves of the plain solver.

    python -m hydrocode_astro1_b200.train_unet --problem stellar_explosion --n 256 --seed 7 \\
        --solves 60 --train-steps 9000 --out hydrocode_astro1_b200/data/unet_stellar_explosion_256.bin

Runs `solves` steps of the problem in FP32 + mixed precision with the
previous-potential warm start (the plain method) for each recorded cycle,
recording one (residual, converged correction) pair per Poisson solve on the
device -- the residual at the start of the first correction cycle (after the
hydro update) or of the second (the smooth remainder the first cycle's sweeps
left), the correction from there to the converged potential; then trains the
network on those pairs with the library's own tensor-core forward/backward
kernels and Adam (hc_unet_train), and writes the weight file plus a JSON
report (same name, .json) with the training losses.  The density noise seed
of the training run differs from the benchmark's (42), so the benchmark
evaluates the network on a realisation it has not seen.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import hydrocode_astro1_b200 as hc  # noqa: E402
from hydrocode_astro1_b200 import problems  # noqa: E402


def make(problem, n, seed):
    if problem == "stellar_explosion":
        return problems.stellar_explosion(n, seed=seed)
    if problem == "polytrope_n1":
        return problems.polytrope_n1(n)
    if problem == "cold_collapse":
        return problems.cold_collapse(n)
    raise SystemExit(f"unknown problem {problem}")


def solver(q, p, warm=hc.HC_WARM_PREVIOUS):
    s = hc.HydroSolver3D(p["shape"], lo=p["lo"], hi=p["hi"], gamma=p["gamma"], G=p["G"], bc=p["bc"],
                         lmax=p["lmax"], cfl=p["cfl"], tol=1e-8, max_iter=2_000_000, precision=hc.FP32,
                         moment_order=hc.MOMENTS_TREE, warm_start=warm)
    s.set_state(q)
    return s


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--problem", default="stellar_explosion")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--solves", type=int, default=25)
    ap.add_argument("--train-steps", type=int, default=2000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--init-seed", type=int, default=1)
    ap.add_argument("--record-cycles", default="1",
                    help="correction cycles to record, `solves` steps each, in this order")
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    t0 = time.time()
    q, p = make(a.problem, a.n, a.seed)
    s = solver(q, p)
    cycles = [int(c) for c in a.record_cycles.split(",")]
    s.unet_collect(a.solves * len(cycles) + 1)
    s.unet_init(a.init_seed)
    iters = []
    for c in cycles:
        s.unet_record_cycle(c)
        for _ in range(a.solves):
            s.step(1)
            iters.append(s.diagnostics()["last_iterations"])
    t_collect = time.time() - t0
    losses = []
    chunk = max(1, a.train_steps // 10)
    # one cosine schedule over all steps, reported in ten chunks
    done = 0
    lr = a.lr
    while done < a.train_steps:
        k = min(chunk, a.train_steps - done)
        losses.append(s.unet_train(k, lr=lr * (1.0 - done / a.train_steps), seed=1000 + done))
        done += k
    t_train = time.time() - t0 - t_collect
    s.unet_save_file(a.out)
    tm = s.timing()
    report = {"problem": a.problem, "n": a.n, "seed": a.seed, "solves": a.solves, "record_cycles": cycles,
              "samples": s.unet_samples(),
              "sor_iterations": iters, "train_steps": a.train_steps, "lr": a.lr,
              "loss_per_chunk": losses, "collect_s": t_collect, "train_s": t_train,
              "unet_device_ms": tm["unet_ms"], "params": hc.lib().hc_unet_param_count()}
    with open(os.path.splitext(a.out)[0] + ".json", "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps(report))
    s.close()


if __name__ == "__main__":
    main()
