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


def solver(q, p, warm=hc.HC_WARM_PREVIOUS, weights=None):
    s = hc.HydroSolver3D(p["shape"], lo=p["lo"], hi=p["hi"], gamma=p["gamma"], G=p["G"], bc=p["bc"],
                         lmax=p["lmax"], cfl=p["cfl"], tol=1e-8, max_iter=2_000_000, precision=hc.FP32,
                         moment_order=hc.MOMENTS_TREE, warm_start=warm)
    if weights:
        s.unet_load_file(weights)
    s.set_state(q)
    return s


def _list(v, n, cast):
    parts = [cast(x) for x in str(v).split(",")]
    if len(parts) == 1:
        parts = parts * n
    if len(parts) != n:
        raise SystemExit(f"expected 1 or {n} comma-separated values, got {v}")
    return parts


def collect(problem, n, seed, solves, every, skip, cycles, init_seed, with_weights=None):
    """A run of the problem that records `solves` samples per recorded cycle,
    one every `every` solves after `skip` unrecorded ones.  The run uses the
    plain solver, or (with_weights) the learned start with those weights,
    which reaches late steps sooner; a sample is the same either way: the
    normalised first residual from the previous potential and the converged
    correction of that potential."""
    q, p = make(problem, n, seed)
    if with_weights:
        s = solver(q, p, hc.HC_WARM_UNET, with_weights)
        params = s.unet_params()
        s.unet_collect(solves * len(cycles) + 1)
        s.unet_init(init_seed)              # training starts from a fresh network ...
        fresh = s.unet_params()
        s.unet_load(params[0], params[1])   # ... the run uses the given one
    else:
        s = solver(q, p)
        s.unet_collect(solves * len(cycles) + 1)
        s.unet_init(init_seed)
        fresh = None
    iters = []
    for _ in range(skip):
        s.unet_record_cycle(0)
        s.step(1)
        iters.append(s.diagnostics()["last_iterations"])
    for c in cycles:
        for _ in range(solves):
            for k in range(every):
                s.unet_record_cycle(c if k == every - 1 else 0)
                s.step(1)
                iters.append(s.diagnostics()["last_iterations"])
    if fresh is not None:
        s.unet_load(fresh[0], fresh[1])
    return s, iters


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--problem", default="stellar_explosion",
                    help="problem, or comma-separated problems trained on together")
    ap.add_argument("--n", default="256", help="grid cells per side (one value, or one per problem)")
    ap.add_argument("--seed", default="7", help="density-noise seed of the explosion (one, or per problem)")
    ap.add_argument("--solves", default="25", help="samples per recorded cycle (one, or per problem)")
    ap.add_argument("--train-steps", type=int, default=2000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--init-seed", type=int, default=1)
    ap.add_argument("--record-cycles", default="1",
                    help="correction cycles to record, `solves` steps each, in this order")
    ap.add_argument("--record-every", default="1",
                    help="record every k-th solve (k - 1 unrecorded steps between samples), so that "
                         "`solves` samples span solves x k steps of the run (one, or per problem)")
    ap.add_argument("--skip", default="0", help="unrecorded steps before the first sample (one, or per problem)")
    ap.add_argument("--collect-with", default=None, metavar="WEIGHTS",
                    help="run the collection with the learned start from this weight file (faster late in a run)")
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    t0 = time.time()
    probs = a.problem.split(",")
    m = len(probs)
    ns, seeds = _list(a.n, m, int), _list(a.seed, m, int)
    solves, every, skip = _list(a.solves, m, int), _list(a.record_every, m, int), _list(a.skip, m, int)
    cycles = [int(c) for c in a.record_cycles.split(",")]
    runs = [collect(probs[q], ns[q], seeds[q], solves[q], every[q], skip[q], cycles, a.init_seed, a.collect_with)
            for q in range(m)]
    t_collect = time.time() - t0
    losses = []
    nchunk = 10 * m
    chunk = max(1, a.train_steps // nchunk)
    # one linearly decaying learning rate over all steps, in chunks (each a
    # cosine cycle); with several problems the chunks alternate between their
    # sample rings, the parameters handed from one context to the next
    done = 0
    lr = a.lr
    cur = 0
    params = None
    while done < a.train_steps:
        k = min(chunk, a.train_steps - done)
        s = runs[cur][0]
        if params is not None and m > 1:
            s.unet_load(params[0], params[1])
        losses.append(s.unet_train(k, lr=lr * (1.0 - done / a.train_steps), seed=1000 + done))
        if m > 1:
            params = s.unet_params()
        done += k
        cur = (cur + 1) % m
    t_train = time.time() - t0 - t_collect
    last = runs[(cur - 1) % m][0]
    last.unet_save_file(a.out)
    tm = last.timing()
    report = {"problem": probs, "n": ns, "seed": seeds, "solves": solves, "record_cycles": cycles,
              "record_every": every, "skip": skip, "collected_with": a.collect_with,
              "samples": [r[0].unet_samples() for r in runs],
              "sor_iterations": [r[1] for r in runs], "train_steps": a.train_steps, "lr": a.lr,
              "init_seed": a.init_seed,
              "loss_per_chunk": losses, "collect_s": t_collect, "train_s": t_train,
              "unet_device_ms": tm["unet_ms"], "params": hc.lib().hc_unet_param_count()}
    with open(os.path.splitext(a.out)[0] + ".json", "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps(report))
    for r in runs:
        r[0].close()


if __name__ == "__main__":
    main()
