"""Single-kernel cases of the benchmark workload, for timing and profiling.

    python -m hydrocode_astro1_b200.kernel_cases hydro N STEPS
    python -m hydrocode_astro1_b200.kernel_cases sor N ITERATIONS [SOR_DEPTH]
    python -m hydrocode_astro1_b200.kernel_cases stream N

`hydro`: the N^3 stellar explosion in FP32 with self-gravity, its Poisson
solve capped at 2 iterations (it does not converge, so g stays the last
converged potential's, zero), STEPS timed steps after 2 untimed ones; prints
the fused hydro kernel's time per launch (CUDA events) and its algorithmic
bandwidth (48 bytes per interior cell).  Few launches precede the hydro
kernels, so an ncu capture of one of them starts at once.

`sor`: two FP32 mixed-precision solves of the explosion's first state from
a cold start, each capped at ITERATIONS correction iterations; prints the
second solve's colour sweeps' time per iteration and algorithmic bandwidth
(6 bytes per interior cell and sweep).

`stream`: the bandwidth a plain streaming kernel reaches for one colour
sweep's transfer at N^3 -- three FP32 arrays of N^3/2 read, one written
(torch.addcmul, a library kernel timed here only as a reference point for
the sweep) -- 50 launches back to back, CUDA events around them.
"""
from __future__ import annotations

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402

import hydrocode_astro1_b200 as hc  # noqa: E402
from hydrocode_astro1_b200 import problems  # noqa: E402


def solver(n, **kw):
    q, p = problems.stellar_explosion(n)
    s = hc.HydroSolver3D(p["shape"], lo=p["lo"], hi=p["hi"], gamma=p["gamma"], G=1.0, bc=p["bc"], lmax=8,
                         cfl=p["cfl"], tol=1e-30, precision=hc.FP32, moment_order=hc.MOMENTS_TREE, **kw)
    s.set_state(q)
    return s


def hydro(n, steps):
    s = solver(n, max_iter=2)
    s.step(2)
    s.timing(reset=True)
    s.step(steps)
    t = s.timing()
    ms = t["hydro_ms"] / max(1, t["hydro_launches"])
    print(f"hydro n={n}: {ms * 1e3:.1f} us per launch, {48 * (n - 2) ** 3 / (ms * 1e-3) / 1e9:.0f} GB/s algorithmic; "
          f"state finite: {bool(np.isfinite(s.state()).all())}", flush=True)
    s.close()


def sor(n, iters, depth=0):
    s = solver(n, max_iter=iters, sor_depth=depth)
    s.gravity_solve()
    s.timing(reset=True)
    s.gravity_solve()
    t = s.timing()
    it = s.diagnostics()["last_iterations"]
    per = t["sor_ms"] / max(1, it)
    print(f"sor n={n} sor_depth={depth}: {it} iterations, {per * 1e3:.1f} us per iteration, "
          f"{6 * (n - 2) ** 3 / (per / 2 * 1e-3) / 1e9:.0f} GB/s algorithmic per sweep", flush=True)
    s.close()


def stream(n):
    import torch
    m = n * n * n // 2
    x, y, z = (torch.rand(m, device="cuda") for _ in range(3))
    out = torch.empty_like(x)
    for _ in range(5):
        torch.addcmul(x, y, z, out=out)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(50):
        torch.addcmul(x, y, z, out=out)
    e1.record()
    torch.cuda.synchronize()
    per = e0.elapsed_time(e1) / 50
    print(f"stream n={n}: {per * 1e3:.1f} us per launch, {16 * m / (per * 1e-3) / 1e9:.0f} GB/s "
          f"({16 * m / 1e6:.0f} MB per launch)", flush=True)


if __name__ == "__main__":
    what = sys.argv[1]
    if what == "hydro":
        hydro(int(sys.argv[2]), int(sys.argv[3]))
    elif what == "sor":
        sor(int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4]) if len(sys.argv) > 4 else 0)
    elif what == "stream":
        stream(int(sys.argv[2]))
    else:
        raise SystemExit("usage: kernel_cases hydro N STEPS | sor N ITERATIONS [SOR_DEPTH] | stream N")
