"""Accuracy report of the FP32 paths against the bit-exact FP64 path, per
benchmark configuration.

    python -m hydrocode_astro1_b200.configs_report [--configs 0,1,2,3,4] [--out report.json]

For each configuration the same initial state is stepped by the FP64 path
(bit-identical to the reference C code, so it stands in for the FP64 oracle
at these sizes) and by FP32 hydro + mixed-precision Poisson (and, where a
trained network applies, with the learned warm start).  Reported per run:
density L1 against FP64, relative mass and total-energy drift of each
path, SOR iterations, and for the n=1 polytrope the central-density drift
and the largest spurious speed; for the learned start the accepted and
fallback counts.  Step counts are bounded so the whole report runs in a few
minutes on one B200 (the long runs of the configurations -- t = 0.8,
shock breakout, 2000 steps -- are not repeated here).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import hydrocode_astro1_b200 as hc  # noqa: E402
from hydrocode_astro1_b200 import problems  # noqa: E402

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "unet_stellar_explosion_256.bin")

# configuration -> (name, builder, steps, t_end): run `steps` steps, or to t_end when given
CONFIGS = {
    0: ("sod_64", lambda: problems.sod_3d(64), None, 0.2),
    1: ("polytrope_n1_128", lambda: problems.polytrope_n1(128), 100, None),
    2: ("cold_collapse_192", lambda: problems.cold_collapse(192), 60, None),
    3: ("stellar_explosion_256", lambda: problems.stellar_explosion(256), 30, None),
    4: ("binary_n1_512", lambda: problems.binary_n1(512), 5, None),
}


def solver(p, precision, warm=hc.HC_WARM_PREVIOUS):
    kw = dict(lo=p["lo"], hi=p["hi"], gamma=p["gamma"], G=p["G"], bc=p["bc"], lmax=p["lmax"], cfl=p["cfl"],
              tol=1e-8, max_iter=2_000_000, precision=precision, moment_order=hc.MOMENTS_TREE, warm_start=warm)
    return hc.HydroSolver3D(p["shape"], **kw)


def run(q0, p, precision, steps, t_end, warm=hc.HC_WARM_PREVIOUS):
    s = solver(p, precision, warm)
    if warm == hc.HC_WARM_UNET:
        s.unet_load_file(WEIGHTS)
    s.set_state(q0)
    t, n, iters = 0.0, 0, []
    t0 = time.time()
    while (t_end is None and n < steps) or (t_end is not None and t < t_end):
        t += float(s.step(1)[0])
        n += 1
        if p["G"] > 0:
            iters.append(s.diagnostics()["last_iterations"])
    q = s.state()
    d = s.diagnostics()
    s.close()
    return q, dict(steps=n, t=t, wall_s=time.time() - t0, sor_iterations=iters,
                   unet_accepted=d["unet_accepted"], unet_fallbacks=d["unet_fallbacks"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", default="0,1,2,3,4")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    out = []
    for c in [int(x) for x in a.configs.split(",")]:
        name, build, steps, t_end = CONFIGS[c]
        q0, p = build()
        dV = np.prod([(p["hi"][t] - p["lo"][t]) / p["shape"][t] for t in range(3)])
        m0, e0 = q0[0].sum() * dV, q0[4].sum() * dV
        q64, r64 = run(q0, p, hc.FP64, steps, t_end)
        arms = [("fp32", hc.HC_WARM_PREVIOUS)]
        if p["G"] > 0 and all(n % 32 == 0 for n in p["shape"]) and os.path.exists(WEIGHTS):
            arms.append(("fp32_unet", hc.HC_WARM_UNET))
        rec = dict(config=c, name=name, shape=list(p["shape"]), fp64=dict(r64, mass_drift=float(q64[0].sum() * dV / m0 - 1),
                                                                          energy_drift=float(q64[4].sum() * dV / e0 - 1)))
        for arm, warm in arms:
            q32, r32 = run(q0, p, hc.FP32, r64["steps"], None, warm)
            rec[arm] = dict(r32, density_l1=float(np.abs(q32[0] - q64[0]).mean() / np.abs(q64[0]).mean()),
                            mass_drift=float(q32[0].sum() * dV / m0 - 1),
                            energy_drift=float(q32[4].sum() * dV / e0 - 1))
            if warm == hc.HC_WARM_UNET:   # which network the learned-start figures belong to
                with open(WEIGHTS, "rb") as f:
                    rec[arm]["weights"] = dict(file=os.path.basename(WEIGHTS),
                                               sha256=hashlib.sha256(f.read()).hexdigest()[:16])
            if c == 1:   # hydrostatic n=1 polytrope: central density and spurious velocities
                ic = tuple(n // 2 for n in p["shape"])
                for tag, q in (("fp64", q64), (arm, q32)):
                    rec[tag]["central_density_drift"] = float(q[0][ic] / q0[0][ic] - 1)
                    rec[tag]["max_speed"] = float((np.sqrt((q[1:4] ** 2).sum(0)) / np.maximum(q[0], 1e-5))[
                        q0[0] > 1e-3 * q0[0].max()].max())
            del q32
        print(json.dumps(rec), flush=True)
        out.append(rec)
        del q64
    if a.out:
        with open(a.out, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
