"""Per-configuration report: the FP32 paths against the FP64 path, at the
configurations' stated run lengths.

    python -m hydrocode_astro1_b200.configs_report [--configs 0,1,2,3,4] [--out report.json]
        [--arms fp64,fp32,fp32_unet] [--weights PATH ...] [--max-steps N]

For each configuration the same initial state is stepped by the FP64 path
(the reference's arithmetic and operation order in FP64; its l_max multipole
moments in a fixed tree order) and by FP32 hydro + mixed-precision Poisson,
without and with the learned warm start (one arm per weight file, each with
the outcome monitor on).  Run lengths, as the configurations state them:

  0  Sod 64^3                    to t = 0.2
  1  n=1 polytrope 128^3         500 steps
  2  cold collapse 192^3         to t = 0.8
  3  stellar explosion 256^3     to shock breakout: the first step (checked
                                 every 50) at which the cell of largest
                                 rho * v_r (radial momentum density about the
                                 star's centre) lies at r >= R; found by the
                                 FP64 arm, the FP32 arms run its step count
                                 (with --fp64-steps N the FP64 arm stops at N
                                 and each FP32 arm finds breakout itself)
  4  two polytropes 512^3        2000 steps, FP32 arms; the FP64 arm runs the
                                 first 20 steps (its full run takes hours) for
                                 the density L1 at step 20

Reported per arm: steps, time reached, wall time; SOR iterations per solve
as per-100-step blocks (mean, median, 90th percentile); for the learned
start the accepted and fallback counts per block and the monitor's counters;
mass and total-energy drift from the FP64 totals each solver forms on the
device (hc_conservation_sums); density L1 against the FP64 arm at the same
step count; for the n=1 polytrope the central-density drift and the largest
spurious speed.
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

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
WEIGHTS = os.path.join(DATA, "unet_stellar_explosion_256.bin")
BLOCK = 100
BREAKOUT_EVERY = 50

# configuration -> (name, builder, stop rule): ("steps", n) | ("t", t_end) | ("breakout", R)
CONFIGS = {
    0: ("sod_64", lambda: problems.sod_3d(64), ("t", 0.2)),
    1: ("polytrope_n1_128", lambda: problems.polytrope_n1(128), ("steps", 500)),
    2: ("cold_collapse_192", lambda: problems.cold_collapse(192), ("t", 0.8)),
    3: ("stellar_explosion_256", lambda: problems.stellar_explosion(256), ("breakout", 0.4)),
    4: ("binary_n1_512", lambda: problems.binary_n1(512), ("steps", 2000)),
}
FP64_STEPS_CAP = {4: 20}


def solver(p, precision, warm=hc.HC_WARM_PREVIOUS):
    kw = dict(lo=p["lo"], hi=p["hi"], gamma=p["gamma"], G=p["G"], bc=p["bc"], lmax=p["lmax"], cfl=p["cfl"],
              tol=1e-8, max_iter=2_000_000, precision=precision, moment_order=hc.MOMENTS_TREE, warm_start=warm)
    return hc.HydroSolver3D(p["shape"], **kw)


def breakout_reached(q, p, R):
    """The cell of largest radial momentum density rho v_r = m . r_hat (about
    the origin, the star's centre) lies at r >= R."""
    X, Y, Z = problems.centres(p["shape"], p["lo"], p["hi"])
    r = np.sqrt(X * X + Y * Y + Z * Z)
    with np.errstate(invalid="ignore", divide="ignore"):
        mr = (q[1] * X + q[2] * Y + q[3] * Z) / np.where(r > 0, r, 1.0)
    i = np.unravel_index(np.argmax(mr), mr.shape)
    return bool(r[i] >= R), float(r[i])


def polytrope_figures(q0, q, p):
    """Hydrostatic n=1 polytrope: drift of the central density and the
    largest speed where the initial density exceeds 1e-3 of its maximum."""
    ic = tuple(n // 2 for n in p["shape"])
    star = q0[0] > 1e-3 * q0[0].max()
    speed = np.sqrt((q[1:4] ** 2).sum(0)) / np.maximum(q[0], 1e-5)
    return dict(central_density_drift=float(q[0][ic] / q0[0][ic] - 1), max_speed=float(speed[star].max()))


def blocks(values, size=BLOCK):
    out = []
    for b in range(0, len(values), size):
        v = np.asarray(values[b:b + size], dtype=float)
        out.append(dict(steps=[b + 1, b + len(v)], mean=float(v.mean()), median=float(np.median(v)),
                        p90=float(np.percentile(v, 90))))
    return out


PARTIAL_EVERY = 500


def run(q0, p, precision, stop, warm=hc.HC_WARM_PREVIOUS, weights=None, max_steps=None, log=None, snap=None,
        partial=None):
    """Steps until the stop rule holds; returns the final state and the
    record (with snap = k, also the density at step k as rec["_snap"]).
    partial(rec), when given, receives the record so far every
    PARTIAL_EVERY steps (a run cut short keeps its blocks)."""
    kind, val = stop
    s = solver(p, precision, warm)
    if warm == hc.HC_WARM_UNET:
        s.unet_load_file(weights)
        s.unet_guard(3)
    s.set_state(q0)
    s.set_conservation_record(True)
    c0 = s.conservation()
    t, n, iters, acc, fb = 0.0, 0, [], [], []
    breakout_r = None
    snap_rho = None
    t0 = time.time()
    d_prev = s.diagnostics()
    while True:
        if kind == "steps" and n >= val:
            break
        if kind == "t" and t >= val:
            break
        if max_steps is not None and n >= max_steps:
            break
        t += float(s.step(1)[0])
        n += 1
        d = s.diagnostics()
        if p["G"] > 0:
            iters.append(d["last_iterations"])
            acc.append(d["unet_accepted"] - d_prev["unet_accepted"])
            fb.append(d["unet_fallbacks"] - d_prev["unet_fallbacks"])
        d_prev = d
        if snap is not None and n == snap:
            snap_rho = s.state()[0]
        if kind == "breakout" and n % BREAKOUT_EVERY == 0:
            hit, rr = breakout_reached(s.state(), p, val)
            if hit:
                breakout_r = rr
                break
        if log and n % 100 == 0:
            log(f"  step {n}, t {t:.5f}, {time.time() - t0:.0f} s")
        if partial and n % PARTIAL_EVERY == 0 and iters:
            partial(dict(steps=n, t=t, wall_s=time.time() - t0, partial=True, sor_iterations_blocks=blocks(iters),
                         sor_iterations_mean=float(np.mean(iters))))
    c1 = np.array(d_prev["cons"]) if n > 0 else c0
    q = s.state()
    d = s.diagnostics()
    s.close()
    rec = dict(steps=n, t=t, wall_s=time.time() - t0,
               mass_drift=float(c1[0] / c0[0] - 1.0), energy_drift=float(c1[4] / c0[4] - 1.0),
               drift_source="hc_conservation_sums (FP64, on the device)")
    if iters:
        rec["sor_iterations_blocks"] = blocks(iters)
        rec["sor_iterations_mean"] = float(np.mean(iters))
        rec["sor_iterations_total"] = int(np.sum(iters))
    if warm == hc.HC_WARM_UNET:
        accb = [dict(steps=b["steps"], accepted=int(np.sum(acc[b["steps"][0] - 1:b["steps"][1]])),
                     fallbacks=int(np.sum(fb[b["steps"][0] - 1:b["steps"][1]]))) for b in blocks(iters)]
        rec.update(unet_accepted=d["unet_accepted"], unet_fallbacks=d["unet_fallbacks"],
                   accepted_blocks=accb,
                   monitor=dict(probes=d["unet_probes"], wins=d["unet_wins"], losses=d["unet_losses"],
                                switch_offs=d["unet_switch_offs"], off_at_end=d["unet_off"]))
    if breakout_r is not None:
        rec["breakout_radius"] = breakout_r
    if snap_rho is not None:
        rec["_snap"] = snap_rho
    return q, rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", default="0,1,2,3,4")
    ap.add_argument("--arms", default="fp64,fp32,fp32_unet")
    ap.add_argument("--weights", nargs="*", default=None,
                    help="weight files of the learned start (one fp32_unet arm each; default: the committed one)")
    ap.add_argument("--max-steps", type=int, default=None, help="cap every run at this many steps")
    ap.add_argument("--fp64-steps", type=int, default=None,
                    help="cap the FP64 arm at this many steps (the FP32 arms then run their own stop rule and "
                         "the density L1 is taken at that step)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    arms = a.arms.split(",")
    weights = a.weights or [WEIGHTS]

    def log(m):
        print(m, file=sys.stderr, flush=True)

    out = []

    def save(recs):   # after every arm: a long run that is cut short keeps what it finished
        if a.out:
            with open(a.out, "w") as f:
                json.dump(recs, f, indent=1)

    for c in [int(x) for x in a.configs.split(",")]:
        name, build, stop = CONFIGS[c]
        q0, p = build()
        rec = dict(config=c, name=name, shape=list(p["shape"]), stop=list(stop))
        q64 = None
        steps = None
        if "fp64" in arms:
            cap = a.fp64_steps or FP64_STEPS_CAP.get(c, a.max_steps)
            log(f"[{name}] fp64")
            q64, r64 = run(q0, p, hc.FP64, stop, max_steps=cap, log=log)
            if c == 1:
                r64.update(polytrope_figures(q0, q64, p))
            rec["fp64"] = r64
            steps = r64["steps"]
            save(out + [rec])
        capped = c in FP64_STEPS_CAP or a.fp64_steps is not None
        fp32_stop = ("steps", steps) if (steps is not None and not capped) else stop
        for arm in arms:
            if arm == "fp64":
                continue
            unet = arm == "fp32_unet"
            if unet and not (p["G"] > 0 and all(n % 32 == 0 for n in p["shape"])):
                continue
            for wf in (weights if unet else [None]):
                tag = arm if not unet or len(weights) == 1 else f"{arm}:{os.path.basename(wf)}"
                log(f"[{name}] {tag}")
                snap = rec["fp64"]["steps"] if (q64 is not None and capped) else None
                def keep(part, tag=tag):
                    rec[tag] = part
                    save(out + [rec])

                q32, r32 = run(q0, p, hc.FP32, fp32_stop, hc.HC_WARM_UNET if unet else hc.HC_WARM_PREVIOUS, wf,
                               max_steps=a.max_steps, log=log, snap=snap, partial=keep)
                rho_snap = r32.pop("_snap", None)
                if q64 is not None and r32["steps"] == rec["fp64"]["steps"]:
                    r32["density_l1"] = float(np.abs(q32[0] - q64[0]).mean() / np.abs(q64[0]).mean())
                elif q64 is not None and rho_snap is not None:
                    r32["density_l1"] = float(np.abs(rho_snap - q64[0]).mean() / np.abs(q64[0]).mean())
                    r32["density_l1_at_step"] = snap
                if unet:
                    with open(wf, "rb") as f:
                        r32["weights"] = dict(file=os.path.basename(wf),
                                              sha256=hashlib.sha256(f.read()).hexdigest()[:16])
                if c == 1:
                    r32.update(polytrope_figures(q0, q32, p))
                rec[tag] = r32
                del q32
                save(out + [rec])
        print(json.dumps(rec), flush=True)
        out.append(rec)
        del q64
        save(out)


if __name__ == "__main__":
    main()
