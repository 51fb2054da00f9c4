"""Generates the golden fixtures of tests/golden/ by running the REFERENCE
itself (oracle/_ref/libhcref.so, built from the reference sources by
oracle/Makefile).  Needs the reference tree at build time; the fixtures are
committed so the tests do not.

  small.npz         full end states of short runs on small grids (Sod 12^3,
                    a moving random state with mixed boundaries, a
                    self-gravitating polytrope with SOR, multipole moments
                    and boundary values)
  digests.json      SHA-256 of the reference's end state (State3D bytes) and
                    potential after N steps of the parity configurations:
                    config 0 (Sod 64^3, 100 steps and to t = 0.2) and
                    config 1 (n=1 polytrope 128^3 with gravity, tol 1e-8;
                    written progressively -- the reference needs hours)

Usage: python tests/golden/make_golden.py [small|sod64|poly128]
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import ics  # noqa: E402
from oracle.oracle import RefSim, soa_to_aos  # noqa: E402

DIGESTS = os.path.join(HERE, "digests.json")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def load_digests():
    if os.path.exists(DIGESTS):
        with open(DIGESTS) as f:
            return json.load(f)
    return {}


def save_digests(d):
    with open(DIGESTS + ".tmp", "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(DIGESTS + ".tmp", DIGESTS)


def small():
    out = {}
    shape = (12, 12, 12)
    q0 = ics.sod(shape)
    r = RefSim(*shape, gamma=1.4, cfl=0.4)
    r.set_state(q0)
    d, _, _ = r.step(20)
    out["sod12_q0"], out["sod12_q"], out["sod12_dt"] = q0, r.state(), d

    shape = (9, 11, 7)
    q0 = ics.smooth_random(shape, seed=11)
    r = RefSim(*shape, cfl=0.3, bc=(1, 2, 0, 0, 2, 1))
    r.set_state(q0)
    d, _, _ = r.step(6)
    out["rand_q0"], out["rand_q"], out["rand_dt"] = q0, r.state(), d

    shape = (12, 12, 12)
    q0, gam = ics.polytrope_n1(shape)
    r = RefSim(*shape, G=1.0, gamma=gam, tol=1e-8, max_iter=20000)
    r.set_state(q0)
    d, it, res = r.step(3)
    out["poly_q0"], out["poly_q"], out["poly_dt"] = q0, r.state(), d
    out["poly_it"], out["poly_res"], out["poly_phi"] = it, res, r.phi()

    shape = (10, 12, 9)
    q0, _ = ics.polytrope_n1(shape, R=0.3, centre=(0.4, 0.6, 0.5))
    rho = q0[0]
    r = RefSim(*shape, G=2.0)
    out["mom_rho"], out["mom"] = rho, r.moments(rho)
    r.boundary(rho)
    out["bnd_phi"] = r.phi()
    np.savez_compressed(os.path.join(HERE, "small.npz"), **out)
    print("wrote small.npz")


def sod64():
    dg = load_digests()
    shape = (64, 64, 64)
    q0 = ics.sod(shape)
    r = RefSim(*shape, gamma=1.4, cfl=0.4)
    r.set_state(q0)
    t = 0.0
    dts = []
    marks = {1, 10, 67, 100}
    rec = {}
    for s in range(1, 101):
        d, _, _ = r.step(1)
        t += d[0]
        dts.append(d[0])
        if s in marks:
            rec[str(s)] = {"state": sha(soa_to_aos(r.state())), "t": t}
    n_to_02 = next(i + 1 for i in range(len(dts)) if sum(dts[:i + 1]) >= 0.2)
    dg["sod64"] = {"steps": rec, "steps_to_t0.2": n_to_02, "dt_first": dts[0]}
    save_digests(dg)
    print("sod64 done; steps to t=0.2:", n_to_02)


def poly128(nsteps=100):
    dg = load_digests()
    shape = (128, 128, 128)
    q0, gam = ics.polytrope_n1(shape)
    r = RefSim(*shape, G=1.0, gamma=gam, tol=1e-8, max_iter=200000)
    r.set_state(q0)
    marks = {1, 2, 5, 10, 25, 50, 75, 100}
    rec = dg.get("poly128", {}).get("steps", {})
    iters = []
    t0 = time.time()
    for s in range(1, nsteps + 1):
        d, it, res = r.step(1)
        iters.append(int(it[0]))
        if s in marks:
            rec[str(s)] = {"state": sha(soa_to_aos(r.state())), "phi": sha(r.phi()),
                           "iterations": iters[:], "dt": float(d[0]), "residual": float(res[0])}
            dg = load_digests()
            dg["poly128"] = {"steps": rec, "tol": 1e-8, "omega": 1.5}
            save_digests(dg)
            print(f"poly128 step {s} ({time.time() - t0:.0f} s)", flush=True)


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "small"
    {"small": small, "sod64": sod64, "poly128": poly128}[what]()
