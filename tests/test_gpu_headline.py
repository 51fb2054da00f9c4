"""The benchmarked configuration against the FP64 oracle.

The bench times FP32 hydro (the TMA-staged interior kernel when nz is a
multiple of 4, the plain FP32 kernel otherwise) with self-gravity from the
mixed-precision Poisson solve (FP64 outer residual, FP32 red-black correction
sweeps, the reference's stop rule max|phi_GS - phi_old| < tol), a multipole
boundary to l_max 8, and the learned warm start.  Here that arm runs 20 steps
beside the FP64 oracle (oracle/hc_oracle.c: the reference step of
hydro_solver_3d.c:637-811 with its gravity solve, gravity_solver_3d.c:510-911,
extended to the l_max multipole) on the same initial state, and:

  * every step's potential passes the reference's convergence test in FP64:
    one more red-black sweep from it (with the density the solve used) moves
    no cell by tol or more (gravity_solver_3d.c:715);
  * after 20 steps each conserved field's relative L1 distance to the oracle
    is at most 1e-4 (density L1 is the north-star's figure; the others are
    held to the same bound);
  * the drift of total mass and total energy from the initial state agrees
    with the oracle's own drift to 10% of that drift plus 1e-6 (the
    reference's step is not conservative -- boundary cells are not
    flux-updated, :729-731; the gravity source is not in flux form,
    :597-631 -- so the oracle drifts too, and FP32 must drift alike).  The
    GPU totals come from the device's FP64 conservation sums.
"""
import os

import numpy as np
import pytest

import ics
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")
problems = pytest.importorskip("hydrocode_astro1_b200.problems")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "hydrocode_astro1_b200", "data", "unet_stellar_explosion_256.bin")

TOL = 1e-8
STEPS = 20
L1_MAX = 1e-4
DRIFT_REL, DRIFT_ABS = 0.10, 1e-6


def polytrope(shape):
    q, gam = ics.polytrope_n1(shape, R=0.35)
    p = dict(shape=shape, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), gamma=gam, G=1.0, bc=(2,) * 6, lmax=8,
             cfl=0.4)
    return q, p


def explosion(n):
    q, p = problems.stellar_explosion(n)
    return q, p


CASES = {
    # nz % 4 == 0: interior_tma_kernel
    "polytrope_48_tma": (lambda: polytrope((48, 48, 48)), False),
    # odd nz: the plain FP32 interior kernel
    "polytrope_45x47x49_plain": (lambda: polytrope((45, 47, 49)), False),
    # the bench's workload at 64^3, with and without the learned start
    "explosion_64_tma": (lambda: explosion(64), False),
    "explosion_64_tma_unet": (lambda: explosion(64), True),
}


@pytest.mark.parametrize("case", list(CASES))
def test_headline_arm_against_fp64_oracle(case):
    make, unet = CASES[case]
    q0, p = make()
    shape = p["shape"]
    common = dict(G=p["G"], gamma=p["gamma"], cfl=p["cfl"], bc=p["bc"], omega=1.5, tol=TOL, lmax=p["lmax"])
    o = OracleSim(*shape, lo=p["lo"], hi=p["hi"], max_iter=400000, **common)
    o.set_state(q0)
    chk = OracleSim(*shape, lo=p["lo"], hi=p["hi"], max_iter=1, **common)

    kw = dict(lo=p["lo"], hi=p["hi"], max_iter=400000, precision=hc.FP32, moment_order=hc.MOMENTS_TREE,
              **common)
    if unet:
        kw["warm_start"] = hc.HC_WARM_UNET
    s = hc.HydroSolver3D(shape, **kw)
    if unet:
        s.unet_load_file(WEIGHTS)
    s.set_state(q0)
    c0 = s.conservation()

    for step in range(STEPS):
        rho_in = s.state()[0]            # the FP32 density the solve uses, exactly
        dt = s.step(1)[0]
        d = s.diagnostics()
        assert d["last_status"] == 0, (step, d)
        norm = chk.sweep_norm(s.phi(), rho_in)
        assert norm < TOL, f"step {step}: one more FP64 red-black sweep moves a cell by {norm:.3e}"
        assert np.isfinite(dt) and dt > 0.0
    o.step(STEPS)

    a, b = s.state(), o.state()
    for f in range(5):
        l1 = np.abs(a[f] - b[f]).sum() / np.abs(b[f]).sum()
        assert l1 <= L1_MAX, (case, f, l1)

    c1 = s.conservation()
    m0, e0 = q0[0].sum(), q0[4].sum()
    for f, ref0 in ((0, m0), (4, e0)):
        drift_gpu = c1[f] / c0[f] - 1.0
        drift_oracle = b[f].sum() / ref0 - 1.0
        assert abs(drift_gpu - drift_oracle) <= DRIFT_REL * abs(drift_oracle) + DRIFT_ABS, \
            (case, f, drift_gpu, drift_oracle)
    if unet:
        d = s.diagnostics()
        assert d["unet_accepted"] + d["unet_fallbacks"] > 0
    s.close()
