"""Opt-in MUSCL-Hancock reconstruction (hc_config.recon = 1, FP64) against
the CPU oracle's restatement of the same scheme, bit for bit, on 3D flows
with every boundary-condition kind and with self-gravity; and against the
exact Sod solution, where it must beat the reference's first-order states."""
import numpy as np
import pytest

import exact_riemann
import ics
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")


def pair(shape, q0, nsteps, **kw):
    okeys = ("G", "gamma", "cfl", "bc", "omega", "max_iter", "tol", "grav_bc", "lmax", "recon")
    o = OracleSim(*shape, **{k: v for k, v in kw.items() if k in okeys})
    o.set_state(q0)
    s = hc.HydroSolver3D(shape, **kw)
    s.set_state(q0)
    d_o, _, _ = o.step(nsteps)
    d_g = [float(s.step(1)[0]) for _ in range(nsteps)]
    return o, s, np.asarray(d_o), np.asarray(d_g)


@pytest.mark.parametrize("bc", [(2, 2, 2, 2, 2, 2), (0, 0, 1, 1, 2, 2), (1, 2, 0, 0, 1, 1)],
                         ids=["outflow", "periodic_reflective_outflow", "mixed"])
@pytest.mark.parametrize("shape", [(20, 18, 24), (17, 23, 13)])
def test_plm_bitwise_vs_oracle(shape, bc):
    q0 = ics.smooth_random(shape, seed=7)
    o, s, d_o, d_g = pair(shape, q0, 8, gamma=1.4, cfl=0.3, bc=bc, recon=1)
    assert np.array_equal(d_o, d_g), (d_o, d_g)
    a, b = s.state(), o.state()
    assert np.array_equal(a, b), np.abs(a - b).max()


def test_plm_with_gravity_bitwise_vs_oracle():
    shape = (20, 22, 18)
    q0, gam = ics.polytrope_n1(shape, R=0.3)
    q0[1] += 0.1 * q0[0]
    o, s, d_o, d_g = pair(shape, q0, 4, G=1.0, gamma=gam, cfl=0.3, tol=1e-8, max_iter=20000, recon=1)
    assert np.array_equal(d_o, d_g)
    assert np.array_equal(s.state(), o.state())
    assert np.array_equal(s.phi(), o.phi)


def test_plm_sod_against_exact_solution():
    nx = 100
    shape = (nx, 4, 4)
    err = {}
    for recon in (0, 1):
        s = hc.HydroSolver3D(shape, gamma=1.4, cfl=0.4, recon=recon)
        s.set_state(ics.sod(shape))
        t = 0.0
        while t < 0.2 - 1e-12:
            t += float(s.step(1)[0])
        x = (np.arange(nx) + 0.5) / nx
        ex = exact_riemann.sample(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 1.4, (x - 0.5) / t)
        err[recon] = np.abs(s.state()[0][:, 2, 2] - ex[0]).mean()
    assert err[1] < 0.7 * err[0], err


def test_plm_is_fp64_only():
    with pytest.raises(hc.HcError, match="FP64"):
        hc.HydroSolver3D((16, 16, 16), precision=hc.FP32, recon=1)
