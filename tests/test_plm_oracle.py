"""The oracle's MUSCL-Hancock step (opt-in higher-order reconstruction, no
reference counterpart) against the exact Sod solution: it must beat the
reference's piecewise-constant scheme, and it leaves a uniform flow
unchanged."""
import numpy as np

import exact_riemann
import ics
from oracle.oracle import OracleSim


def sod_l1(recon, nx=100, t_end=0.2):
    shape = (nx, 3, 3)
    q0 = ics.sod(shape)
    o = OracleSim(*shape, gamma=1.4, cfl=0.4, recon=recon)
    o.set_state(q0)
    t = 0.0
    while t < t_end - 1e-12:
        dts, _, _ = o.step(1)
        t += float(np.asarray(dts).ravel()[0])
    x = (np.arange(nx) + 0.5) / nx
    ex = exact_riemann.sample(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 1.4, (x - 0.5) / t)
    rho = o.state()[0][:, 1, 1]
    return np.abs(rho - ex[0]).mean(), t


def test_exact_riemann_star_state():
    p, u = exact_riemann.star(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 1.4)
    assert abs(p - 0.30313) < 1e-5 and abs(u - 0.92745) < 1e-5   # Toro, table 4.3, test 1


def test_plm_beats_piecewise_constant_on_sod():
    e0, t0 = sod_l1(0)
    e1, t1 = sod_l1(1)
    assert e1 < 0.7 * e0, (e0, e1)
    assert e1 < 0.012, e1


def test_plm_keeps_uniform_flow():
    shape = (12, 10, 8)
    q = np.zeros((5,) + shape)
    q[0] = 1.3
    q[1], q[2], q[3] = 1.3 * 0.2, -1.3 * 0.1, 1.3 * 0.05
    q[4] = 2.0 / 0.4 + 0.5 * 1.3 * (0.2 ** 2 + 0.1 ** 2 + 0.05 ** 2)
    o = OracleSim(*shape, gamma=1.4, cfl=0.4, bc=(0, 0, 0, 0, 0, 0), recon=1)
    o.set_state(q)
    o.step(5)
    assert np.allclose(o.state(), q, rtol=1e-13, atol=1e-13)
