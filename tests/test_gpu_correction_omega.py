"""Relaxation factor of the FP32 correction sweeps (hc_set_correction_omega).

The reference relaxes every SOR sweep with one omega (1.5 by default,
gravity_solver_3d.c:78) and stops when a red-black sweep moves no cell by tol
(max|phi_GS - phi_old|, :700-709), a test that does not depend on omega.  In
the mixed-precision solve only the FP32 correction sweeps relax, so their
factor can differ from the solve's: the solution must still pass the
reference's test in FP64, and near the optimal factor of the grid the solve
needs far fewer sweeps.
"""
import numpy as np
import pytest

import ics
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")


def test_correction_omega_same_test_fewer_sweeps():
    shape = (40, 40, 40)
    q0, gam = ics.polytrope_n1(shape)
    tol = 1e-8
    o = OracleSim(*shape, G=1.0, gamma=gam, tol=1e-11, max_iter=200000)
    o.gravity_solve(q0[0])
    r32 = q0[0].astype(np.float32).astype(np.float64)
    # optimal SOR factor of the 38-cell interior: 2 / (1 + sin(pi / 39))
    w_opt = 2.0 / (1.0 + np.sin(np.pi / 39.0))
    iters = {}
    for w in (0.0, round(w_opt, 3)):
        s = hc.HydroSolver3D(shape, G=1.0, gamma=gam, tol=tol, max_iter=200000, precision=hc.FP32,
                             moment_order=hc.MOMENTS_TREE)
        if w:
            s.correction_omega(w)
        s.set_state(q0.astype(np.float32).astype(np.float64))
        assert s.gravity_solve() == 0, s.diagnostics()
        phi = s.phi()
        # the reference's test on the mixed solution, in FP64 by the oracle
        assert o.sweep_norm(phi, r32) < tol, w
        assert np.abs(phi - o.phi).max() < 2e-4 * np.abs(o.phi).max(), w
        iters[w] = s.diagnostics()["last_iterations"]
        s.close()
    w = round(w_opt, 3)
    assert iters[w] < 0.5 * iters[0.0], iters


def test_correction_omega_range():
    s = hc.HydroSolver3D((32, 32, 32), G=1.0, precision=hc.FP32, moment_order=hc.MOMENTS_TREE)
    for bad in (-0.5, 2.0, 2.5, float("nan")):
        with pytest.raises(hc.HcError):
            s.correction_omega(bad)
    s.correction_omega(1.9)
    s.correction_omega(0.0)
    s.close()
