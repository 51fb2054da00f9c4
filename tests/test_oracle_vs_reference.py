"""Pins the CPU oracle (oracle/hc_oracle.c) to the reference itself.

oracle/_ref/libhcref.so is the reference's own hydro_solver_3d.c +
gravity_solver_3d.c + input_deck.c, compiled unmodified from the reference
tree by oracle/Makefile.  These tests need it (skipped where the reference
tree was not available at build time); tests/test_golden.py pins the oracle
against fixtures the reference produced, without it.
"""
import numpy as np
import pytest

import ics
from oracle.oracle import OracleSim, RefSim, have_reference

pytestmark = pytest.mark.skipif(not have_reference(), reason="oracle/_ref not built")


def same(a, b):
    return np.array_equal(a, b)


def test_sod_bitwise():
    shape = (16, 16, 16)
    q0 = ics.sod(shape)
    o = OracleSim(*shape, gamma=1.4)
    r = RefSim(*shape, gamma=1.4)
    o.set_state(q0)
    r.set_state(q0)
    d1, _, _ = o.step(25)
    d2, _, _ = r.step(25)
    assert same(d1, d2) and same(o.state(), r.state())


@pytest.mark.parametrize("bc", [(0, 0, 0, 0, 0, 0), (1, 2, 1, 2, 1, 2), (2, 1, 0, 0, 1, 1),
                                (0, 1, 2, 0, 2, 2)])
def test_mixed_bc_bitwise(bc):
    shape = (11, 13, 9)
    q0 = ics.smooth_random(shape, seed=7)
    o = OracleSim(*shape, cfl=0.3, bc=bc)
    r = RefSim(*shape, cfl=0.3, bc=bc)
    o.set_state(q0)
    r.set_state(q0)
    d1, _, _ = o.step(6)
    d2, _, _ = r.step(6)
    assert same(d1, d2) and same(o.state(), r.state())


def test_gravity_step_bitwise():
    shape = (16, 16, 16)
    q0, gam = ics.polytrope_n1(shape)
    o = OracleSim(*shape, G=1.0, gamma=gam, tol=1e-8, max_iter=20000)
    r = RefSim(*shape, G=1.0, gamma=gam, tol=1e-8, max_iter=20000)
    o.set_state(q0)
    r.set_state(q0)
    d1, i1, r1 = o.step(3)
    d2, i2, r2 = r.step(3)
    assert list(i1) == list(i2) and same(r1, r2) and same(d1, d2)
    assert same(o.state(), r.state()) and same(o.phi, r.phi())
    gx, gy, gz = r.grav_g()
    assert same(o.gx, gx) and same(o.gy, gy) and same(o.gz, gz)


@pytest.mark.parametrize("gbc", [0, 1, 2])
def test_gravity_solve_bcs_bitwise(gbc):
    shape = (12, 14, 10)
    q0, _ = ics.polytrope_n1(shape, R=0.3)
    rho = q0[0]
    o = OracleSim(*shape, G=1.0, tol=1e-8, max_iter=4000, grav_bc=gbc)
    r = RefSim(*shape, G=1.0, tol=1e-8, max_iter=4000, grav_bc=gbc)
    so = o.gravity_solve(rho)
    sr = r.gravity_solve(rho)
    assert so == sr
    assert same(o.phi, r.phi())


def test_moments_and_boundary_bitwise():
    shape = (13, 11, 17)
    q0, _ = ics.polytrope_n1(shape, R=0.3, centre=(0.4, 0.6, 0.5))
    rho = q0[0]
    o = OracleSim(*shape, G=2.0)
    r = RefSim(*shape, G=2.0)
    assert same(o.moments_ref(rho), r.moments(rho))
    o.boundary(rho)
    r.boundary(rho)
    assert same(o.phi, r.phi())


def test_not_converged_bitwise():
    shape = (12, 12, 12)
    q0, gam = ics.polytrope_n1(shape)
    o = OracleSim(*shape, G=1.0, gamma=gam, tol=1e-12, max_iter=5)
    r = RefSim(*shape, G=1.0, gamma=gam, tol=1e-12, max_iter=5)
    o.set_state(q0)
    r.set_state(q0)
    _, i1, r1 = o.step(2)
    _, i2, r2 = r.step(2)
    assert list(i1) == list(i2) == [5, 5] and same(r1, r2)
    assert same(o.state(), r.state())
