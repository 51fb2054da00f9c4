"""CUDA path vs the CPU oracle, through the C ABI.

FP64 path: bit-for-bit equality with the oracle (which is itself bit-exact
with the reference C build, see test_oracle_vs_reference.py), on the Sod
shock tube, odd grids with partial tiles, every boundary-condition mix, and
self-gravity with the multipole boundary.
"""
import numpy as np
import pytest

import ics
from oracle.oracle import OracleSim

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")


def assert_bitwise(a, b, what):
    if not np.array_equal(a, b):
        d = np.abs(a - b)
        i = np.unravel_index(np.argmax(d), d.shape)
        raise AssertionError(f"{what}: not bit-identical, max |diff| {d.max():.3e} at {i}: "
                             f"{a[i]!r} vs {b[i]!r}")


def run_pair(shape, q0, nsteps, **kw):
    okw = dict(kw)
    lo = okw.pop("lo", (0.0, 0.0, 0.0))
    hi = okw.pop("hi", (1.0, 1.0, 1.0))
    o = OracleSim(*shape, lo=lo, hi=hi, **{k: v for k, v in okw.items()
                                            if k in ("G", "gamma", "cfl", "bc", "omega", "max_iter",
                                                     "tol", "grav_bc", "lmax")})
    o.set_state(q0)
    gkw = {k: v for k, v in kw.items() if k not in ("lo", "hi")}
    s = hc.HydroSolver3D(shape, lo=lo, hi=hi, **gkw)
    s.set_state(q0)
    d_o, i_o, r_o = o.step(nsteps)
    d_g = []
    its = []
    for _ in range(nsteps):
        d_g.append(s.step(1)[0])
        its.append(s.diagnostics()["last_iterations"])
    return o, s, d_o, np.array(d_g), i_o, np.array(its)


def test_sod_16_bitwise():
    shape = (16, 16, 16)
    q0 = ics.sod(shape)
    o, s, d_o, d_g, _, _ = run_pair(shape, q0, 20, gamma=1.4, cfl=0.4)
    assert_bitwise(d_g, d_o, "dt")
    assert_bitwise(s.state(), o.state(), "state")


@pytest.mark.parametrize("bc", [(0, 0, 0, 0, 0, 0), (1, 2, 1, 2, 1, 2), (2, 1, 0, 0, 1, 1),
                                (1, 1, 1, 1, 1, 1)])
def test_odd_grid_bc_bitwise(bc):
    shape = (11, 13, 37)   # partial tiles in j and k, short i chunks
    q0 = ics.smooth_random(shape, seed=3)
    o, s, d_o, d_g, _, _ = run_pair(shape, q0, 7, cfl=0.3, bc=bc)
    assert_bitwise(d_g, d_o, "dt")
    assert_bitwise(s.state(), o.state(), "state")


def test_aos_roundtrip_and_step_host():
    shape = (9, 10, 12)
    q0 = ics.smooth_random(shape, seed=5)
    from oracle.oracle import soa_to_aos, aos_to_soa
    s = hc.HydroSolver3D(shape, cfl=0.35)
    U = soa_to_aos(q0)
    s.set_state_aos(U)
    assert_bitwise(s.state_aos(), U, "aos roundtrip")
    o = OracleSim(*shape, cfl=0.35)
    o.set_state(q0)
    o.step(1)
    dt = s.step_host(U)
    assert dt == o.g.dt
    assert_bitwise(aos_to_soa(U, shape), o.state(), "step_host")


def test_gravity_polytrope_bitwise():
    shape = (24, 24, 24)
    q0, gam = ics.polytrope_n1(shape)
    kw = dict(G=1.0, gamma=gam, tol=1e-8, max_iter=20000, cfl=0.4)
    o, s, d_o, d_g, i_o, i_g = run_pair(shape, q0, 3, **kw)
    assert list(i_g) == list(i_o)
    assert_bitwise(d_g, d_o, "dt")
    assert_bitwise(s.phi(), o.phi, "phi")
    assert_bitwise(s.state(), o.state(), "state")
    gx, gy, gz = s.accel()
    assert_bitwise(gx, o.gx, "gx")
    assert_bitwise(gy, o.gy, "gy")
    assert_bitwise(gz, o.gz, "gz")


def test_gravity_solve_standalone_and_moments():
    shape = (20, 18, 22)
    q0, _ = ics.polytrope_n1(shape, R=0.3)
    rho = q0[0] * (1.0 + 0.1 * np.sin(np.arange(q0[0].size).reshape(shape)))
    o = OracleSim(*shape, G=1.0, tol=1e-9, max_iter=5000)
    s = hc.HydroSolver3D(shape, G=1.0, tol=1e-9, max_iter=5000)
    st_o, it_o, r_o = o.gravity_solve(rho)
    rc = s.gravity_solve(rho)
    d = s.diagnostics()
    assert (rc == 0) == (st_o == 0)
    assert d["last_iterations"] == it_o
    assert d["last_residual"] == r_o
    assert_bitwise(s.moments(), o.moments_ref(rho), "moments")
    assert_bitwise(s.phi(), o.phi, "phi")


def test_gravity_not_converged_keeps_stale_g():
    """max_iter too small: -1 and g unchanged (gravity_solver_3d.c:906-909)."""
    shape = (16, 16, 16)
    q0, gam = ics.polytrope_n1(shape)
    kw = dict(G=1.0, gamma=gam, tol=1e-12, max_iter=7, cfl=0.4)
    o, s, d_o, d_g, i_o, i_g = run_pair(shape, q0, 2, **kw)
    assert list(i_g) == [7, 7] and list(i_o) == [7, 7]
    assert s.last_rc == hc.HC_NOT_CONVERGED
    assert_bitwise(s.state(), o.state(), "state")
    assert_bitwise(s.phi(), o.phi, "phi")


@pytest.mark.parametrize("gbc", [0, 2])
def test_gravity_other_bcs(gbc):
    shape = (14, 16, 12)
    q0, gam = ics.polytrope_n1(shape)
    kw = dict(G=1.0, gamma=gam, tol=1e-7, max_iter=3000, grav_bc=gbc)
    o, s, d_o, d_g, i_o, i_g = run_pair(shape, q0, 2, **kw)
    assert list(i_g) == list(i_o)
    assert_bitwise(s.state(), o.state(), "state")


def test_tree_moments_close():
    shape = (32, 30, 28)
    q0, _ = ics.polytrope_n1(shape, R=0.3)
    rho = q0[0]
    o = OracleSim(*shape, G=1.0, tol=1e-8, max_iter=1)
    s = hc.HydroSolver3D(shape, G=1.0, tol=1e-8, max_iter=1, moment_order=hc.MOMENTS_TREE)
    s.gravity_solve(rho)
    m_o = o.moments_ref(rho)
    m_g = s.moments()
    np.testing.assert_allclose(m_g, m_o, rtol=1e-12, atol=1e-14 * abs(m_o[0]))


@pytest.mark.parametrize("lmax,shape", [(2, (20, 22, 18)), (4, (20, 22, 18)), (8, (20, 22, 18)),
                                         (12, (20, 22, 18)), (8, (8, 6, 300)), (12, (30, 28, 33))])
def test_lmax_boundary_matches_oracle(lmax, shape):
    """Row-factored moments (rows longer than one pass of a warp, odd sizes)
    against the oracle's direct per-cell sums, and the boundary values."""
    q0, _ = ics.polytrope_n1(shape, R=0.25, centre=(0.45, 0.55, 0.5))
    rho = q0[0] * (1.0 + 0.3 * (ics.centres(shape, (0, 0, 0), (1, 1, 1))[0] > 0.5))
    o = OracleSim(*shape, G=1.0, tol=1e-8, max_iter=1, lmax=lmax)
    s = hc.HydroSolver3D(shape, G=1.0, tol=1e-8, max_iter=1, lmax=lmax,
                         moment_order=hc.MOMENTS_TREE)
    s.gravity_solve(rho)   # one iteration, then the lmax boundary
    com, cs = o.multipole_lmax(rho, lmax)
    m = s.moments()
    np.testing.assert_allclose(m[1:4], com, rtol=1e-11)
    np.testing.assert_allclose(m[4:], cs, rtol=1e-10, atol=1e-12 * np.abs(cs).max())
    o.gravity_solve(rho)
    pg, po = s.phi(), o.phi
    face = np.zeros(shape, bool)
    face[0] = face[-1] = True
    face[:, 0] = face[:, -1] = True
    face[:, :, 0] = face[:, :, -1] = True
    np.testing.assert_allclose(pg[face], po[face], rtol=1e-11)


def test_lmax2_equals_reference_quadrupole():
    """The solid-harmonic expansion at lmax=2 reproduces M + Q_ij."""
    shape = (16, 18, 20)
    q0, _ = ics.polytrope_n1(shape, R=0.3, centre=(0.4, 0.55, 0.5))
    rho = q0[0]
    s2 = hc.HydroSolver3D(shape, G=1.0, tol=1e-8, max_iter=1, lmax=2, moment_order=hc.MOMENTS_TREE)
    s0 = hc.HydroSolver3D(shape, G=1.0, tol=1e-8, max_iter=1, lmax=0)
    s2.gravity_solve(rho)
    s0.gravity_solve(rho)
    np.testing.assert_allclose(s2.phi(), s0.phi(), rtol=1e-12, atol=1e-14)


def test_gravity_simple_sweeps_bitwise():
    """The per-colour in-place kernels (sor_depth=-1) give the same iterates."""
    shape = (18, 20, 22)
    q0, gam = ics.polytrope_n1(shape)
    kw = dict(G=1.0, gamma=gam, tol=1e-8, max_iter=20000, cfl=0.4)
    o, s, d_o, d_g, i_o, i_g = run_pair(shape, q0, 2, sor_depth=-1, **kw)
    assert list(i_g) == list(i_o)
    assert_bitwise(s.state(), o.state(), "state")
    assert_bitwise(s.phi(), o.phi, "phi")


@pytest.mark.parametrize("depth", [0, 1])
@pytest.mark.parametrize("shape", [(40, 37, 70), (130, 20, 33), (9, 300, 5)])
def test_sor_layouts_chunks_bitwise(shape, depth):
    """Grids with several i-chunks, partial tiles and odd nz: the colour-split
    sweeps (sor_depth 0) and the wavefront passes (1) give the oracle's
    iterates bit for bit."""
    q0, gam = ics.polytrope_n1(shape, R=0.3)
    rho = q0[0]
    o = OracleSim(*shape, G=1.0, tol=1e-7, max_iter=700)
    s = hc.HydroSolver3D(shape, G=1.0, tol=1e-7, max_iter=700, sor_depth=depth)
    st_o, it_o, r_o = o.gravity_solve(rho)
    s.gravity_solve(rho)
    d = s.diagnostics()
    assert d["last_iterations"] == it_o and d["last_residual"] == r_o
    assert_bitwise(s.phi(), o.phi, "phi")


@pytest.mark.parametrize("depth", [0, -2, -1, 1, 2, 4])
def test_mixed_precision_poisson_converges(depth):
    """FP64 residual + FP32 correction sweeps reach the same tolerance; the
    potential agrees with the FP64 solution to the accuracy the tolerance
    implies."""
    shape = (40, 40, 40)
    q0, gam = ics.polytrope_n1(shape)
    rho = q0[0]
    tol = 1e-8
    o = OracleSim(*shape, G=1.0, gamma=gam, tol=1e-11, max_iter=200000)
    o.gravity_solve(rho)
    s = hc.HydroSolver3D(shape, G=1.0, gamma=gam, tol=tol, max_iter=200000, precision=hc.FP32,
                         moment_order=hc.MOMENTS_TREE, sor_depth=depth)
    s.set_state(q0.astype(np.float32).astype(np.float64))
    rc = s.gravity_solve()
    assert rc == 0, s.diagnostics()
    phi = s.phi()
    # the reference's convergence test on the mixed solution, in FP64 by the
    # oracle: one more red-black sweep moves no cell by tol or more
    r32 = q0[0].astype(np.float32).astype(np.float64)
    assert o.sweep_norm(phi, r32) < tol
    # distance to the converged FP64 potential (error amplification ~ N^2)
    assert np.abs(phi - o.phi).max() < 2e-4 * np.abs(o.phi).max()


@pytest.mark.parametrize("shape", [(40, 37, 72), (130, 20, 32), (24, 60, 40), (70, 70, 64), (10, 12, 392)])
def test_mixed_two_iteration_passes_match_sweeps(shape):
    """The colour-split passes of two iterations each (sor_depth -2: row tiles,
    plane chunks, recomputed halo rows and planes, out of place) give the
    iterates of the per-colour vector sweeps (nz = 392: the longest rows the
    pass's shared-memory rings hold): after the same even number of correction
    iterations the potentials are identical."""
    q0, gam = ics.polytrope_n1(shape, R=0.3)
    phis, norms = [], []
    for depth in (0, -2):
        s = hc.HydroSolver3D(shape, G=1.0, gamma=gam, tol=1e-30, max_iter=30, precision=hc.FP32,
                             moment_order=hc.MOMENTS_TREE, sor_depth=depth)
        s.set_state(q0.astype(np.float32).astype(np.float64))
        s.gravity_solve()
        d = s.diagnostics()
        assert d["last_iterations"] == 30, d
        phis.append(s.phi())
        norms.append(d["last_residual"])
    # every FP32 sweep kernel forms the update with the same explicit
    # multiply-adds, so the iterates are the same bits
    assert np.array_equal(phis[0], phis[1]), np.abs(phis[0] - phis[1]).max()
    assert norms[0] == norms[1], norms


def test_fp32_sod_close_to_fp64():
    shape = (48, 16, 16)
    q0 = ics.sod(shape)
    o = OracleSim(*shape, gamma=1.4)
    o.set_state(q0)
    s = hc.HydroSolver3D(shape, gamma=1.4, precision=hc.FP32)
    s.set_state(q0)
    o.step(30)
    s.step(30)
    a, b = s.state()[0], o.state()[0]
    l1 = np.abs(a - b).mean() / np.abs(b).mean()
    assert l1 < 1e-4, l1


@pytest.mark.parametrize("shape", [(24, 40, 72), (20, 18, 35)])
def test_fp32_3d_flow_close_to_fp64(shape):
    """FP32 step on a 3D flow whose velocity components take both signs, so
    every face direction uses both the left and the right HLLC state.  nz a
    multiple of 4 runs the TMA-staged kernel, odd nz the plain one.  Each
    field's L1 distance to the FP64 oracle after 10 steps stays at FP32
    rounding level (2e-6 relative)."""
    q0 = ics.smooth_random(shape, seed=4)
    o = OracleSim(*shape, gamma=5.0 / 3.0, cfl=0.3)
    o.set_state(q0)
    s = hc.HydroSolver3D(shape, gamma=5.0 / 3.0, cfl=0.3, precision=hc.FP32)
    s.set_state(q0)
    o.step(10)
    s.step(10)
    a, b = s.state(), o.state()
    for f in range(5):
        l1 = np.abs(a[f] - b[f]).mean() / np.abs(b[f]).mean()
        assert l1 < 2e-6, (f, l1)


@pytest.mark.parametrize("shape", [(40, 37, 72), (130, 20, 32), (24, 60, 40), (70, 70, 64), (10, 12, 392),
                                   (21, 19, 38), (33, 31, 37)])
def test_mixed_tma_sweeps_match_vector_sweeps(shape):
    """The TMA-staged colour sweeps (sor_depth -3: whole rows of up to 256
    cells per colour, row lengths a multiple of 4; plane tiles of 4, or 2 for
    rows over 128 cells; partial tiles in i and j) give the register vector
    sweeps' iterates (the default, sor_depth 0) bit for bit after the same
    number of correction iterations (shapes outside the TMA kernel's limits
    take the vector or scalar sweeps in both runs)."""
    q0, gam = ics.polytrope_n1(shape, R=0.3)
    phis, norms = [], []
    for depth in (0, -3):
        s = hc.HydroSolver3D(shape, G=1.0, gamma=gam, tol=1e-30, max_iter=30, precision=hc.FP32,
                             moment_order=hc.MOMENTS_TREE, sor_depth=depth)
        s.set_state(q0.astype(np.float32).astype(np.float64))
        s.gravity_solve()
        d = s.diagnostics()
        assert d["last_iterations"] == 30, d
        phis.append(s.phi())
        norms.append(d["last_residual"])
        s.close()
    assert np.array_equal(phis[0], phis[1]), np.abs(phis[0] - phis[1]).max()
    assert norms[0] == norms[1], norms
