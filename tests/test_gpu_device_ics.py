"""Profile-based initial conditions built on the device (hc_ic_profile_stars):
bit-identical to a numpy restatement of the host set-ups (one star; two
stars with the overlap rules; FP64 and FP32 state), and, through the
reference driver, to the host-built state (device_ics = 1 against 0)."""
import filecmp
import os
import subprocess

import numpy as np
import pytest

from hydrocode_astro1_b200 import problems

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "oracle", "_ref", "hydro3d_b200")


def prof_at(R, RHO, U, r):
    lo = np.clip(np.searchsorted(R, r, side="right") - 1, 0, len(R) - 2)
    f = (r - R[lo]) / (R[lo + 1] - R[lo])
    rho = RHO[lo] + f * (RHO[lo + 1] - RHO[lo])
    u = U[lo] + f * (U[lo + 1] - U[lo])
    inner, outer = r <= R[0], r >= R[-1]
    rho = np.where(inner, RHO[0], np.where(outer, 1e-6, rho))
    u = np.where(inner, U[0], np.where(outer, 1e-6, u))
    return rho, u


def centres(shape, lo, hi):
    ax = [lo[a] + (np.arange(shape[a]) + 0.5) * ((hi[a] - lo[a]) / shape[a]) for a in range(3)]
    return np.meshgrid(*ax, indexing="ij")


def p2c(rho, u, v, w, p, gam):
    rho = np.where(rho > 1e-5, rho, 1e-5)
    p = np.where(p > 1e-6, p, 1e-6)
    ke = 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, p / (gam - 1.0) + ke])


def dist(X, Y, Z, c):
    dx, dy, dz = X - c[0], Y - c[1], Z - c[2]
    return np.sqrt(dx * dx + dy * dy + dz * dz)


@pytest.mark.parametrize("precision", [hc.FP64, hc.FP32])
def test_one_star(precision):
    shape, lo, hi, gam = (24, 20, 28), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 2.0
    R, RHO, U = problems.polytrope_profile(1, 1.0, 0.3, gamma=gam, points=700)
    s = hc.HydroSolver3D(shape, lo=lo, hi=hi, gamma=gam, precision=precision)
    s.ic_profile_stars([(R, RHO, U)], [(0.5, 0.5, 0.5)])
    X, Y, Z = centres(shape, lo, hi)
    rho, u = prof_at(R, RHO, U, dist(X, Y, Z, (0.5, 0.5, 0.5)))
    z = np.zeros(shape)
    want = p2c(rho, z, z, z, (gam - 1.0) * rho * u, gam)
    if precision == hc.FP32:
        want = want.astype(np.float32).astype(np.float64)
    assert np.array_equal(s.state(), want)


def test_two_stars():
    shape, lo, hi, gam = (32, 24, 20), (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0), 2.0
    p1 = problems.polytrope_profile(1, 0.5, 0.3, gamma=gam, points=500)
    p2 = problems.polytrope_profile(1, 0.3, 0.25, gamma=gam, points=400)
    c = [(-0.2, 0.0, 0.0), (0.15, 0.05, 0.0)]     # overlapping: all four rules occur
    v = [(0.0, 0.3, 0.0), (0.0, -0.5, 0.1)]
    Rs = [0.29, 0.24]
    s = hc.HydroSolver3D(shape, lo=lo, hi=hi, gamma=gam)
    s.ic_profile_stars([p1, p2], c, R_star=Rs, vel=v)
    X, Y, Z = centres(shape, lo, hi)
    r1, r2 = dist(X, Y, Z, c[0]), dist(X, Y, Z, c[1])
    rho1, u1 = prof_at(*p1, r1)
    rho2, u2 = prof_at(*p2, r2)
    in1, in2 = r1 < Rs[0], r2 < Rs[1]
    gm1 = gam - 1.0
    rt = rho1 + rho2
    w1, w2 = rho1 / rt, rho2 / rt
    both = in1 & in2
    assert both.any() and (in1 & ~in2).any() and (in2 & ~in1).any() and (~in1 & ~in2).any()
    rho = np.where(in1 & ~in2, rho1, np.where(in2 & ~in1, rho2, np.where(both, rt, 1e-5)))
    vel = []
    for d in range(3):
        vel.append(np.where(in1 & ~in2, v[0][d], np.where(in2 & ~in1, v[1][d],
                                                          np.where(both, w1 * v[0][d] + w2 * v[1][d], 0.0))))
    p = np.where(in1 & ~in2, gm1 * rho1 * u1, np.where(in2 & ~in1, gm1 * rho2 * u2,
                                                      np.where(both, gm1 * rho1 * u1 + gm1 * rho2 * u2, 1e-6)))
    want = p2c(rho, vel[0], vel[1], vel[2], p, gam)
    assert np.array_equal(s.state(), want)


@pytest.mark.skipif(not os.path.exists(OURS), reason="drop-in binary not built")
def test_driver_device_and_host_set_ups_identical(tmp_path):
    """The reference driver with a binary-star deck: the state built on the
    device (device_ics = 1) and on the host (0) give byte-identical outputs,
    at t = 0 and after the run."""
    outs = {}
    for dev in (0, 1):
        d = tmp_path / f"d{dev}"
        os.makedirs(d / "output")
        for name, (M, R) in (("s1.txt", (0.5, 0.15)), ("s2.txt", (0.3, 0.15))):
            r, rho, u = problems.polytrope_profile(1, M, R, gamma=2.0, points=300)
            np.savetxt(d / name, np.stack([r, rho, u], 1), header="r rho u")
        deck = ("problem = BINARY_STAR_3D\nnx = 24\nny = 24\nnz = 24\nxmin = -1.0\nxmax = 1.0\nymin = -1.0\n"
                "ymax = 1.0\nzmin = -1.0\nzmax = 1.0\nt_end = 0.004\noutput_dt = 0.002\ngamma = 2.0\n"
                "G_const = 1.0\nstar1_profile = s1.txt\nstar2_profile = s2.txt\nbinary_auto_orbit = true\n"
                f"binary_separation = 0.5\noutput_dir = output\ndevice_ics = {dev}\n")
        (d / "deck.txt").write_text(deck)
        r = subprocess.run([OURS, "deck.txt"], cwd=d, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        outs[dev] = sorted(os.listdir(d / "output"))
    assert outs[0] == outs[1] and len(outs[0]) >= 2
    for fn in outs[0]:
        assert filecmp.cmp(tmp_path / "d0" / "output" / fn, tmp_path / "d1" / "output" / fn, shallow=False), fn
