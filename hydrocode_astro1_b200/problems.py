"""Seeded synthetic initial conditions of the benchmark configurations.

Every builder returns ``(q, params)``: the conserved state as an array
(5, nx, ny, nz) -- rho, rhou, rhov, rhow, E, k fastest -- made with the
reference's prim_to_cons_3d arithmetic (hydro_solver_3d.c:177-189), and the
solver parameters (domain, gamma, G, boundary conditions, multipole degree).
The numbers are analytic or come from seeded generators; no external data.

  sod_3d              64^3 Sod shock tube, gamma 1.4, outflow, no gravity
  polytrope_n1        128^3 self-gravitating n=1 polytrope, G=M=1, R=0.35
  cold_collapse       192^3 rho ~ 1/r sphere on [-2,2]^3, e = 0.05 GM/R
  octant_explosion    256^3 n=3 Lane-Emden star (M=1, R=0.4) in the octant
                      layout of the reference's STELLAR_OCTANT_EXPLOSION_3D
                      (hydro_solver_3d.c:1864-2020): reflective min faces,
                      outflow max faces, thermal energy 1.0 inside r < 0.02 R,
                      1% log-normal density noise from the reference's LCG and
                      Box-Muller generator (hydro_solver_3d.c:1522-1539)
  stellar_explosion   the same star and explosion centred in [-0.75, 0.75]^3
                      with outflow faces (multipole boundary outside the star)
  binary_n1           512^3 two n=1 polytropes (M=0.5, 0.3, R=0.15) on a
                      circular orbit, separation 0.5, box [-1,1]^3
"""
from __future__ import annotations

import math

import numpy as np

RHO_FLOOR = 1.0e-5   # hydro_solver_3d.h:10
P_FLOOR = 1.0e-6     # hydro_solver_3d.h:11


def prim_to_cons(rho, u, v, w, p, gamma):
    ke = 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, p / (gamma - 1.0) + ke])


def centres(shape, lo, hi):
    d = [(hi[a] - lo[a]) / shape[a] for a in range(3)]
    ax = [lo[a] + (np.arange(shape[a]) + 0.5) * d[a] for a in range(3)]
    return np.meshgrid(*ax, indexing="ij", sparse=True)


def _params(shape, lo, hi, gamma, G, bc, lmax, cfl=0.4):
    return dict(shape=tuple(shape), lo=tuple(lo), hi=tuple(hi), gamma=gamma, G=G,
                bc=tuple(bc), lmax=lmax, cfl=cfl)


# --------------------------------------------------------------------------
# the reference's random generator, vectorised
# --------------------------------------------------------------------------
_LCG_A, _LCG_C, _M32 = 1664525, 1013904223, 0xFFFFFFFF


def lcg_states(seed, count):
    """The first `count` states of rng_state = (rng_state*1664525 + 1013904223)
    mod 2^32 after seed_rng(seed) (hydro_solver_3d.c:1522-1532), by doubling the
    affine map instead of a Python loop."""
    s = np.empty(count, dtype=np.uint64)
    if count == 0:
        return s
    s[0] = (np.uint64(seed & _M32) * np.uint64(_LCG_A) + np.uint64(_LCG_C)) & np.uint64(_M32)
    A, Cc, m = _LCG_A, _LCG_C, 1          # f^m(x) = A x + Cc
    while m < count:
        t = min(m, count - m)
        s[m:m + t] = (s[:t] * np.uint64(A) + np.uint64(Cc)) & np.uint64(_M32)
        A, Cc = (A * A) & _M32, (A * Cc + Cc) & _M32
        m += t
    return s


def lcg_normals(seed, count):
    """rand_normal() count times (Box-Muller of two consecutive uniforms,
    hydro_solver_3d.c:1534-1539)."""
    u = lcg_states(seed, 2 * count).astype(np.float64) / 4294967296.0
    u1, u2 = u[0::2], u[1::2]
    return np.sqrt(-2.0 * np.log(u1 + 1e-10)) * np.cos(2.0 * math.pi * u2)


# --------------------------------------------------------------------------
# Lane-Emden profiles
# --------------------------------------------------------------------------
def lane_emden(n, h=1e-4):
    """RK4 integration of theta'' + 2 theta'/xi + theta^n = 0 from the series
    start; returns xi, theta, dtheta up to the first zero xi1."""
    xi = 1e-6
    th = 1.0 - xi * xi / 6.0
    dth = -xi / 3.0

    def f(x, y, dy):
        return dy, -(max(y, 0.0) ** n) - 2.0 * dy / x

    xs, ths, dths = [0.0, xi], [1.0, th], [0.0, dth]
    while th > 0.0:
        k1 = f(xi, th, dth)
        k2 = f(xi + h / 2, th + h / 2 * k1[0], dth + h / 2 * k1[1])
        k3 = f(xi + h / 2, th + h / 2 * k2[0], dth + h / 2 * k2[1])
        k4 = f(xi + h, th + h * k3[0], dth + h * k3[1])
        th_n = th + h / 6 * (k1[0] + 2 * k2[0] + 2 * k3[0] + k4[0])
        dth_n = dth + h / 6 * (k1[1] + 2 * k2[1] + 2 * k3[1] + k4[1])
        if th_n <= 0.0:
            frac = th / (th - th_n)
            xi1 = xi + frac * h
            xs.append(xi1); ths.append(0.0); dths.append(dth + frac * (dth_n - dth))
            break
        xi += h
        th, dth = th_n, dth_n
        xs.append(xi); ths.append(th); dths.append(dth)
    return np.array(xs), np.array(ths), np.array(dths)


def polytrope_profile(n, M, R, G=1.0, gamma=5.0 / 3.0, points=2000):
    """Table r, rho, u (specific internal energy) of an index-n polytrope of
    mass M and radius R -- the 'r rho u' layout of the reference's stellar
    profile files (stellar_profile.txt:1-6)."""
    xs, th, dth = lane_emden(n, h=2e-4 if n < 2 else 1e-4)
    xi1 = xs[-1]
    omega = -xi1 * xi1 * dth[-1]
    alpha = R / xi1
    rho_c = M / (4.0 * math.pi * alpha ** 3 * omega)
    K = 4.0 * math.pi * G * alpha * alpha * rho_c ** (1.0 - 1.0 / n) / (n + 1.0)
    r = np.linspace(0.0, R, points)
    theta = np.interp(r / alpha, xs, th)
    rho = rho_c * np.maximum(theta, 0.0) ** n
    p = K * rho ** (1.0 + 1.0 / n)
    with np.errstate(invalid="ignore", divide="ignore"):
        u = np.where(rho > 0, p / ((gamma - 1.0) * np.where(rho > 0, rho, 1.0)), 0.0)
    return r, rho, u


def interpolate_profile(r_tab, rho_tab, u_tab, r):
    """interpolate_profile (hydro_solver_3d.c:889-925): central value inside
    the first point, 1e-6 atmosphere beyond the last, linear in between."""
    rho = np.interp(r, r_tab, rho_tab)
    u = np.interp(r, r_tab, u_tab)
    rho = np.where(r <= r_tab[0], rho_tab[0], rho)
    u = np.where(r <= r_tab[0], u_tab[0], u)
    out = r >= r_tab[-1]
    return np.where(out, 1e-6, rho), np.where(out, 1e-6, u)


# --------------------------------------------------------------------------
# configurations
# --------------------------------------------------------------------------
def sod_3d(n=64, gamma=1.4):
    shape = (n, n, n)
    X, _, _ = centres(shape, (0, 0, 0), (1, 1, 1))
    left = np.broadcast_to(X < 0.5, shape)
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    z = np.zeros(shape)
    q = prim_to_cons(rho, z, z, z, p, gamma)
    return q, _params(shape, (0, 0, 0), (1, 1, 1), gamma, 0.0, (2,) * 6, 0)


def polytrope_n1(n=128, M=1.0, R=0.35, G=1.0, lmax=4, lo=(0, 0, 0), hi=(1, 1, 1), centre=None):
    gamma = 2.0
    shape = (n, n, n)
    if centre is None:
        centre = tuple(0.5 * (lo[a] + hi[a]) for a in range(3))
    X, Y, Z = centres(shape, lo, hi)
    r = np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2)
    rho_c = math.pi * M / (4.0 * R ** 3)
    xi = math.pi * r / R
    with np.errstate(invalid="ignore", divide="ignore"):
        prof = np.where(xi > 0, np.sin(xi) / np.where(xi > 0, xi, 1.0), 1.0)
    rho = np.maximum(np.where(r < R, rho_c * prof, 0.0), 1e-6 * rho_c)
    K = 2.0 * G * R * R / math.pi
    p = K * rho * rho
    z = np.zeros(shape)
    q = prim_to_cons(rho, z, z, z, p, gamma)
    return q, _params(shape, lo, hi, gamma, G, (2,) * 6, lmax)


def cold_collapse(n=192, G=1.0, M=1.0, R=1.0, lmax=8):
    gamma = 5.0 / 3.0
    shape = (n, n, n)
    lo, hi = (-2.0, -2.0, -2.0), (2.0, 2.0, 2.0)
    dx = 4.0 / n
    X, Y, Z = centres(shape, lo, hi)
    r = np.sqrt(X * X + Y * Y + Z * Z)
    rs = np.maximum(r, 2.0 * dx)
    rho = np.where(r < R, M / (2.0 * math.pi * R * R * rs), 1e-5)
    # normalise the discrete mass inside R to M
    inside = r < R
    m_disc = rho[inside].sum() * dx ** 3
    rho = np.where(inside, rho * (M / m_disc), rho)
    e = 0.05 * G * M / R
    p = (gamma - 1.0) * rho * e
    z = np.zeros(shape)
    q = prim_to_cons(rho, z, z, z, p, gamma)
    return q, _params(shape, lo, hi, gamma, G, (2,) * 6, lmax)


def _stellar_explosion(n, lo, hi, bc, M, R, E, r_exp_frac, seed, noise, lmax, G):
    """n=3 Lane-Emden star centred on the origin, per-cell log-normal density
    noise, thermal energy E shared by the cells with r < r_exp_frac R
    (STELLAR_OCTANT_EXPLOSION_3D set-up, hydro_solver_3d.c:1864-2020)."""
    gamma = 5.0 / 3.0
    shape = (n, n, n)
    d = [(hi[a] - lo[a]) / n for a in range(3)]
    dV = d[0] * d[1] * d[2]
    r_tab, rho_tab, u_tab = polytrope_profile(3, M, R, G=G, gamma=gamma)
    X, Y, Z = centres(shape, lo, hi)
    r = np.sqrt(X * X + Y * Y + Z * Z)
    rho, u = interpolate_profile(r_tab, rho_tab, u_tab, r)
    rho = rho * np.exp(noise * lcg_normals(seed, rho.size).reshape(shape))
    p = rho * u * (gamma - 1.0)
    r_exp = r_exp_frac * R
    hot = r < r_exp
    count = int(hot.sum())
    if count > 0:
        e_cell = E / count
        u_hot = u + e_cell / (rho * dV)
        p = np.where(hot, rho * u_hot * (gamma - 1.0), p)
    z = np.zeros(shape)
    q = prim_to_cons(rho, z, z, z, p, gamma)
    return q, _params(shape, lo, hi, gamma, G, bc, lmax)


def octant_explosion(n=256, M=1.0, R=0.4, E=1.0, r_exp_frac=0.02, L=1.5, seed=42,
                     noise=0.01, lmax=8, G=1.0):
    """The reference's octant layout: [0, L]^3, reflective min faces, outflow
    max faces.  Its multipole boundary is evaluated on the symmetry planes,
    which cut through the star; for l_max > 2 the expansion diverges there and
    the first step already produces |v| ~ 1e6 next to the centre, in the
    reference's own FP64 arithmetic."""
    return _stellar_explosion(n, (0.0, 0.0, 0.0), (L, L, L), (1, 2, 1, 2, 1, 2), M, R, E, r_exp_frac,
                              seed, noise, lmax, G)


def stellar_explosion(n=256, M=1.0, R=0.4, E=1.0, r_exp_frac=0.02, H=0.75, seed=42,
                      noise=0.01, lmax=8, G=1.0):
    """The same star and explosion centred in [-H, H]^3 with outflow faces:
    every boundary point lies outside the star (H > R), so the l_max multipole
    boundary converges.  H = 0.75 keeps the octant layout's cell size at equal n."""
    return _stellar_explosion(n, (-H, -H, -H), (H, H, H), (2,) * 6, M, R, E, r_exp_frac, seed, noise,
                              lmax, G)


def binary_n1(n=512, M1=0.5, M2=0.3, R=0.15, sep=0.5, G=1.0, lmax=12):
    gamma = 2.0
    shape = (n, n, n)
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    Mt = M1 + M2
    x1, x2 = -sep * M2 / Mt, sep * M1 / Mt
    v_orb = math.sqrt(G * Mt / sep)
    v1, v2 = v_orb * M2 / Mt, -v_orb * M1 / Mt
    X, Y, Z = centres(shape, lo, hi)
    rho = np.full(shape, RHO_FLOOR)
    vy = np.zeros(shape)
    p = np.full(shape, P_FLOOR)
    for xc, M, v in ((x1, M1, v1), (x2, M2, v2)):
        r = np.sqrt((X - xc) ** 2 + Y * Y + Z * Z)
        rho_c = math.pi * M / (4.0 * R ** 3)
        xi = math.pi * r / R
        with np.errstate(invalid="ignore", divide="ignore"):
            prof = np.where(xi > 0, np.sin(xi) / np.where(xi > 0, xi, 1.0), 1.0)
        inside = r < R
        rs = np.where(inside, rho_c * prof, 0.0)
        K = 2.0 * G * R * R / math.pi
        rho = np.where(inside, np.maximum(rs, RHO_FLOOR), rho)
        p = np.where(inside, np.maximum(K * rs * rs, P_FLOOR), p)
        vy = np.where(inside, v, vy)
    z = np.zeros(shape)
    q = prim_to_cons(rho, z, vy, z, p, gamma)
    return q, _params(shape, lo, hi, gamma, G, (2,) * 6, lmax)


CONFIGS = {
    0: ("sod_64", sod_3d),
    1: ("polytrope_n1_128", polytrope_n1),
    2: ("cold_collapse_192", cold_collapse),
    3: ("stellar_explosion_256", stellar_explosion),
    4: ("binary_n1_512", binary_n1),
}
