"""Seeded synthetic initial states for the parity tests (numpy, FP64).

Each builder returns the conserved state as an array (5, nx, ny, nz) --
rho, rhou, rhov, rhow, E -- made from primitives with the reference's
prim_to_cons_3d arithmetic (hydro_solver_3d.c:177-189).  The same array is
handed to the CPU oracle, to the reference build and to the CUDA path, so
step parity does not depend on how an initial condition is produced.
"""
import numpy as np


def prim_to_cons(rho, u, v, w, p, gamma):
    ke = 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, p / (gamma - 1.0) + ke])


def centres(shape, lo, hi):
    n = np.array(shape)
    d = (np.array(hi) - np.array(lo)) / n
    ax = [lo[a] + (np.arange(shape[a]) + 0.5) * d[a] for a in range(3)]
    return np.meshgrid(*ax, indexing="ij")


def sod(shape, gamma=1.4, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), axis=0):
    """Sod shock tube along `axis` (x by default): rho,p = 1,1 | 0.125,0.1."""
    X = centres(shape, lo, hi)[axis]
    left = X < 0.5
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    z = np.zeros(shape)
    return prim_to_cons(rho, z, z, z, p, gamma)


def smooth_random(shape, seed=0, gamma=5.0 / 3.0, amp=0.3, vamp=0.5):
    """Smooth random positive state with moving fluid (exercises every HLLC branch)."""
    rng = np.random.default_rng(seed)
    X, Y, Z = centres(shape, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    rho = 1.0 + amp * np.sin(2 * np.pi * (X + rng.random())) * np.cos(2 * np.pi * (Y + rng.random()))
    p = 1.0 + amp * np.cos(2 * np.pi * (Z + rng.random()))
    u = vamp * np.sin(2 * np.pi * (Y + Z + rng.random()))
    v = vamp * np.cos(2 * np.pi * (X + rng.random())) * 2.0
    w = vamp * np.sin(2 * np.pi * (X - Y + rng.random())) * 3.0
    noise = 1.0 + 0.05 * rng.standard_normal(shape)
    return prim_to_cons(rho * noise, u, v, w, p, gamma)


def polytrope_n1(shape, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), M=1.0, R=0.35, G=1.0,
                 centre=None, floor_frac=1e-6):
    """n=1 polytrope in hydrostatic equilibrium: rho = rho_c sin(x)/x, x = pi r/R,
    p = K rho^2 with K = 2 G R^2 / pi, gamma = 2; floor_frac*rho_c outside R."""
    gamma = 2.0
    if centre is None:
        centre = tuple(0.5 * (lo[a] + hi[a]) for a in range(3))
    X, Y, Z = centres(shape, lo, hi)
    r = np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2)
    rho_c = np.pi * M / (4.0 * R ** 3)
    xi = np.pi * r / R
    with np.errstate(invalid="ignore", divide="ignore"):
        prof = np.where(xi > 0, np.sin(xi) / np.where(xi > 0, xi, 1.0), 1.0)
    rho = np.where(r < R, rho_c * prof, 0.0)
    rho = np.maximum(rho, floor_frac * rho_c)
    K = 2.0 * G * R * R / np.pi
    p = K * rho * rho
    z = np.zeros(shape)
    return prim_to_cons(rho, z, z, z, p, gamma), gamma


def gravity_blob(shape, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """An off-centre n=1 polytrope (gamma = 2, G = 1) given a smooth shearing
    velocity, so that the density and the potential change every step."""
    q, gamma = polytrope_n1(shape, lo, hi, R=0.3, centre=(0.46, 0.53, 0.49))
    X, Y, Z = centres(shape, lo, hi)
    rho = q[0]
    p = (gamma - 1.0) * q[4]
    u = 0.2 * np.sin(2 * np.pi * Y)
    v = 0.15 * np.cos(2 * np.pi * Z)
    w = 0.1 * np.sin(2 * np.pi * X)
    return prim_to_cons(rho, u, v, w, p, gamma)
