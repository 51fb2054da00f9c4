"""ctypes front end to the CPU oracle (TEST INFRASTRUCTURE ONLY).

``OracleSim`` drives ``liboracle.so`` (hc_oracle.c, the plain-C restatement
of the reference time step).  ``RefSim`` drives ``_ref/libhcref.so``, the
unmodified reference sources built by ``oracle/Makefile`` (present only where
the reference tree was available at build time).  Nothing in the product
imports this module; tests, ``__graft_entry__.smoke`` and ``bench.py``'s CPU
baseline do.

Arrays are numpy float64.  Conserved state is exchanged as an array of shape
``(5, nx, ny, nz)`` (structure of arrays: rho, rhou, rhov, rhow, E) with the
reference's IDX3D ordering (k fastest, hydro_solver_3d.h:12).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "liboracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libhcref.so")

_dp = C.POINTER(C.c_double)


def _ptr(a):
    return a.ctypes.data_as(_dp)


class _Grid(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
        ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("gamma", C.c_double), ("cfl", C.c_double), ("G", C.c_double),
        ("bc", C.c_int * 6), ("gravity", C.c_int), ("grav_bc", C.c_int),
        ("lmax", C.c_int), ("omega", C.c_double), ("tol", C.c_double),
        ("max_iter", C.c_int),
        ("q", _dp * 5), ("phi", _dp), ("gx", _dp), ("gy", _dp), ("gz", _dp),
        ("dt", C.c_double), ("last_iter", C.c_int), ("last_res", C.c_double),
        ("recon", C.c_int),
    ]


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle/liboracle.so not built (run `make -C oracle`)")
        lib = C.CDLL(ORACLE_SO)
        gp = C.POINTER(_Grid)
        lib.hco_step.argtypes = [gp]
        lib.hco_step.restype = C.c_int
        lib.hco_cfl_dt.argtypes = [gp]
        lib.hco_cfl_dt.restype = C.c_double
        lib.hco_signal_max.argtypes = [gp]
        lib.hco_signal_max.restype = C.c_double
        lib.hco_step_dt.argtypes = [gp, C.c_double]
        lib.hco_step_dt.restype = C.c_int
        lib.hco_gravity_solve.argtypes = [gp, _dp]
        lib.hco_gravity_solve.restype = C.c_int
        lib.hco_gravity_solve_potential.argtypes = [gp, _dp]
        lib.hco_gravity_solve_potential.restype = C.c_int
        lib.hco_gravity_acceleration.argtypes = [gp]
        lib.hco_moments_ref.argtypes = [gp, _dp, _dp]
        lib.hco_boundary.argtypes = [gp, _dp]
        lib.hco_multipole_lmax.argtypes = [gp, _dp, C.c_int, _dp, _dp]
        lib.hco_boundary_lmax.argtypes = [gp, C.c_int, _dp, _dp]
        lib.hco_residual_norm.argtypes = [gp, _dp, _dp]
        lib.hco_residual_norm.restype = C.c_double
        lib.hco_sweep_norm.argtypes = [gp, _dp, _dp]
        lib.hco_sweep_norm.restype = C.c_double
        lib.hco_step_ext.argtypes = [gp, C.c_double]
        lib.hco_step_ext.restype = C.c_int
        lib.hco_moments_acc.argtypes = [gp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp]
        lib.hco_moments_com.argtypes = [gp, _dp, _dp]
        lib.hco_boundary_mom.argtypes = [gp, _dp, C.c_int, C.c_int, C.c_int, C.c_int]
        lib.hco_sor_half.argtypes = [gp, _dp, C.c_int]
        lib.hco_sor_half.restype = C.c_double
        _olib = lib
    return _olib


class OracleSim:
    """CPU oracle of one solver instance (structure-of-arrays FP64)."""

    def __init__(self, nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
                 G=0.0, gamma=5.0 / 3.0, cfl=0.4, bc=(2, 2, 2, 2, 2, 2),
                 omega=1.5, max_iter=10000, tol=1e-6, grav_bc=1, lmax=0, recon=0):
        self.lib = oracle_lib()
        self.shape = (nx, ny, nz)
        n = nx * ny * nz
        self.q = np.zeros((5, nx, ny, nz))
        self.phi = np.zeros((nx, ny, nz))
        self.gx = np.zeros((nx, ny, nz))
        self.gy = np.zeros((nx, ny, nz))
        self.gz = np.zeros((nx, ny, nz))
        g = _Grid()
        g.nx, g.ny, g.nz = nx, ny, nz
        g.xmin, g.ymin, g.zmin = lo
        g.xmax, g.ymax, g.zmax = hi
        g.dx = (hi[0] - lo[0]) / nx
        g.dy = (hi[1] - lo[1]) / ny
        g.dz = (hi[2] - lo[2]) / nz
        g.gamma, g.cfl, g.G = gamma, cfl, G
        for t in range(6):
            g.bc[t] = int(bc[t])
        g.gravity = 1 if G > 0.0 else 0
        g.grav_bc = grav_bc
        g.lmax = lmax
        g.omega, g.tol, g.max_iter = omega, tol, max_iter
        g.recon = recon
        for v in range(5):
            g.q[v] = _ptr(self.q[v])
        g.phi, g.gx, g.gy, g.gz = (_ptr(self.phi), _ptr(self.gx), _ptr(self.gy), _ptr(self.gz))
        self.g = g
        self.n = n

    # state -----------------------------------------------------------------
    def set_state(self, q):
        self.q[...] = q

    def state(self):
        return self.q.copy()

    # steps -----------------------------------------------------------------
    def step(self, nsteps=1):
        dts, its, res = [], [], []
        for _ in range(nsteps):
            self.lib.hco_step(C.byref(self.g))
            dts.append(self.g.dt)
            its.append(self.g.last_iter)
            res.append(self.g.last_res)
        return np.array(dts), np.array(its), np.array(res)

    def cfl_dt(self):
        return self.lib.hco_cfl_dt(C.byref(self.g))

    # gravity ---------------------------------------------------------------
    def gravity_solve(self, rho):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        st = self.lib.hco_gravity_solve(C.byref(self.g), _ptr(rho))
        return st, self.g.last_iter, self.g.last_res

    def gravity_solve_potential(self, rho):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        st = self.lib.hco_gravity_solve_potential(C.byref(self.g), _ptr(rho))
        return st, self.g.last_iter, self.g.last_res

    def moments_ref(self, rho):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        out = np.zeros(13)
        self.lib.hco_moments_ref(C.byref(self.g), _ptr(rho), _ptr(out))
        return out

    def boundary(self, rho):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        self.lib.hco_boundary(C.byref(self.g), _ptr(rho))

    def multipole_lmax(self, rho, lmax):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        com = np.zeros(3)
        cs = np.zeros((lmax + 1) ** 2)
        self.lib.hco_multipole_lmax(C.byref(self.g), _ptr(rho), lmax, _ptr(com), _ptr(cs))
        return com, cs

    def residual_norm(self, phi, rho):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        return self.lib.hco_residual_norm(C.byref(self.g), _ptr(phi), _ptr(rho))

    def sweep_norm(self, phi, rho):
        """Update norm of one red-black sweep from phi: the reference's test."""
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        return self.lib.hco_sweep_norm(C.byref(self.g), _ptr(phi), _ptr(rho))


def have_reference():
    return os.path.exists(REF_SO)


_rlib = None


def ref_lib():
    global _rlib
    if _rlib is None:
        if not have_reference():
            raise RuntimeError("oracle/_ref/libhcref.so not built (run `make -C oracle ref`)")
        lib = C.CDLL(REF_SO)
        lib.ref_create.argtypes = [C.c_int] * 3 + [C.c_double] * 9 + [C.POINTER(C.c_int)]
        lib.ref_create.restype = C.c_void_p
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_has_gravity.argtypes = [C.c_void_p]
        lib.ref_has_gravity.restype = C.c_int
        lib.ref_enable_gravity.argtypes = [C.c_void_p, C.c_int]
        lib.ref_set_grav.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_int]
        lib.ref_set_state.argtypes = [C.c_void_p, _dp]
        lib.ref_get_state.argtypes = [C.c_void_p, _dp]
        lib.ref_steps.argtypes = [C.c_void_p, C.c_int, _dp, C.POINTER(C.c_int), _dp]
        lib.ref_steps.restype = C.c_int
        lib.ref_get_phi.argtypes = [C.c_void_p, _dp]
        lib.ref_set_phi.argtypes = [C.c_void_p, _dp]
        lib.ref_get_grav_g.argtypes = [C.c_void_p, _dp, _dp, _dp]
        lib.ref_get_hydro_g.argtypes = [C.c_void_p, _dp, _dp, _dp]
        for f in ("ref_gravity_solve", "ref_gravity_solve_potential"):
            getattr(lib, f).argtypes = [C.c_void_p, _dp, C.POINTER(C.c_int), _dp]
            getattr(lib, f).restype = C.c_int
        lib.ref_moments.argtypes = [C.c_void_p, _dp, _dp]
        lib.ref_grav_boundary.argtypes = [C.c_void_p, _dp]
        lib.ref_grav_acceleration.argtypes = [C.c_void_p]
        lib.ref_ic_from_deck.argtypes = [C.c_void_p, C.c_char_p]
        lib.ref_ic_from_deck.restype = C.c_int
        lib.ref_ic_problem.argtypes = [C.c_void_p, C.c_int]
        lib.ref_parse_deck.argtypes = [C.c_char_p, C.POINTER(C.c_int), _dp, C.c_char_p]
        lib.ref_parse_deck.restype = C.c_int
        _rlib = lib
    return _rlib


def soa_to_aos(q):
    """(5, nx, ny, nz) -> (nx*ny*nz*5,) State3D array."""
    return np.ascontiguousarray(np.moveaxis(q, 0, -1)).reshape(-1)


def aos_to_soa(a, shape):
    nx, ny, nz = shape
    return np.ascontiguousarray(np.moveaxis(a.reshape(nx, ny, nz, 5), -1, 0))


class RefSim:
    """The reference's own time step, run through oracle/_ref/libhcref.so."""

    def __init__(self, nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
                 G=0.0, gamma=5.0 / 3.0, cfl=0.4, bc=(2, 2, 2, 2, 2, 2),
                 omega=1.5, max_iter=10000, tol=1e-6, grav_bc=1):
        self.lib = ref_lib()
        self.shape = (nx, ny, nz)
        bcs = (C.c_int * 6)(*[int(b) for b in bc])
        self.h = self.lib.ref_create(nx, ny, nz, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2],
                                     G, gamma, cfl, bcs)
        if not self.h:
            raise RuntimeError("ref_create failed")
        if self.lib.ref_has_gravity(self.h):
            self.lib.ref_set_grav(self.h, omega, max_iter, tol, grav_bc)

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, q):
        a = soa_to_aos(np.asarray(q, dtype=np.float64))
        self.lib.ref_set_state(self.h, _ptr(a))

    def state(self):
        a = np.zeros(np.prod(self.shape) * 5)
        self.lib.ref_get_state(self.h, _ptr(a))
        return aos_to_soa(a, self.shape)

    def step(self, nsteps=1):
        dts = np.zeros(nsteps)
        its = np.zeros(nsteps, dtype=np.int32)
        res = np.zeros(nsteps)
        self.lib.ref_steps(self.h, nsteps, _ptr(dts), its.ctypes.data_as(C.POINTER(C.c_int)),
                           _ptr(res))
        return dts, its, res

    def phi(self):
        out = np.zeros(self.shape)
        self.lib.ref_get_phi(self.h, _ptr(out))
        return out

    def set_phi(self, phi):
        p = np.ascontiguousarray(phi, dtype=np.float64)
        self.lib.ref_set_phi(self.h, _ptr(p))

    def grav_g(self):
        gx, gy, gz = (np.zeros(self.shape) for _ in range(3))
        self.lib.ref_get_grav_g(self.h, _ptr(gx), _ptr(gy), _ptr(gz))
        return gx, gy, gz

    def gravity_solve(self, rho, potential_only=False):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        it = C.c_int(0)
        res = C.c_double(0.0)
        f = self.lib.ref_gravity_solve_potential if potential_only else self.lib.ref_gravity_solve
        st = f(self.h, _ptr(rho), C.byref(it), C.byref(res))
        return st, it.value, res.value

    def moments(self, rho):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        out = np.zeros(13)
        self.lib.ref_moments(self.h, _ptr(rho), _ptr(out))
        return out

    def boundary(self, rho):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        self.lib.ref_grav_boundary(self.h, _ptr(rho))

    def enable_gravity(self, on):
        self.lib.ref_enable_gravity(self.h, 1 if on else 0)
