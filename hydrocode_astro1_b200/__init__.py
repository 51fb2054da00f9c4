"""hydrocode_astro1_b200 -- B200 (sm_100a) hydro + self-gravity time step.

Python mirror of the reference solver interface (hydro_solver_3d.h,
gravity_solver_3d.h) over the C ABI of ``include/hydrocode_b200.h``, served by
the in-tree shared library ``_lib/libhydrocode_b200.so``.  There is no CPU
fallback: every compute call runs the CUDA kernels of that library, and
constructing a solver fails loudly when the library or a GPU is missing.

Conventions (the reference's): conserved state per cell rho, rhou, rhov,
rhow, E; IDX3D ordering with k fastest (hydro_solver_3d.h:12); BCType 0
periodic / 1 reflective / 2 outflow (input_deck.h:30-34); GravBCType 0
periodic / 1 isolated / 2 dirichlet (gravity_solver_3d.h:10-14).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libhydrocode_b200.so")

BC_PERIODIC, BC_REFLECTIVE, BC_OUTFLOW = 0, 1, 2
GRAV_BC_PERIODIC, GRAV_BC_ISOLATED, GRAV_BC_DIRICHLET = 0, 1, 2
FP64, FP32 = 0, 1
MOMENTS_SEQUENTIAL, MOMENTS_TREE = 0, 1
HC_WARM_PREVIOUS, HC_WARM_UNET = 0, 1
WARM_PREVIOUS, WARM_UNET = 0, 1

HC_OK, HC_NOT_CONVERGED = 0, -1


class HcError(RuntimeError):
    pass


class Config(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
        ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
        ("gamma", C.c_double), ("cfl", C.c_double), ("G", C.c_double),
        ("bc", C.c_int * 6), ("precision", C.c_int), ("moment_order", C.c_int),
        ("grav_bc", C.c_int), ("lmax", C.c_int), ("omega", C.c_double),
        ("tol", C.c_double), ("max_iter", C.c_int), ("sor_depth", C.c_int),
        ("warm_start", C.c_int), ("device", C.c_int), ("gravity_only", C.c_int),
        ("recon", C.c_int), ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
    ]


class Diag(C.Structure):
    _fields_ = [
        ("last_iterations", C.c_int), ("last_residual", C.c_double),
        ("last_status", C.c_int), ("warm_start_used", C.c_int),
        ("outer_cycles", C.c_int), ("dt", C.c_double), ("steps", C.c_longlong),
        ("total_iterations", C.c_longlong), ("overshoot", C.c_int),
        ("unet_accepted", C.c_longlong), ("unet_fallbacks", C.c_longlong),
        ("cons", C.c_double * 5),
        ("unet_probes", C.c_longlong), ("unet_wins", C.c_longlong), ("unet_losses", C.c_longlong),
        ("unet_switch_offs", C.c_longlong), ("unet_off", C.c_int),
    ]


class Timing(C.Structure):
    _fields_ = [
        ("hydro_ms", C.c_double), ("bc_ms", C.c_double), ("sor_ms", C.c_double),
        ("residual_ms", C.c_double), ("moments_ms", C.c_double), ("unet_ms", C.c_double),
        ("hydro_launches", C.c_longlong), ("sor_launches", C.c_longlong),
        ("launches", C.c_longlong),
    ]


_dp = C.POINTER(C.c_double)
_lib = None

# name -> (restype, argtypes) of every C-ABI entry point in include/hydrocode_b200.h
CAPI = {
    "hc_config_default": (None, [C.POINTER(Config)]),
    "hc_create": (C.c_void_p, [C.POINTER(Config)]),
    "hc_destroy": (None, [C.c_void_p]),
    "hc_ncells": (C.c_size_t, [C.c_void_p]),
    "hc_set_state": (C.c_int, [C.c_void_p, _dp]),
    "hc_get_state": (C.c_int, [C.c_void_p, _dp]),
    "hc_set_state_soa": (C.c_int, [C.c_void_p, _dp]),
    "hc_get_state_soa": (C.c_int, [C.c_void_p, _dp]),
    "hc_step": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "hc_step_host": (C.c_int, [C.c_void_p, _dp, _dp]),
    "hc_gravity_solve": (C.c_int, [C.c_void_p, _dp, C.c_int]),
    "hc_gravity_acceleration": (C.c_int, [C.c_void_p]),
    "hc_set_gravity_params": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_double]),
    "hc_set_gravity_bc": (C.c_int, [C.c_void_p, C.c_int]),
    "hc_get_phi": (C.c_int, [C.c_void_p, _dp]),
    "hc_set_phi": (C.c_int, [C.c_void_p, _dp]),
    "hc_get_accel": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "hc_get_moments": (C.c_int, [C.c_void_p, _dp, C.c_int]),
    "hc_residual_norm": (C.c_int, [C.c_void_p, _dp]),
    "hc_conservation_sums": (C.c_int, [C.c_void_p, _dp]),
    "hc_get_signal_speed": (C.c_int, [C.c_void_p, _dp]),
    "hc_set_signal_speed": (C.c_int, [C.c_void_p, C.c_double]),
    "hc_copy_planes": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]),
    "hc_set_slab": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "hc_slab_moment_layout": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hc_slab_moments": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "hc_slab_set_moments": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int]),
    "hc_slab_sor_begin": (C.c_int, [C.c_void_p]),
    "hc_slab_sor_sweep": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "hc_slab_sor_boundary": (C.c_int, [C.c_void_p]),
    "hc_slab_sor_norm": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "hc_slab_sor_end": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int]),
    "hc_slab_phi_planes": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]),
    "hc_set_conservation_record": (C.c_int, [C.c_void_p, C.c_int]),
    "hc_get_diag": (C.c_int, [C.c_void_p, C.POINTER(Diag)]),
    "hc_get_timing": (C.c_int, [C.c_void_p, C.POINTER(Timing), C.c_int]),
    "hc_sync": (C.c_int, [C.c_void_p]),
    "hc_timer_start": (C.c_int, [C.c_void_p]),
    "hc_timer_stop": (C.c_int, [C.c_void_p, _dp]),
    "hc_unet_param_count": (C.c_int, []),
    "hc_unet_init": (C.c_int, [C.c_void_p, C.c_uint]),
    "hc_unet_load": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int, C.c_double]),
    "hc_unet_save": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_double)]),
    "hc_unet_load_file": (C.c_int, [C.c_void_p, C.c_char_p]),
    "hc_unet_save_file": (C.c_int, [C.c_void_p, C.c_char_p]),
    "hc_unet_collect": (C.c_int, [C.c_void_p, C.c_int]),
    "hc_unet_samples": (C.c_int, [C.c_void_p]),
    "hc_set_unet_passes": (C.c_int, [C.c_void_p, C.c_int]),
    "hc_set_unet_cycles": (C.c_int, [C.c_void_p, C.c_int]),
    "hc_set_unet_guard": (C.c_int, [C.c_void_p, C.c_int]),
    "hc_set_unet_record_cycle": (C.c_int, [C.c_void_p, C.c_int]),
    "hc_set_correction_omega": (C.c_int, [C.c_void_p, C.c_double]),
    "hc_checkpoint_save": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_longlong]),
    "hc_checkpoint_wait": (C.c_int, [C.c_void_p]),
    "hc_ic_profile_stars": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(_dp), C.POINTER(_dp),
                                      C.POINTER(_dp), _dp, _dp, _dp]),
    "hc_checkpoint_load": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    "hc_unet_train": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_uint, C.POINTER(C.c_double)]),
    "hc_unet_loss_grad": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float),
                                    C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_float),
                                    C.POINTER(C.c_float)]),
    "hc_unet_conv_test": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16),
                                    C.POINTER(C.c_float), C.c_int, C.c_int, C.POINTER(C.c_float)]),
    "hc_unet_wgrad_test": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16),
                                     C.c_int, C.POINTER(C.c_float)]),
    "hc_sor_solve_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double,
                                        C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                        C.c_double, C.c_void_p, C.POINTER(C.c_int), _dp]),
    "hc_host_register": (C.c_int, [C.c_void_p, C.c_size_t]),
    "hc_host_unregister": (C.c_int, [C.c_void_p]),
    "hc_last_error": (C.c_char_p, []),
    "hc_device_count": (C.c_int, []),
}


def lib():
    """Load the in-tree CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HcError(f"{LIB_PATH} missing: build it with `make -C hydrocode_astro1_b200` "
                          "or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in CAPI.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error():
    return lib().hc_last_error().decode(errors="replace")


def device_count():
    return lib().hc_device_count()


def _check(rc, what):
    if rc not in (HC_OK, HC_NOT_CONVERGED):
        raise HcError(f"{what} failed ({rc}): {last_error()}")
    return rc


def _p(a):
    return a.ctypes.data_as(_dp)


def default_config(**kw):
    cfg = Config()
    lib().hc_config_default(C.byref(cfg))
    for k, v in kw.items():
        if k == "bc":
            for t in range(6):
                cfg.bc[t] = int(v[t])
        elif k in ("lo", "hi"):
            names = ("xmin", "ymin", "zmin") if k == "lo" else ("xmax", "ymax", "zmax")
            for nm, val in zip(names, v):
                setattr(cfg, nm, float(val))
        elif k == "shape":
            cfg.nx, cfg.ny, cfg.nz = (int(x) for x in v)
        else:
            setattr(cfg, k, v)
    return cfg


class HydroSolver3D:
    """One device solver: the reference's GodunovHLLC3D with its GravitySolver3D.

    Mirrors solver3d_create / godunov_step_3d / gravity_solve and friends
    (hydro_solver_3d.h:69-95, gravity_solver_3d.h:64-149).
    """

    def __init__(self, shape=None, **kw):
        if shape is not None:
            kw["shape"] = shape
        self.cfg = default_config(**kw)
        self.L = lib()
        h = self.L.hc_create(C.byref(self.cfg))
        if not h:
            raise HcError(f"hc_create failed: {last_error()}")
        self.h = h
        self.shape = (self.cfg.nx, self.cfg.ny, self.cfg.nz)
        self.n = self.cfg.nx * self.cfg.ny * self.cfg.nz

    def close(self):
        if getattr(self, "h", None):
            self.L.hc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # state -------------------------------------------------------------
    def set_state(self, q):
        """q: (5, nx, ny, nz) float64 conserved fields."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        assert q.shape == (5,) + self.shape
        _check(self.L.hc_set_state_soa(self.h, _p(q)), "hc_set_state_soa")

    def state(self):
        q = np.empty((5,) + self.shape)
        _check(self.L.hc_get_state_soa(self.h, _p(q)), "hc_get_state_soa")
        return q

    def set_state_aos(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.size == 5 * self.n
        _check(self.L.hc_set_state(self.h, _p(U)), "hc_set_state")

    def state_aos(self):
        U = np.empty(5 * self.n)
        _check(self.L.hc_get_state(self.h, _p(U)), "hc_get_state")
        return U

    # stepping ------------------------------------------------------------
    def step(self, nsteps=1):
        """godunov_step_3d nsteps times; returns the dt of each step."""
        dts = np.zeros(max(nsteps, 1))
        rc = _check(self.L.hc_step(self.h, nsteps, _p(dts)), "hc_step")
        self.last_rc = rc
        return dts[:nsteps]

    def step_host(self, U):
        """One step on a host State3D array (upload, step, download) in place."""
        dt = C.c_double(0.0)
        rc = _check(self.L.hc_step_host(self.h, _p(U), C.byref(dt)), "hc_step_host")
        self.last_rc = rc
        return dt.value

    # gravity ---------------------------------------------------------------
    def gravity_solve(self, rho=None, with_accel=True):
        if rho is None:
            rc = self.L.hc_gravity_solve(self.h, None, int(with_accel))
        else:
            rho = np.ascontiguousarray(rho, dtype=np.float64)
            rc = self.L.hc_gravity_solve(self.h, _p(rho), int(with_accel))
        return _check(rc, "hc_gravity_solve")

    def set_gravity_params(self, omega, max_iter, tol):
        _check(self.L.hc_set_gravity_params(self.h, omega, max_iter, tol), "hc_set_gravity_params")

    def set_gravity_bc(self, bc):
        _check(self.L.hc_set_gravity_bc(self.h, bc), "hc_set_gravity_bc")

    def phi(self):
        out = np.empty(self.shape)
        _check(self.L.hc_get_phi(self.h, _p(out)), "hc_get_phi")
        return out

    def set_phi(self, phi):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        _check(self.L.hc_set_phi(self.h, _p(phi)), "hc_set_phi")

    def accel(self):
        gx, gy, gz = (np.empty(self.shape) for _ in range(3))
        _check(self.L.hc_get_accel(self.h, _p(gx), _p(gy), _p(gz)), "hc_get_accel")
        return gx, gy, gz

    def gravity_acceleration(self):
        _check(self.L.hc_gravity_acceleration(self.h), "hc_gravity_acceleration")

    def moments(self):
        cap = 4 + 13 * 13
        out = np.zeros(cap)
        _check(self.L.hc_get_moments(self.h, _p(out), cap), "hc_get_moments")
        if self.cfg.lmax == 0:
            return out[:13]
        return out[:4 + (self.cfg.lmax + 1) ** 2]

    def residual_norm(self):
        v = C.c_double(0.0)
        _check(self.L.hc_residual_norm(self.h, C.byref(v)), "hc_residual_norm")
        return v.value

    def conservation(self):
        """FP64 sums over all cells of (rho, rho u, rho v, rho w, E), formed on
        the device in a fixed order; times the cell volume they are totals."""
        out = np.zeros(5)
        _check(self.L.hc_conservation_sums(self.h, _p(out)), "hc_conservation_sums")
        return out

    # slabs of a larger grid ---------------------------------------------------
    def signal_speed(self):
        """The CFL maximum of |u_d| + c the next step's dt is formed from."""
        v = C.c_double(0.0)
        _check(self.L.hc_get_signal_speed(self.h, C.byref(v)), "hc_get_signal_speed")
        return v.value

    def set_signal_speed(self, s):
        _check(self.L.hc_set_signal_speed(self.h, float(s)), "hc_set_signal_speed")

    def copy_planes(self, i0, count, dev_ptr, to_ctx):
        """Planes [i0, i0+count) of the 5 state fields to (to_ctx False) or
        from (True) the device buffer at dev_ptr, field by field."""
        _check(self.L.hc_copy_planes(self.h, int(i0), int(count), C.c_void_p(int(dev_ptr)), int(bool(to_ctx))),
               "hc_copy_planes")

    def set_slab(self, gnx, ioff):
        """Declare this context the global planes [ioff, ioff + nx) of a grid
        of gnx planes (its config's x bounds the whole grid's)."""
        _check(self.L.hc_set_slab(self.h, int(gnx), int(ioff)), "hc_set_slab")

    def slab_moment_layout(self, p):
        """(sequential, width) of moment pass p across slabs."""
        sq, w = C.c_int(0), C.c_int(0)
        _check(self.L.hc_slab_moment_layout(self.h, int(p), C.byref(sq), C.byref(w)), "hc_slab_moment_layout")
        return bool(sq.value), w.value

    def slab_moments(self, p, buf):
        """Pass p over the own planes: continues the sums in buf (sequential)
        or fills buf with the own planes' partials; buf is FP64 numpy."""
        assert buf.dtype == np.float64 and buf.flags.c_contiguous
        _check(self.L.hc_slab_moments(self.h, int(p), buf.ctypes.data_as(_dp)), "hc_slab_moments")
        return buf

    def slab_set_moments(self, p, all_parts, nplanes):
        a = np.ascontiguousarray(all_parts, dtype=np.float64)
        _check(self.L.hc_slab_set_moments(self.h, int(p), a.ctypes.data_as(_dp), int(nplanes)),
               "hc_slab_set_moments")

    def slab_sor_begin(self):
        _check(self.L.hc_slab_sor_begin(self.h), "hc_slab_sor_begin")

    def slab_sor_sweep(self, it, colour):
        _check(self.L.hc_slab_sor_sweep(self.h, int(it), int(colour)), "hc_slab_sor_sweep")

    def slab_sor_boundary(self):
        _check(self.L.hc_slab_sor_boundary(self.h), "hc_slab_sor_boundary")

    def slab_sor_norm(self, it):
        v = C.c_double(0.0)
        _check(self.L.hc_slab_sor_norm(self.h, int(it), C.byref(v)), "hc_slab_sor_norm")
        return v.value

    def slab_sor_end(self, iterations, residual, converged):
        _check(self.L.hc_slab_sor_end(self.h, int(iterations), float(residual), int(bool(converged))),
               "hc_slab_sor_end")

    def slab_phi_planes(self, i0, count, ptr, to_ctx):
        """Planes [i0, i0+count) of the colour-split potential (both colours,
        [2][count][ny (nz+1)/2] FP64) to (to_ctx False) or from (True) ptr."""
        _check(self.L.hc_slab_phi_planes(self.h, int(i0), int(count), C.c_void_p(int(ptr)), int(bool(to_ctx))),
               "hc_slab_phi_planes")

    def set_conservation_record(self, on=True):
        """Form the sums after every hc_step call (hc_diag 'cons')."""
        _check(self.L.hc_set_conservation_record(self.h, int(bool(on))), "hc_set_conservation_record")

    def diagnostics(self):
        d = Diag()
        _check(self.L.hc_get_diag(self.h, C.byref(d)), "hc_get_diag")
        out = {f: getattr(d, f) for f, _ in Diag._fields_}
        out["cons"] = list(d.cons)
        return out

    def timing(self, reset=False):
        t = Timing()
        _check(self.L.hc_get_timing(self.h, C.byref(t), int(reset)), "hc_get_timing")
        return {f: getattr(t, f) for f, _ in Timing._fields_}

    def sync(self):
        _check(self.L.hc_sync(self.h), "hc_sync")

    def timer_start(self):
        _check(self.L.hc_timer_start(self.h), "hc_timer_start")

    def timer_stop(self):
        v = C.c_double(0.0)
        _check(self.L.hc_timer_stop(self.h, C.byref(v)), "hc_timer_stop")
        return v.value

    # learned warm start --------------------------------------------------------
    def unet_init(self, seed=0):
        _check(self.L.hc_unet_init(self.h, seed), "hc_unet_init")

    def unet_load(self, params, kscale):
        p = np.ascontiguousarray(params, dtype=np.float32)
        _check(self.L.hc_unet_load(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size, float(kscale)),
               "hc_unet_load")

    def unet_params(self):
        n = self.L.hc_unet_param_count()
        p = np.zeros(n, np.float32)
        k = C.c_double(0.0)
        _check(self.L.hc_unet_save(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), n, C.byref(k)), "hc_unet_save")
        return p, k.value

    def unet_load_file(self, path):
        _check(self.L.hc_unet_load_file(self.h, str(path).encode()), "hc_unet_load_file")

    def unet_save_file(self, path):
        _check(self.L.hc_unet_save_file(self.h, str(path).encode()), "hc_unet_save_file")

    def unet_collect(self, capacity):
        _check(self.L.hc_unet_collect(self.h, int(capacity)), "hc_unet_collect")

    def unet_samples(self):
        return self.L.hc_unet_samples(self.h)

    def unet_passes(self, n):
        _check(self.L.hc_set_unet_passes(self.h, int(n)), "hc_set_unet_passes")

    def unet_guard(self, consecutive_losses=3):
        """Outcome monitor of the learned start: switch the network off after
        this many consecutive solves where it saved no iterations (0: off)."""
        _check(self.L.hc_set_unet_guard(self.h, int(consecutive_losses)), "hc_set_unet_guard")

    def unet_cycles(self, n):
        """Correction cycles that start from the network's prediction (default 2)."""
        _check(self.L.hc_set_unet_cycles(self.h, int(n)), "hc_set_unet_cycles")

    def checkpoint_save(self, path, t=0.0, step=0):
        """Pack the state (and potentials) on the device and write `path` in
        the background; the solver may keep stepping.  checkpoint_wait()
        returns when the file is complete."""
        _check(self.L.hc_checkpoint_save(self.h, os.fsencode(path), float(t), int(step)), "hc_checkpoint_save")

    def ic_profile_stars(self, profiles, centres, R_star=None, vel=None):
        """Initial state built on the device from radial profiles: one star
        (profiles = [(r, rho, u)], centres = [(x, y, z)]) or two (with R_star
        and vel per star), as the stellar-profile / binary-star set-ups."""
        ns = len(profiles)
        tabs = [tuple(np.ascontiguousarray(a, dtype=np.float64) for a in pr) for pr in profiles]
        n = (C.c_int * ns)(*[len(t[0]) for t in tabs])
        rr = (_dp * ns)(*[_p(t[0]) for t in tabs])
        rh = (_dp * ns)(*[_p(t[1]) for t in tabs])
        uu = (_dp * ns)(*[_p(t[2]) for t in tabs])
        cen = np.ascontiguousarray(np.asarray(centres, dtype=np.float64).ravel())
        Rs = None if R_star is None else np.ascontiguousarray(np.asarray(R_star, dtype=np.float64))
        vv = None if vel is None else np.ascontiguousarray(np.asarray(vel, dtype=np.float64).ravel())
        _check(self.L.hc_ic_profile_stars(self.h, ns, n, rr, rh, uu, None if Rs is None else _p(Rs), _p(cen),
                                          None if vv is None else _p(vv)), "hc_ic_profile_stars")

    def checkpoint_wait(self):
        _check(self.L.hc_checkpoint_wait(self.h), "hc_checkpoint_wait")

    def checkpoint_load(self, path):
        """Restore a checkpoint written by checkpoint_save; returns (t, step)."""
        t = C.c_double(0.0)
        n = C.c_longlong(0)
        _check(self.L.hc_checkpoint_load(self.h, os.fsencode(path), C.byref(t), C.byref(n)), "hc_checkpoint_load")
        return t.value, n.value

    def unet_record_cycle(self, c):
        """With collection on: the correction cycle whose residual is recorded."""
        _check(self.L.hc_set_unet_record_cycle(self.h, int(c)), "hc_set_unet_record_cycle")

    def correction_omega(self, omega):
        """Relaxation factor of the FP32 correction sweeps of the mixed solve
        (0 < omega < 2; 0: the solve's own omega, the default)."""
        _check(self.L.hc_set_correction_omega(self.h, float(omega)), "hc_set_correction_omega")

    def unet_train(self, steps, lr=1e-3, seed=0):
        loss = C.c_double(0.0)
        _check(self.L.hc_unet_train(self.h, int(steps), float(lr), int(seed), C.byref(loss)), "hc_unet_train")
        return loss.value

    def unet_loss_grad(self, x, t):
        """One forward/backward pass at the network's level-0 dims (x.shape)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        n = self.L.hc_unet_param_count()
        g = np.zeros(n, np.float32)
        out = np.zeros(x.shape, np.float32)
        loss = C.c_double(0.0)
        fp = C.POINTER(C.c_float)
        _check(self.L.hc_unet_loss_grad(self.h, *x.shape, x.ctypes.data_as(fp), t.ctypes.data_as(fp), C.byref(loss),
                                        g.ctypes.data_as(fp), out.ctypes.data_as(fp)), "hc_unet_loss_grad")
        return loss.value, g, out


def pin(array):
    """Page-lock a numpy array's memory (cudaHostRegister); returns it."""
    _check(lib().hc_host_register(array.ctypes.data, array.nbytes), "hc_host_register")
    return array


def unpin(array):
    _check(lib().hc_host_unregister(array.ctypes.data), "hc_host_unregister")
