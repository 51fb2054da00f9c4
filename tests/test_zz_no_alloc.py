"""hc_sor_solve_noalloc: the SOR solve for callers that cannot allocate device
memory (they own a fixed arena or pool, or must not trigger the device-wide
synchronisation of cudaMalloc) gives the same potential and iteration count as
the context entry point hc_gravity_solve, on two calls in a row.

The caller's device buffers are made here with torch (the test may allocate;
the entry point under test does not).  This file is collected last so that a
run stopping at the first failure has run every other test already.
"""
import ctypes as C

import numpy as np
import pytest

import ics

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")
torch = pytest.importorskip("torch")


def noalloc_solve(phi_dev, rho_dev, shape, d, G, omega, max_iter, tol):
    it = C.c_int(0)
    res = C.c_double(0.0)
    rc = hc.lib().hc_sor_solve_noalloc(C.c_void_p(phi_dev.data_ptr()), C.c_void_p(rho_dev.data_ptr()),
                                       shape[0], shape[1], shape[2], d[0], d[1], d[2], G, omega,
                                       max_iter, tol, None, C.byref(it), C.byref(res))
    return rc, it.value, res.value


@pytest.mark.skipif(not torch.cuda.is_available(), reason="no CUDA device")
@pytest.mark.parametrize("shape,max_iter,expect", [
    ((34, 30, 38), 20000, 0),      # even nz, converges
    ((33, 31, 37), 20000, 0),      # odd sizes: the colour start k0 and the grid rounding along k
    ((33, 31, 37), 7, -1),         # stops at max_iter: iterations and residual as the context reports them
])
def test_noalloc_matches_context_solve_twice(shape, max_iter, expect):
    lo, hi = (0.0, 0.0, 0.0), (1.0, 1.0, 1.0)
    d = tuple((hi[a] - lo[a]) / shape[a] for a in range(3))
    G, omega, tol = 1.0, 1.5, 1e-9
    q, _ = ics.polytrope_n1(shape, R=0.3)
    rho1 = q[0]
    rho2 = rho1 * (1.0 + 0.05 * np.cos(np.arange(rho1.size).reshape(shape) * 0.37))
    # the same Dirichlet boundary in both paths: a smooth potential on the faces
    X, Y, Z = ics.centres(shape, lo, hi)
    phi0 = -1.0 / np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2 + 0.5)

    ctx = hc.HydroSolver3D(shape, lo=lo, hi=hi, G=G, omega=omega, tol=tol, max_iter=max_iter,
                           gravity_only=1, grav_bc=hc.GRAV_BC_DIRICHLET)
    ctx.set_phi(phi0)
    phi_dev = torch.tensor(phi0, dtype=torch.float64, device="cuda")

    for rho in (rho1, rho2):           # two calls in a row, each warm-started
        rho_dev = torch.tensor(rho, dtype=torch.float64, device="cuda")
        rc_ref = ctx.gravity_solve(rho)
        ref_phi = ctx.phi()
        ref_it = ctx.diagnostics()["last_iterations"]
        ref_res = ctx.diagnostics()["last_residual"]

        rc, it, res = noalloc_solve(phi_dev, rho_dev, shape, d, G, omega, max_iter, tol)
        torch.cuda.synchronize()
        assert rc == rc_ref == expect, hc.last_error()
        assert it == ref_it and res == ref_res
        got = phi_dev.cpu().numpy()
        # FP64 with the same operation order: the tolerance of the FP64 parity
        # tests, bit-for-bit equality
        assert np.array_equal(got, ref_phi)
    ctx.close()


@pytest.mark.skipif(not torch.cuda.is_available(), reason="no CUDA device")
def test_noalloc_rejects_too_many_iterations():
    shape = (8, 8, 8)
    phi = torch.zeros(shape, dtype=torch.float64, device="cuda")
    rho = torch.ones(shape, dtype=torch.float64, device="cuda")
    rc, _, _ = noalloc_solve(phi, rho, shape, (0.1, 0.1, 0.1), 1.0, 1.5, 65537, 1e-8)
    assert rc == -2 and "65536" in hc.last_error()
    for om, tol in ((2.0, 1e-8), (0.0, 1e-8), (float("nan"), 1e-8), (1.5, float("nan")), (1.5, 0.0),
                    (1.5, float("inf"))):
        rc, _, _ = noalloc_solve(phi, rho, shape, (0.1, 0.1, 0.1), 1.0, om, 100, tol)
        assert rc == -2, (om, tol)
