"""The slab decomposition on the GPU: the grid split into 2 or 3 slab
contexts on one device (ghost planes exchanged through device buffers, the
signal speed reduced over the slabs) steps bit for bit as one context of the
whole grid, in FP64 and in FP32 (every kernel's arithmetic per cell is
independent of where a chunk of planes starts), state and every dt; with
self-gravity (FP64) also the potential, the SOR iterations and the final
update norm of every solve."""
import numpy as np
import pytest

import ics

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")
torch = pytest.importorskip("torch")
from hydrocode_astro1_b200 import slab  # noqa: E402

BC = (1, 2, 2, 1, 1, 2)


@pytest.mark.skipif(not torch.cuda.is_available(), reason="no CUDA device")
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shape,parts", [((40, 24, 32), 2), ((45, 19, 36), 3)])
def test_slabs_match_whole_grid(precision, shape, parts):
    prec = hc.FP64 if precision == "fp64" else hc.FP32
    steps = 8
    q0 = ics.smooth_random(shape, seed=21)
    whole = hc.HydroSolver3D(shape, cfl=0.35, bc=BC, precision=prec)
    whole.set_state(q0)
    dts = [float(whole.step(1)[0]) for _ in range(steps)]
    ref = whole.state()
    whole.close()
    slabs = [slab.GpuSlab(shape, e, cfl=0.35, bc=BC, precision=prec) for e in slab.plan(shape[0], parts)]
    for s in slabs:
        s.set_state(q0)
    comm = slab.LocalComm(slabs)
    got_dt = [comm.step() for _ in range(steps)]
    got = np.concatenate([s.own_state() for s in slabs], axis=1)
    for s in slabs:
        s.close()
    assert got_dt == dts
    assert np.array_equal(got, ref), np.abs(got - ref).max()


GBC = (2, 2, 2, 2, 2, 2)


def gravity_kw(lmax, order):
    return dict(G=1.0, gamma=2.0, cfl=0.3, omega=1.7, tol=1e-8, max_iter=20000, lmax=lmax,
                moment_order=hc.MOMENTS_SEQUENTIAL if order == "seq" else hc.MOMENTS_TREE, precision=hc.FP64)


@pytest.mark.skipif(not torch.cuda.is_available(), reason="no CUDA device")
@pytest.mark.parametrize("lmax,order", [(0, "seq"), (0, "tree"), (6, "tree")])
@pytest.mark.parametrize("shape,parts", [((40, 24, 32), 2), ((45, 19, 36), 3)])
def test_gravity_slabs_match_whole_grid(lmax, order, shape, parts):
    """Self-gravity across 2 or 3 slab contexts (moment chain or per-plane
    partials, half sweeps with ghost exchanges of the colour-split
    potential, the norm maximum) against one FP64 context of the whole grid:
    state, potential, dt, SOR iterations and final norm bit for bit over
    three steps; the 3-slab grids give odd global plane offsets."""
    kw = gravity_kw(lmax, order)
    steps = 3
    q0 = ics.gravity_blob(shape)
    whole = hc.HydroSolver3D(shape, bc=GBC, **kw)
    whole.set_state(q0)
    dts, its, res = [], [], []
    for _ in range(steps):
        dts.append(float(whole.step(1)[0]))
        d = whole.diagnostics()
        its.append(d["last_iterations"])
        res.append(d["last_residual"])
    ref, phi = whole.state(), whole.phi()
    whole.close()
    assert min(its) > 10
    slabs = [slab.GpuSlab(shape, e, bc=GBC, **kw) for e in slab.plan(shape[0], parts)]
    for s in slabs:
        s.set_state(q0)
    comm = slab.LocalComm(slabs)
    got_dt = []
    for _ in range(steps):
        got_dt.append(comm.step())
        for s in slabs:
            d = s.s.diagnostics()
            assert (d["last_iterations"], d["last_residual"]) == (its[len(got_dt) - 1], res[len(got_dt) - 1])
    got = np.concatenate([s.own_state() for s in slabs], axis=1)
    got_phi = np.concatenate([s.s.phi()[s.entry["own"][0] - s.entry["local"][0]:
                                        s.entry["own"][1] - s.entry["local"][0]] for s in slabs], axis=0)
    for s in slabs:
        s.close()
    assert got_dt == dts
    assert np.array_equal(got_phi, phi), np.abs(got_phi - phi).max()
    assert np.array_equal(got, ref), np.abs(got - ref).max()


@pytest.mark.skipif(not torch.cuda.is_available(), reason="no CUDA device")
def test_gravity_slabs_match_oracle():
    """The sequential-moment slabs against the CPU oracle's single grid (the
    reference's arithmetic): state and potential bit for bit."""
    from oracle.oracle import OracleSim
    shape, steps = (33, 18, 22), 2
    kw = gravity_kw(0, "seq")
    q0 = ics.gravity_blob(shape)
    o = OracleSim(*shape, bc=GBC, G=1.0, gamma=2.0, cfl=0.3, omega=1.7, tol=1e-8, max_iter=20000)
    o.set_state(q0)
    o.step(steps)
    slabs = [slab.GpuSlab(shape, e, bc=GBC, **kw) for e in slab.plan(shape[0], 2)]
    for s in slabs:
        s.set_state(q0)
    comm = slab.LocalComm(slabs)
    for _ in range(steps):
        comm.step()
    got = np.concatenate([s.own_state() for s in slabs], axis=1)
    for s in slabs:
        s.close()
    assert np.array_equal(got, o.state()), np.abs(got - o.state()).max()


@pytest.mark.skipif(not torch.cuda.is_available(), reason="no CUDA device")
def test_gravity_slab_rejects_fp32_and_single_solve():
    sl = slab.plan(24, 2)[0]
    with pytest.raises(hc.HcError):
        slab.GpuSlab((24, 16, 16), sl, bc=GBC, G=1.0, precision=hc.FP32)
    s = slab.GpuSlab((24, 16, 16), sl, bc=GBC, **gravity_kw(0, "seq"))
    with pytest.raises(hc.HcError):
        s.s.gravity_solve()
    s.close()
