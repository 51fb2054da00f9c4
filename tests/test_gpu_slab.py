"""The slab decomposition on the GPU: the grid split into 2 or 3 slab
contexts on one device (ghost planes exchanged through device buffers, the
signal speed reduced over the slabs) steps bit for bit as one context of the
whole grid, in FP64 and in FP32 (every kernel's arithmetic per cell is
independent of where a chunk of planes starts), state and every dt."""
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
