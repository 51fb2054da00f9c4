"""FP64 conservation sums formed on the device (hc_conservation_sums) against
numpy's sums of the same state, in both precisions.

The sums run in a fixed order (fixed pieces per block, fixed shuffle trees),
so the same state gives the same bits on every call; against numpy's pairwise
sums they agree to 1e-13 of the sum of absolute values (both are FP64 sums of
the same numbers in different orders).
"""
import numpy as np
import pytest

import ics

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(9, 11, 7), (40, 37, 72), (130, 64, 65)])
def test_sums_match_numpy_and_repeat(precision, shape):
    q0 = ics.smooth_random(shape, seed=9)
    prec = hc.FP64 if precision == "fp64" else hc.FP32
    s = hc.HydroSolver3D(shape, precision=prec, cfl=0.3)
    s.set_state(q0)
    q = s.state()                      # FP32 values exactly, promoted
    a = s.conservation()
    b = s.conservation()
    assert np.array_equal(a, b), "the same state gave different sums"
    ref = q.reshape(5, -1).sum(axis=1)
    scale = np.abs(q).reshape(5, -1).sum(axis=1)
    assert np.all(np.abs(a - ref) <= 1e-13 * scale), (a, ref)
    s.close()


def test_record_after_each_step():
    shape = (24, 20, 28)
    q0 = ics.smooth_random(shape, seed=2)
    s = hc.HydroSolver3D(shape, precision=hc.FP32, cfl=0.3)
    s.set_state(q0)
    s.set_conservation_record(True)
    for _ in range(3):
        s.step(1)
        rec = np.array(s.diagnostics()["cons"])
        assert np.array_equal(rec, s.conservation())
    s.close()
