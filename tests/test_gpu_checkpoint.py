"""Binary checkpoint / restart through the C ABI (hc_checkpoint_save / _load).

A run restarted from a checkpoint continues bit for bit as the uninterrupted
run (state, potential, dt), in FP64 and in FP32 with the mixed-precision solve
and the learned warm start; the write happens in the background while the
context keeps stepping and still holds the state of the moment of the save;
the file's layout is the one documented (read back with the Python reader);
a checkpoint of another grid or a corrupt one is refused and leaves the
state untouched.
"""
import numpy as np
import pytest

import ics

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")
from hydrocode_astro1_b200.checkpoint import read_checkpoint  # noqa: E402


def make(shape, precision, warm=None):
    kw = dict(G=1.0, gamma=2.0, tol=1e-8, max_iter=200000, cfl=0.3, lmax=4, moment_order=hc.MOMENTS_TREE,
              precision=precision)
    if warm is not None:
        kw["warm_start"] = warm
    s = hc.HydroSolver3D(shape, **kw)
    if warm == hc.HC_WARM_UNET:
        s.unet_init(3)   # fixed random weights: predictions are deterministic (accepted or not)
    return s


@pytest.mark.parametrize("precision,warm,shape", [(hc.FP64, None, (24, 20, 28)),
                                                  (hc.FP32, None, (24, 20, 28)),
                                                  (hc.FP32, hc.HC_WARM_UNET, (32, 32, 32))])
def test_restart_is_bit_exact(tmp_path, precision, warm, shape):
    q0, _ = ics.polytrope_n1(shape, R=0.3)
    q0[1] += 0.05 * q0[0]   # some motion
    a = make(shape, precision, warm)
    a.set_state(q0)
    dts_a = list(a.step(6))
    qa, pa = a.state(), a.phi()
    b = make(shape, precision, warm)
    b.set_state(q0)
    dts_b = list(b.step(3))
    path = str(tmp_path / "run.ckpt")
    b.checkpoint_save(path, t=float(sum(dts_b)), step=3)
    b.checkpoint_wait()
    c = make(shape, precision, warm)
    t, step = c.checkpoint_load(path)
    assert step == 3 and t == float(sum(dts_b))
    dts_c = list(c.step(3))
    assert dts_b + dts_c == dts_a
    assert np.array_equal(c.state(), qa)
    assert np.array_equal(c.phi(), pa)


def test_background_write_keeps_the_saved_state(tmp_path):
    shape = (24, 20, 28)
    q0, _ = ics.polytrope_n1(shape, R=0.3)
    s = make(shape, hc.FP32)
    s.set_state(q0)
    s.step(2)
    q_saved, phi_saved = s.state(), s.phi()
    path = str(tmp_path / "bg.ckpt")
    s.checkpoint_save(path, t=1.5, step=2)
    s.step(3)                          # the context keeps stepping while the file is written
    s.checkpoint_wait()
    r = make(shape, hc.FP32)
    assert r.checkpoint_load(path) == (1.5, 2)
    assert np.array_equal(r.state(), q_saved)
    assert np.array_equal(r.phi(), phi_saved)
    # the documented layout, read back in Python
    ck = read_checkpoint(path, verify=True)
    assert ck["shape"] == shape and int(ck["step"]) == 2 and ck["state"].dtype == np.float32
    assert np.array_equal(ck["state"].astype(np.float64), q_saved)
    assert np.array_equal(ck["phi"], phi_saved)


def test_mismatch_and_corruption_are_refused(tmp_path):
    shape = (24, 20, 28)
    q0, _ = ics.polytrope_n1(shape, R=0.3)
    s = make(shape, hc.FP64)
    s.set_state(q0)
    s.step(1)
    path = str(tmp_path / "a.ckpt")
    s.checkpoint_save(path, t=0.0, step=1)
    s.checkpoint_wait()
    other = make((24, 20, 30), hc.FP64)
    with pytest.raises(hc.HcError, match="grid"):
        other.checkpoint_load(path)
    other32 = make(shape, hc.FP32)
    with pytest.raises(hc.HcError, match="precision"):
        other32.checkpoint_load(path)
    raw = bytearray(open(path, "rb").read())
    raw[200] ^= 0x40
    bad = str(tmp_path / "bad.ckpt")
    open(bad, "wb").write(bytes(raw))
    r = make(shape, hc.FP64)
    r.set_state(q0)
    before = r.state()
    with pytest.raises(hc.HcError, match="checksum"):
        r.checkpoint_load(bad)
    assert np.array_equal(r.state(), before)
    short = str(tmp_path / "short.ckpt")
    open(short, "wb").write(bytes(raw[:1000]))
    with pytest.raises(hc.HcError, match="shorter"):
        r.checkpoint_load(short)
    assert np.array_equal(r.state(), before)
