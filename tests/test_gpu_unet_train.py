"""The warm-start U-Net on the device: forward pass and gradients against
the CPU oracle (oracle/unet_ref.py, FP64 autograd at the BF16-rounded
weights), training on samples the solver records, and the effect of the
trained network inside mixed-precision solves.

Tolerances: the device keeps activations in BF16 between layers (8-bit
mantissa), so outputs agree to ~1% and each parameter block's gradient to
cosine similarity > 0.99 and norm within 5%."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")
torch = pytest.importorskip("torch")
from oracle import unet_ref  # noqa: E402
from hydrocode_astro1_b200 import problems  # noqa: E402


def smooth(shape, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape)
    for ax in range(3):
        a = (np.roll(a, 1, ax) + 2 * a + np.roll(a, -1, ax)) / 4
    return (a / a.std()).astype(np.float32)


def test_param_count():
    assert hc.lib().hc_unet_param_count() == 56305


@pytest.mark.parametrize("seed", [3, 11])
def test_forward_and_gradient_match_oracle(seed):
    s = hc.HydroSolver3D((32, 32, 32), G=1.0, precision=hc.FP32)
    s.unet_init(seed)
    p, k = s.unet_params()
    assert k == 30.0
    x = smooth((16, 16, 32), seed)
    t = smooth((16, 16, 32), seed + 100) * 0.5
    lg, gg, og = s.unet_loss_grad(x, t)
    lr_, gr, orf = unet_ref.loss_and_grad(p, x, t)
    assert np.linalg.norm(og - orf) / np.linalg.norm(orf) < 2e-2
    assert abs(lg - lr_) / lr_ < 3e-2
    for a, b, name in unet_ref.blocks():
        u, v = gg[a:b].astype(np.float64), gr[a:b]
        if np.linalg.norm(v) == 0:
            continue
        cos = u @ v / (np.linalg.norm(u) * np.linalg.norm(v))
        assert cos > 0.99, (name, cos)
        assert abs(np.linalg.norm(u) / np.linalg.norm(v) - 1) < 0.05, name
    s.close()


def _explosion_solver(n, warm):
    q, p = problems.stellar_explosion(n, r_exp_frac=0.06)
    s = hc.HydroSolver3D(p["shape"], lo=p["lo"], hi=p["hi"], gamma=p["gamma"], G=p["G"], bc=p["bc"],
                         lmax=p["lmax"], cfl=p["cfl"], tol=1e-8, max_iter=200000, precision=hc.FP32,
                         moment_order=hc.MOMENTS_TREE, warm_start=warm)
    s.set_state(q)
    return s


def test_training_and_learned_warm_start_in_solver():
    """Record (residual, correction) pairs from 30 solves, train on them on
    the device, then run the next steps with the learned start: fewer SOR
    iterations than the previous-potential start at the same tolerance, and
    the same flow."""
    n = 64
    a = _explosion_solver(n, hc.HC_WARM_PREVIOUS)
    a.unet_collect(32)
    a.unet_init(1)
    a.step(30)
    assert a.unet_samples() == 30
    l0 = a.unet_train(20, lr=1e-3, seed=2)
    l1 = a.unet_train(600, lr=1e-3, seed=3)
    assert l1 < 0.25 * l0, (l0, l1)
    params, kscale = a.unet_params()
    b = _explosion_solver(n, hc.HC_WARM_UNET)
    b.set_state(a.state())
    b.set_phi(a.phi())
    b.unet_load(params, kscale)
    it_a, it_b = [], []
    for _ in range(6):
        a.step(1)
        it_a.append(a.diagnostics()["last_iterations"])
        b.step(1)
        it_b.append(b.diagnostics()["last_iterations"])
    d = b.diagnostics()
    assert d["unet_accepted"] + d["unet_fallbacks"] == 6
    assert d["unet_accepted"] >= 4, d
    assert np.mean(it_b) < 0.9 * np.mean(it_a), (it_a, it_b)
    ra, rb = a.state()[0], b.state()[0]
    assert np.abs(ra - rb).mean() / np.abs(ra).mean() < 1e-5
    a.close()
    b.close()
