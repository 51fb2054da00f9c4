"""Tensor-core (tcgen05) convolution kernels of the learned warm start vs
torch CPU (FP32/FP64) on the same BF16-rounded operands.

The kernels multiply BF16 operands exactly and accumulate in FP32, so the FP32
outputs agree with an FP64 reference to FP32 summation error (tolerance 1e-5
of the output scale); BF16-rounded outputs to one BF16 ulp (2^-8 relative).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

hc = pytest.importorskip("hydrocode_astro1_b200")
torch = pytest.importorskip("torch")


def bf16(a):
    """float array -> (BF16-rounded float32 array, uint16 bits)."""
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16)
    return t.float().numpy(), t.view(torch.int16).numpy().view(np.uint16).copy()


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def conv_gpu(x16, w16, bias, shape, mode, act):
    L = hc.lib()
    L.hc_unet_conv_test.restype = C.c_int
    n = int(np.prod(shape))
    out = np.zeros(n * (1 if mode == 2 else 16), np.float32)
    rc = L.hc_unet_conv_test(*shape, _p(x16, C.c_uint16), _p(w16, C.c_uint16), _p(bias, C.c_float), mode, act,
                             _p(out, C.c_float))
    assert rc == 0, hc.lib().hc_last_error()
    return out


def conv_ref(x, w, bias, shape):
    """x [n,16], w [co][tap][ci] -> y [n,16] in FP64 (zero padding)."""
    xt = torch.from_numpy(x.astype(np.float64)).reshape(*shape, 16).permute(3, 0, 1, 2)[None]
    wt = torch.from_numpy(w.astype(np.float64)).reshape(16, 3, 3, 3, 16).permute(0, 4, 1, 2, 3)
    y = torch.nn.functional.conv3d(xt, wt, torch.from_numpy(bias.astype(np.float64)), padding=1)
    return y[0].permute(1, 2, 3, 0).reshape(-1, 16).numpy()


@pytest.mark.parametrize("shape", [(5, 6, 7), (16, 16, 16), (3, 40, 9)])
def test_conv_forward_modes(shape):
    rng = np.random.default_rng(1)
    n = int(np.prod(shape))
    x, x16 = bf16(rng.standard_normal((n, 16)))
    w, w16 = bf16(rng.standard_normal((16, 27, 16)) * 0.1)
    bias = rng.standard_normal(16).astype(np.float32)
    ref = conv_ref(x, w, bias, shape)
    scale = np.abs(ref).max()
    y3 = conv_gpu(x16, w16, bias, shape, 3, 0).reshape(n, 16)
    np.testing.assert_allclose(y3, ref, atol=1e-5 * scale)
    y2 = conv_gpu(x16, w16, bias, shape, 2, 0)
    np.testing.assert_allclose(y2, ref[:, 0], atol=1e-5 * scale)
    y0 = conv_gpu(x16, w16, bias, shape, 0, 1).reshape(n, 16)
    lk = np.where(ref > 0, ref, 0.1 * ref)
    np.testing.assert_allclose(y0, lk, rtol=2 ** -8, atol=1e-5 * scale)


def test_conv_input_gradient_by_flipped_weights():
    """dX = conv(dY, W') with W'[ci][tap][co] = W[co][26-tap][ci] equals
    torch's gradient of the forward convolution."""
    shape = (7, 9, 6)
    rng = np.random.default_rng(2)
    n = int(np.prod(shape))
    x, _ = bf16(rng.standard_normal((n, 16)))
    w, _ = bf16(rng.standard_normal((16, 27, 16)) * 0.1)
    dy, dy16 = bf16(rng.standard_normal((n, 16)))
    wf = np.ascontiguousarray(w[:, ::-1, :].transpose(2, 1, 0))
    _, wf16 = bf16(wf)
    got = conv_gpu(dy16, wf16, np.zeros(16, np.float32), shape, 3, 0).reshape(n, 16)
    xt = torch.from_numpy(x.astype(np.float64)).reshape(*shape, 16).permute(3, 0, 1, 2)[None].requires_grad_()
    wt = torch.from_numpy(w.astype(np.float64)).reshape(16, 3, 3, 3, 16).permute(0, 4, 1, 2, 3)
    y = torch.nn.functional.conv3d(xt, wt, padding=1)
    g = torch.from_numpy(dy.astype(np.float64)).reshape(*shape, 16).permute(3, 0, 1, 2)[None]
    y.backward(g)
    ref = xt.grad[0].permute(1, 2, 3, 0).reshape(-1, 16).numpy()
    np.testing.assert_allclose(got, ref, atol=1e-5 * np.abs(ref).max())


@pytest.mark.parametrize("shape,parts", [((5, 6, 7), 1), ((16, 16, 16), 3), ((9, 11, 13), 148)])
def test_weight_gradient(shape, parts):
    rng = np.random.default_rng(3)
    n = int(np.prod(shape))
    x, x16 = bf16(rng.standard_normal((n, 16)))
    dy, dy16 = bf16(rng.standard_normal((n, 16)))
    L = hc.lib()
    dw = np.zeros((16, 27, 16), np.float32)
    rc = L.hc_unet_wgrad_test(*shape, _p(x16, C.c_uint16), _p(dy16, C.c_uint16), parts, _p(dw, C.c_float))
    assert rc == 0
    xt = torch.from_numpy(x.astype(np.float64)).reshape(*shape, 16).permute(3, 0, 1, 2)[None]
    wt = torch.zeros(16, 16, 3, 3, 3, dtype=torch.float64, requires_grad=True)
    y = torch.nn.functional.conv3d(xt, wt, padding=1)
    y.backward(torch.from_numpy(dy.astype(np.float64)).reshape(*shape, 16).permute(3, 0, 1, 2)[None])
    ref = wt.grad.permute(0, 2, 3, 4, 1).reshape(16, 27, 16).numpy()
    np.testing.assert_allclose(dw, ref, atol=1e-5 * np.abs(ref).max())
