"""CPU oracle of the warm-start U-Net (test infrastructure only).

A torch CPU restatement of the network the library runs on the tensor cores
(hydrocode_astro1_b200/csrc/unet.cu): the same compact parameter vector, the
same operations (3x3x3 zero-padded convolutions, LeakyReLU(0.1), 2x average
pooling, 2x nearest upsampling with skip addition), the same loss
sum((out - t)^2) / sum(t^2).  Used to check the device forward pass and its
gradients.  The library has no counterpart in the reference code.
"""
import numpy as np
import torch
import torch.nn.functional as F

CH, NTAP, NLEV = 16, 27, 4
NCONV = 2 * NLEV + 2


def unpack(params, dtype=torch.float64):
    """compact vector -> list of (weight [co, ci, 3, 3, 3], bias [co])."""
    p = np.asarray(params, dtype=np.float64)
    q = 0
    out = []
    for l in range(NCONV):
        if l == 0:
            w = p[q:q + CH * NTAP].reshape(CH, NTAP, 1); q += CH * NTAP
            b = p[q:q + CH]; q += CH
        elif l == NCONV - 1:
            w = p[q:q + NTAP * CH].reshape(1, NTAP, CH); q += NTAP * CH
            b = p[q:q + 1]; q += 1
        else:
            w = p[q:q + CH * NTAP * CH].reshape(CH, NTAP, CH); q += CH * NTAP * CH
            b = p[q:q + CH]; q += CH
        wt = torch.tensor(w, dtype=dtype).reshape(w.shape[0], 3, 3, 3, w.shape[2]).permute(0, 4, 1, 2, 3)
        out.append((wt.contiguous(), torch.tensor(b, dtype=dtype)))
    assert q == p.size
    return out


def forward(layers, x):
    """x: [nx, ny, nz] level-0 input -> output [nx, ny, nz].  Encoder convs
    0..NLEV (pooling before each but the first), decoder convs NLEV+1..2 NLEV
    on (nearest upsample + skip), output conv 2 NLEV + 1."""
    f = lambda z: F.leaky_relu(z, 0.1)
    conv = lambda h, l: F.conv3d(h, layers[l][0], layers[l][1], padding=1)
    up = lambda h: F.interpolate(h, scale_factor=2, mode="nearest")
    e = [f(conv(x[None, None], 0))]
    for l in range(1, NLEV + 1):
        e.append(f(conv(F.avg_pool3d(e[-1], 2), l)))
    h = e[NLEV]
    for l in range(NLEV - 1, -1, -1):
        h = f(conv(up(h) + e[l], 2 * NLEV - l))
    return conv(h, NCONV - 1)[0, 0]


def loss_and_grad(params, x, t, bf16_weights=True):
    """Loss and compact gradient (FP64 autograd).  bf16_weights: evaluate at
    the BF16-rounded weights the device computes with (biases stay FP32)."""
    p = np.asarray(params, dtype=np.float32)
    layers = unpack(p)
    if bf16_weights:
        layers = [(w.to(torch.bfloat16).to(torch.float64), b) for w, b in layers]
    for w, b in layers:
        w.requires_grad_(True)
        b.requires_grad_(True)
    xt = torch.tensor(np.asarray(x), dtype=torch.float64)
    tt = torch.tensor(np.asarray(t), dtype=torch.float64)
    out = forward(layers, xt)
    loss = ((out - tt) ** 2).sum() / (tt ** 2).sum()
    loss.backward()
    g = []
    for l, (w, b) in enumerate(layers):
        gw = w.grad.permute(0, 2, 3, 4, 1).reshape(w.shape[0], NTAP, w.shape[1]).numpy()
        if l == 0:
            g.append(gw[:, :, 0].ravel())
        elif l == NCONV - 1:
            g.append(gw[0].ravel())
        else:
            g.append(gw.ravel())
        g.append(b.grad.numpy().ravel())
    return float(loss.detach()), np.concatenate(g), out.detach().numpy()


def blocks():
    """(start, stop, name) of each parameter block of the compact vector."""
    res, q = [], 0
    for l in range(NCONV):
        nw = CH * NTAP if l in (0, NCONV - 1) else CH * NTAP * CH
        nb = 1 if l == NCONV - 1 else CH
        res.append((q, q + nw, f"w{l}"))
        q += nw
        res.append((q, q + nb, f"b{l}"))
        q += nb
    return res
