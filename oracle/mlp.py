"""CPU restatement of the gravity surrogate's network, for checking the GPU's
forward pass and gradients.

TEST INFRASTRUCTURE ONLY (tests/).  The network and its parameter layout are
this build's own (the reference has no such surrogate): input x[4], four
hidden layers of 256 with SiLU, output y[3]; FP32 parameter vector
W0[256][4] b0[256] W1..W3[256][256] b1..b3[256] W4[3][256] b4[3].  The BF16
roundings follow the device: hidden activations and the hidden weight
matrices enter the 256 x 256 products as BF16, the back-propagated dZ of the
hidden layers is stored as BF16; everything else is FP32 (computed here in
FP64 and compared with a tolerance).
"""
from __future__ import annotations

import numpy as np

H = 256
OFF_W0 = 0
OFF_B0 = OFF_W0 + H * 4
OFF_W1 = OFF_B0 + H
OFF_B1 = OFF_W1 + 3 * H * H
OFF_W4 = OFF_B1 + 3 * H
OFF_B4 = OFF_W4 + 3 * H
PARAMS = OFF_B4 + 3


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32).copy()
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    W0 = p[OFF_W0:OFF_B0].reshape(H, 4)
    b0 = p[OFF_B0:OFF_W1]
    Ws = [p[OFF_W1 + l * H * H:OFF_W1 + (l + 1) * H * H].reshape(H, H) for l in range(3)]
    bs = [p[OFF_B1 + l * H:OFF_B1 + (l + 1) * H] for l in range(3)]
    W4 = p[OFF_W4:OFF_B4].reshape(3, H)
    b4 = p[OFF_B4:OFF_B4 + 3]
    return W0, b0, Ws, bs, W4, b4


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward_backward(p, x, t):
    """(loss, grad[PARAMS], y) with the device's BF16 roundings."""
    W0, b0, Ws, bs, W4, b4 = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    B = x.shape[0]
    z = [x @ W0.T + b0]
    h = [bf16(silu(z[0]))]
    for l in range(3):
        z.append(h[l] @ bf16(Ws[l]).T + bs[l])
        h.append(bf16(silu(z[l + 1])))
    y = h[3] @ W4.T + b4
    d = y - t
    loss = float((d * d).sum() / (3 * B))
    dy = 2.0 * d / (3 * B)
    g = np.zeros(PARAMS)
    g[OFF_W4:OFF_B4] = (dy.T @ h[3]).ravel()
    g[OFF_B4:OFF_B4 + 3] = dy.sum(axis=0)
    dz = bf16((dy @ W4) * silu_grad(z[3]))
    for l in (2, 1, 0):
        g[OFF_W1 + l * H * H:OFF_W1 + (l + 1) * H * H] = (dz.T @ h[l]).ravel()
        g[OFF_B1 + l * H:OFF_B1 + (l + 1) * H] = dz.sum(axis=0)
        dh = dz @ bf16(Ws[l])
        dz = bf16(dh * silu_grad(z[l]))
    g[OFF_B0:OFF_W1] = dz.sum(axis=0)
    g[OFF_W0:OFF_B0] = (dz.T @ x).ravel()
    return loss, g, y
