"""FP64 restatement of the neural radiance cache's network (test
infrastructure: only tests and the bench's checks use it).

Mirrors csrc/nrc.cu: the encoding (10 inputs x 12 frequencies x (sin, cos),
the raw inputs, a constant 1, zero padding to 256), 5 bias-free layers
256 -> 64 -> 64 -> 64 -> 64 -> 16 (rows 3..15 zero) with ReLU, the relative
L2 loss (y - t)^2 / (sg(y)^2 + 0.01) averaged over samples and RGB, its
backward pass, and Adam. With `bf16=True` the operands are rounded to
bfloat16 where the GPU rounds them (weights, encoded inputs, hidden
activations, the gradient operand of each tensor-core product); sums stay
in FP64. There is no reference counterpart to pin against; the gradient is
checked against finite differences of this same model.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT, LAYERS, FREQS, USED = 256, 64, 16, 5, 12, 10
SHAPES = [(HID, IN), (HID, HID), (HID, HID), (HID, HID), (OUT, HID)]
OFFS = np.cumsum([0] + [a * b for a, b in SHAPES])
PARAMS = int(OFFS[-1])


def bf16(a):
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, np.float64)
    return [w[OFFS[l]:OFFS[l + 1]].reshape(SHAPES[l]) for l in range(LAYERS)]


def pack(mats):
    return np.concatenate([m.reshape(-1) for m in mats])


def encode(x):
    """x: (n, 12) inputs (10 used) -> (n, 256)."""
    x = np.asarray(x, np.float32).astype(np.float64)[:, :USED]
    n = x.shape[0]
    f = np.zeros((n, IN))
    for i in range(USED):
        for j in range(FREQS):
            a = np.pi * x[:, i] * (2.0 ** j)
            f[:, 2 * FREQS * i + 2 * j] = np.sin(a)
            f[:, 2 * FREQS * i + 2 * j + 1] = np.cos(a)
    f[:, 2 * FREQS * USED:2 * FREQS * USED + USED] = x
    f[:, 2 * FREQS * USED + USED] = 1.0
    return f


def forward(w, x, bf=True):
    """Returns the outputs (n, 16) and the layer inputs [enc, h0, h1, h2, h3]."""
    W = unpack(w)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    a = r(encode(x))
    inputs = [a]
    for l in range(LAYERS):
        z = a @ r(W[l]).T
        if l < LAYERS - 1:
            a = r(np.maximum(z, 0.0))
            inputs.append(a)
        else:
            y = z
    return y, inputs


def loss_grad(w, x, t, bf=True):
    """Mean relative L2 loss and its gradient with respect to w."""
    W = unpack(w)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    y, ins = forward(w, x, bf)
    t = np.asarray(t, np.float64)[:, :3]
    n = y.shape[0]
    yc = y[:, :3]
    den = yc * yc + 0.01
    loss = float(np.sum((yc - t) ** 2 / den) / (3 * n))
    g = np.zeros_like(y)
    g[:, :3] = 2.0 * (yc - t) / den / (3 * n)
    grads = [None] * LAYERS
    for l in range(LAYERS - 1, -1, -1):
        grads[l] = g.T @ ins[l]
        if l > 0:
            d = r(g) @ r(W[l])
            g = d * (ins[l] > 0)
    return loss, pack(grads)


def adam(w, g, m, v, step, lr=1e-2, b1=0.9, b2=0.99, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return w - lr * mh / (np.sqrt(vh) + eps), m, v


def init(seed=1):
    """Random weights in the library's shapes (not its generator)."""
    rng = np.random.default_rng(seed)
    mats = []
    for l, (o, i) in enumerate(SHAPES):
        m = rng.uniform(-1, 1, (o, i)) * np.sqrt(6.0 / i)
        if l == LAYERS - 1:
            m[3:] = 0.0
        mats.append(m)
    return pack(mats).astype(np.float32)
