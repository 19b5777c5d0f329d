"""The FP64 model of the radiance cache's network (oracle/nrc.py), the
checker of the GPU kernels' gradients: its analytic gradient against
central finite differences, in exact arithmetic (no bf16 rounding)."""
from __future__ import annotations

import numpy as np

from oracle import nrc


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 12), np.float32)
    x[:, :10] = rng.random((n, 10))
    t = np.zeros((n, 4), np.float32)
    t[:, :3] = rng.random((n, 3)) * 2.0
    return x, t


def _fixed_loss(w, x, t, den):
    # the loss with its denominator held at the unperturbed prediction: the
    # relative L2 loss stops the gradient through sg(y)^2
    y, _ = nrc.forward(w, x, bf=False)
    return float(np.sum((y[:, :3] - t[:, :3]) ** 2 / den) / (3 * y.shape[0]))


def test_gradient_matches_finite_differences():
    x, t = _data(37, 1)
    w = nrc.init(3).astype(np.float64)
    _, g = nrc.loss_grad(w, x, t, bf=False)
    y0, _ = nrc.forward(w, x, bf=False)
    den = y0[:, :3] ** 2 + 0.01
    rng = np.random.default_rng(5)
    # a few weights of every layer, away from ReLU kinks with high probability
    for l in range(nrc.LAYERS):
        lo, hi = int(nrc.OFFS[l]), int(nrc.OFFS[l + 1])
        rows = 3 if l == nrc.LAYERS - 1 else nrc.SHAPES[l][0]
        for _ in range(6):
            i = lo + int(rng.integers(rows * nrc.SHAPES[l][1]))
            h = 1e-6 * max(1.0, abs(w[i]))
            wp, wm = w.copy(), w.copy()
            wp[i] += h
            wm[i] -= h
            lp = _fixed_loss(wp, x, t, den)
            lm = _fixed_loss(wm, x, t, den)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)) + 1e-7, (l, i, fd, g[i])


def test_loss_is_the_mean_relative_l2():
    x, t = _data(9, 2)
    w = nrc.init(4)
    y, _ = nrc.forward(w, x, bf=False)
    want = np.mean((y[:, :3] - t[:, :3]) ** 2 / (y[:, :3] ** 2 + 0.01))
    got, _ = nrc.loss_grad(w, x, t, bf=False)
    assert abs(got - want) <= 1e-12 * max(1.0, want)


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3], np.float32)
    r = nrc.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 3.0e-3 * 2 ** -8
