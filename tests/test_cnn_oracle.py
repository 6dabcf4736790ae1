"""The warm-start network's CPU oracle (oracle/cnn_oracle.py): its backward passes
against central finite differences of its forward pass, and BF16 rounding."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import cnn_oracle as co  # noqa: E402  (the oracle is test infrastructure)


def small_net(rng, ci=3, hidden=4, cout=2):
    layers = []
    chans = [ci, hidden, hidden, cout]
    for i in range(3):
        a, b = chans[i], chans[i + 1]
        w = rng.standard_normal((b, co.kpad(a))) * 0.3
        w[:, 9 * a:] = 0.0
        layers.append((w, rng.standard_normal(b) * 0.1, i < 2))
    return layers


def loss_of(x, layers, target):
    out = co.forward(x, layers)[-1]
    return co.mse(out, target, target.shape[-1])[0]


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, 5, 6, 3))
    layers = small_net(rng)
    target = rng.standard_normal((2, 5, 6, 2))
    acts = co.forward(x, layers)
    L, g = co.mse(acts[-1], target, 2)
    grads = co.backward(acts, layers, g)
    h = 1e-6
    for li, (r, c) in [(0, (1, 5)), (1, (3, 20)), (2, (0, 30)), (0, (2, 26))]:
        w = layers[li][0]
        w0 = w[r, c]
        w[r, c] = w0 + h; Lp = loss_of(x, layers, target)
        w[r, c] = w0 - h; Lm = loss_of(x, layers, target)
        w[r, c] = w0
        fd = (Lp - Lm) / (2 * h)
        assert abs(fd - grads[li][0][r, c]) <= 1e-6 * max(1.0, abs(fd)), (li, r, c, fd, grads[li][0][r, c])
    for li in range(3):
        b = layers[li][1]
        b0 = b[0]
        b[0] = b0 + h; Lp = loss_of(x, layers, target)
        b[0] = b0 - h; Lm = loss_of(x, layers, target)
        b[0] = b0
        assert abs((Lp - Lm) / (2 * h) - grads[li][1][0]) <= 1e-6 * max(1.0, abs(grads[li][1][0]))


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.01171875, -3.140625, 65504.0, 1e-30], dtype=np.float32)
    r = co.bf16(x)
    # 1 + 2^-8 is the midpoint of 1 and 1 + 2^-7: ties go to the even mantissa (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.015625)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)
