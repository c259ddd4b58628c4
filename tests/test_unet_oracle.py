"""The CPU oracle of the learned stage (oracle/unet_ref.py) checked against
itself: analytic gradients against central finite differences (float64, no
rounding), the bf16 rounding helper against torch's, and the adjoint pairs
(pool / pool_t, up / up_t, conv / conv_dgrad) by the dot-product test."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import unet_ref as U  # noqa: E402


def _setup(n=8, seed=3):
    rng = np.random.default_rng(seed)
    W = U.init_weights(seed)
    r = rng.standard_normal((n, n, n))
    logd = rng.standard_normal((n, n, n)) * 0.5
    x0, _ = U.make_input(r, logd)
    t = rng.standard_normal((n, n, n))
    return W, x0, t


def test_bf16_matches_torch():
    import torch
    x = np.random.default_rng(0).standard_normal(10000) * 10.0 ** np.random.default_rng(1).integers(-8, 8, 10000)
    want = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(U.bf16(x), want)


def test_adjoints():
    rng = np.random.default_rng(5)
    a = rng.standard_normal((8, 6, 4, 3))
    b = rng.standard_normal((4, 3, 2, 3))
    assert abs(np.sum(U.pool(a) * b) - np.sum(a * U.pool_t(b))) < 1e-12
    assert abs(np.sum(U.up(b) * a) - np.sum(b * U.up_t(a))) < 1e-12
    w = rng.standard_normal((27, 5, 3))
    g = rng.standard_normal((8, 6, 4, 5))
    assert abs(np.sum(U.conv(a, w) * g) - np.sum(a * U.conv_dgrad(g, w))) < 1e-9
    # weight gradient: d<conv(a, w), g>/dw
    assert abs(np.sum(U.conv(a, w) * g) - np.sum(w * U.conv_wgrad(a, g))) < 1e-9


@pytest.mark.parametrize("name", ["W0", "W1", "W3", "W4", "W6", "w7"])
def test_gradients_match_finite_differences(name):
    W, x0, t = _setup()
    A = U.forward(x0, W, rounded=False)
    L, gy = U.loss(A["y"], t)
    G = U.backward(A, W, gy)
    rng = np.random.default_rng(11)
    w = W[name]
    for _ in range(4):
        idx = tuple(rng.integers(0, s) for s in w.shape)
        if name == "W0" and idx[2] >= 2:
            continue
        h = 1e-6
        w0 = w[idx]
        w[idx] = w0 + h
        Lp, _ = U.loss(U.forward(x0, W, rounded=False)["y"], t)
        w[idx] = w0 - h
        Lm, _ = U.loss(U.forward(x0, W, rounded=False)["y"], t)
        w[idx] = w0
        fd = (Lp - Lm) / (2 * h)
        assert abs(fd - G[name][idx]) <= 1e-6 * max(1.0, abs(fd)), (name, idx, fd, G[name][idx])
