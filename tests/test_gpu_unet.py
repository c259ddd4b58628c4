"""GPU kernels of the learned stage (csrc/unet.cu) against the CPU oracle
(oracle/unet_ref.py): forward output and weight gradients of one sample.

Tolerances: the GPU accumulates in FP32 and rounds the gradient tensors it
feeds the backward convolutions to bf16 (the oracle keeps them in float64),
so outputs are held to 1e-2 of their maximum and the gradient of each weight
tensor to 5e-2 in relative 2-norm (W0's gradient passes through seven such
bf16 roundings, about 3e-2 observed).
"""
import os
import sys

import numpy as np
import pytest

import problems as P

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import unet_ref as U  # noqa: E402

pytestmark = pytest.mark.gpu


def _flat(W):
    return np.concatenate([W[k].reshape(-1) for k in U.NAMES] + [W["w7"]]).astype(np.float32)


def _unflat(w):
    out, o = {}, 0
    for k in U.NAMES:
        cin, cout = U.CH[k]
        n = 27 * cin * cout
        out[k] = w[o:o + n].reshape(27, cout, cin).astype(np.float64)
        o += n
    out["w7"] = w[o:o + 16].astype(np.float64)
    return out


def _logd(s, n):
    d = s.a[s.ia[:-1]]  # diagonal first in each row of the upper storage
    ld = np.log(np.abs(d) + 1e-300)
    sd = ld.std()
    return U.bf16((ld - ld.mean()) / (sd if sd ** 2 > 1e-30 else 1.0)).reshape(n, n, n)


@pytest.fixture(scope="module", params=[16, 32])
def setup(ctx, request):
    """16^3 runs the direct kernel at every level; 32^3 puts the finest level
    on the shared-memory tiled kernel (x extent a multiple of 32)."""
    import bsg
    n = request.param
    s = P.heat3d(n, n, n, sigma=1.0, seed=9)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    W = U.init_weights(2)
    rng = np.random.default_rng(4)
    r = rng.standard_normal(s.n)
    t = rng.standard_normal(s.n)
    return s, m, W, r, t, _logd(s.upper(), n), n


def test_unet_forward_matches_oracle(ctx, setup):
    import bsg
    import torch
    s, m, W, r, _, logd, n = setup
    net = bsg.UNet(ctx, n, n, n)
    net.set_weights(_flat(W))
    net.set_matrix(m)
    y = torch.empty(s.n, dtype=torch.float64, device="cuda")
    net.forward(torch.as_tensor(r, device="cuda"), y)
    x0, nr = U.make_input(r.reshape(n, n, n), logd)
    want = U.forward(x0, W)["y"].reshape(-1)
    got = y.cpu().numpy()
    assert np.all(np.isfinite(got))
    assert np.abs(got - want).max() <= 1e-2 * np.abs(want).max()
    assert np.linalg.norm(got - want) <= 5e-3 * np.linalg.norm(want)


def test_unet_gradients_match_oracle(ctx, setup):
    import bsg
    import torch
    s, m, W, r, t, logd, n = setup
    net = bsg.UNet(ctx, n, n, n, train=True)
    net.set_weights(_flat(W))
    net.set_matrix(m)
    loss = net.train_sample(torch.as_tensor(r, device="cuda"), torch.as_tensor(t, device="cuda"), want_loss=True)
    G = _unflat(net.grads())
    x0, nr = U.make_input(r.reshape(n, n, n), logd)
    A = U.forward(x0, W)
    L, gy = U.loss(A["y"], t.reshape(n, n, n))
    want = U.backward(A, W, gy)
    assert abs(loss - L) <= 1e-3 * max(L, 1e-3)
    for k in list(U.NAMES) + ["w7"]:
        err = np.linalg.norm(G[k] - want[k]) / np.linalg.norm(want[k])
        assert err <= 5e-2, (k, err)


def test_unet_adam_step_lowers_loss(ctx, setup):
    import bsg
    import torch
    s, m, W, r, t, _, n = setup
    net = bsg.UNet(ctx, n, n, n, train=True)
    net.set_weights(_flat(W))
    net.set_matrix(m)
    rt, tt = torch.as_tensor(r, device="cuda"), torch.as_tensor(t, device="cuda")
    losses = []
    for step in range(1, 41):
        losses.append(net.train_sample(rt, tt, want_loss=True))
        net.adam(2e-3, step)
    assert losses[-1] < 0.95 * losses[0], losses[::10]
    w = net.weights()
    assert np.all(_unflat(w)["W0"][:, :, 2:] == 0.0)


@pytest.mark.parametrize("ny,nz", [(16, 8), (120, 40)])
def test_unet_forward_tensor_core_level_matches_oracle(ctx, ny, nz):
    """A grid 128 voxels wide puts the level-0 convolutions (16 -> 16 and the
    decoder's 32 -> 16 with its upsampled half) on the tcgen05 kernel (x-lines
    of 128 voxels, TMA-staged, the accumulators in tensor memory); the whole
    forward still matches the oracle within the bf16 tolerance of the other
    forward test.  Each CTA takes a contiguous range of the nz * ny output
    rows: at 16 x 8 one row each (128 CTAs), at 120 x 40 about 16 rows
    (296 CTAs) that often span two z planes, so the ring of row accumulators
    wraps across segments."""
    import bsg
    import torch
    nx = 128
    s = P.heat3d(nx, ny, nz, sigma=1.0, seed=19)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    W = U.init_weights(3)
    r = np.random.default_rng(14).standard_normal(s.n)
    u = s.upper()
    d = u.a[u.ia[:-1]]
    ld = np.log(np.abs(d) + 1e-300)
    logd = U.bf16((ld - ld.mean()) / ld.std()).reshape(nz, ny, nx)
    net = bsg.UNet(ctx, nx, ny, nz)
    net.set_weights(_flat(W))
    net.set_matrix(m)
    y = torch.empty(s.n, dtype=torch.float64, device="cuda")
    for _ in range(2):  # the second call reuses the kernels' state (TMEM, barriers)
        net.forward(torch.as_tensor(r, device="cuda"), y)
    x0, nr = U.make_input(r.reshape(nz, ny, nx), logd)
    want = U.forward(x0, W)["y"].reshape(-1)
    got = y.cpu().numpy()
    assert np.all(np.isfinite(got))
    assert np.abs(got - want).max() <= 1e-2 * np.abs(want).max()
    assert np.linalg.norm(got - want) <= 5e-3 * np.linalg.norm(want)
