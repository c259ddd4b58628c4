"""The learned FGMRES stage end to end on the GPU: training lowers the loss,
the trained network (weights/unet_heat64.npz, trained by learned.py on 2000
pairs from 64^3 instances) cuts FGMRES iterations on an instance it never
saw, the answer is the FP64 one, and a useless network falls back to the
plain ILU2 step."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def _solve(ctx, s, net_w, grid, restart=30, eps=1e-8):
    import bsg
    import learned as L
    import torch
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", L.ilu2_param(6))
    b = torch.as_tensor(s.rhs[0], device="cuda")
    p = L.ilu2_param(6, krylov=2, restart=restart, eps=eps, sttype=1, niter=2000)
    net = None
    if net_w is not None:
        net = bsg.UNet(ctx, grid, grid, grid)
        net.set_weights(net_w)
        net.set_matrix(m)
        p.learned = net.h.value
    x = torch.zeros_like(b)
    bsg.gmres(ctx, m, f, b, x, p)
    return x.cpu().numpy(), p


def test_training_lowers_loss(ctx):
    import learned as L
    data = L.make_pairs(ctx, grid=16, instances=12, per=8, sigma=1.5, seed0=500, log=None)
    _, hist = L.train(ctx, data, 16, epochs=4, batch=4, lr=2e-3, seed=1, log=None)
    assert hist[-1] < 0.95 * hist[0], hist


def test_learned_fgmres_gain_on_unseen_instance(ctx):
    import learned as L
    w = L.load()
    g = 64
    s = P.heat3d(g, g, g, sigma=1.5, seed=4)  # training used seeds 1000..1099
    x0, p0 = _solve(ctx, s, None, g)
    x1, p1 = _solve(ctx, s, w, g)
    assert p0.resfin <= 1e-8 and p1.resfin <= 1e-8
    assert p1.nitperf <= 0.85 * p0.nitperf, (p1.nitperf, p0.nitperf)
    A = s.to_scipy()
    b = s.rhs[0]
    assert np.linalg.norm(b - A @ x1) <= 1e-8 * np.linalg.norm(b)
    assert np.linalg.norm(x1 - x0) <= 1e-6 * np.linalg.norm(x0)


def test_useless_network_falls_back_to_ilu2(ctx):
    import learned as L
    g = 32
    s = P.heat3d(g, g, g, sigma=1.5, seed=7)
    _, p0 = _solve(ctx, s, None, g)
    _, p1 = _solve(ctx, s, np.zeros(L.NPARAM, np.float32), g)  # output 0: no step
    assert p1.nitperf == p0.nitperf and p1.resfin <= 1e-8
