"""Training of the learned FGMRES stage (the U-Net of csrc/unet.cu).

The network learns the error that one FP32 ILU2 step leaves behind.  For an
iterate x_k of a seeded ILU2-PCG solve of A x = b (3-D heat, 7-point
stencil, lognormal conductivity):

    r_k = b - A x_k,  z0 = M^{-1} r_k  (the ILU2 step used inside FGMRES)
    input  r1 = r_k - A z0            (residual after the ILU2 step)
    target e1 = x* - x_k - z0         (error after the ILU2 step)

with x* the converged solution.  FGMRES then applies z = z0 + alpha N(r1/|r1|),
alpha = (r1 . y) / (y . A y) the A-norm-optimal step of the direction y.
Every product, solve and training step runs in the library's kernels through
bsg; this module only drives them.

    python learned.py --grid 64 --instances 100 --per 20 --epochs 6 --out weights/unet_heat64.npz
    python learned.py --time-forward 128     # time the committed network's forward at 128^3
"""
import argparse
import math
import os
import time

import numpy as np

import bsg
import problems as P

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "unet_heat64.npz")

# (cin, cout) of W0..W6; W0 reads 16 channels of which the first two are used
LAYERS = ((16, 16), (16, 32), (32, 64), (64, 64), (128, 32), (64, 16), (32, 16))
NPARAM = sum(27 * ci * co for ci, co in LAYERS) + 16


def init_weights(seed=0):
    """He-normal initial weights in the flat layout of bsg_unet_set_weights."""
    rng = np.random.default_rng(seed)
    parts = []
    for k, (cin, cout) in enumerate(LAYERS):
        fan = 27 * (2 if k == 0 else cin)
        w = rng.standard_normal((27, cout, cin)) * np.sqrt(2.0 / fan)
        if k == 0:
            w[:, :, 2:] = 0.0
        parts.append(w.reshape(-1))
    parts.append(rng.standard_normal(16) * np.sqrt(1.0 / 16))
    return np.concatenate(parts).astype(np.float32)


def ilu2_param(nsweeps=6, **kw):
    """The preconditioner setting of the learned FGMRES: FP32 IC2/ILU2 factor
    (tau 1e-3), triangular solves by Jacobi sweeps."""
    base = dict(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, precision=1, trisolve=1,
                nsweeps=nsweeps, ittype=0)
    base.update(kw)
    return bsg.default_param(**base)


def precond(f, r, nsweeps):
    import torch
    t = torch.empty_like(r)
    z = torch.empty_like(r)
    f.solve_l(r, t, mode=1, nsweeps=nsweeps)
    f.solve_u(t, z, mode=1, nsweeps=nsweeps)
    return z


def make_pairs(ctx, grid=64, instances=100, per=20, sigma=1.5, seed0=1000, nsweeps=6, kstep=2, log=print):
    """(r1, e1) pairs from the iterates 0, kstep, 2 kstep, ... of ILU2-PCG
    solves on `instances` seeded grid^3 heat problems.  Returns device
    tensors R, T (float32, [pairs, n]), D (float64 diagonals, [instances, n])
    and the instance index of each pair."""
    import torch
    n = grid ** 3
    npair = instances * per
    R = torch.empty((npair, n), dtype=torch.float32, device="cuda")
    T = torch.empty((npair, n), dtype=torch.float32, device="cuda")
    D = torch.empty((instances, n), dtype=torch.float64, device="cuda")
    inst = np.repeat(np.arange(instances), per)
    t0 = time.time()
    q = 0
    for i in range(instances):
        s = P.heat3d(grid, grid, grid, sigma=sigma, seed=seed0 + i)
        u = s.upper()
        D[i] = torch.as_tensor(u.a[u.ia[:-1]], device="cuda")
        m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
        f = bsg.Factor(ctx, m, "ich2", ilu2_param(nsweeps))
        b = torch.as_tensor(s.rhs[0], device="cuda")
        xs = torch.zeros_like(b)
        bsg.pcg(ctx, m, f, b, xs, ilu2_param(nsweeps, eps=1e-12, niter=2000))
        Ax = torch.empty_like(b)
        for j in range(per):
            k = j * kstep
            x = torch.zeros_like(b)
            if k > 0:
                try:
                    bsg.pcg(ctx, m, f, b, x, ilu2_param(nsweeps, eps=1e-30, niter=k, true_residual=0))
                except bsg.BsgError as e:
                    if e.code != bsg.ERR_NOCONV:
                        raise
            m.mvm(x, Ax)
            r = b - Ax
            z0 = precond(f, r, nsweeps)
            m.mvm(z0, Ax)
            R[q] = (r - Ax).float()
            T[q] = (xs - x - z0).float()
            q += 1
        f.free()
        m.free()
        if log and (i + 1) % max(1, instances // 10) == 0:
            log(f"pairs: {q}/{npair} ({time.time() - t0:.1f} s)")
    return R, T, D, inst


def evaluate(net, data, idx):
    """Mean loss 1 - cos^2 of the network over the pairs `idx` (the
    gradients this accumulates are discarded)."""
    import torch
    R, T, D, inst = data
    n = R.shape[1]
    r64 = torch.empty(n, dtype=torch.float64, device="cuda")
    t64 = torch.empty(n, dtype=torch.float64, device="cuda")
    out = []
    for i in idx:
        net.set_diag(D[inst[i]])
        r64.copy_(R[i])
        t64.copy_(T[i])
        out.append(net.train_sample(r64, t64, want_loss=True))
    net.zero_grads()
    return float(np.mean(out))


def train(ctx, data, grid, epochs=6, batch=8, lr=2e-3, seed=0, weights=None, neval=64, log=print):
    """Adam over the pairs with a cosine learning-rate decay.  Returns the
    trained flat weights and the mean loss on a fixed set of `neval` pairs
    before training and after each epoch."""
    import torch
    R, T, D, inst = data
    npair, n = R.shape
    net = bsg.UNet(ctx, grid, grid, grid, train=True)
    net.set_weights(init_weights(seed) if weights is None else weights)
    rng = np.random.default_rng(seed)
    ev = np.random.default_rng(seed + 12345).choice(npair, size=min(neval, npair), replace=False)
    r64 = torch.empty(n, dtype=torch.float64, device="cuda")
    t64 = torch.empty(n, dtype=torch.float64, device="cuda")
    nsteps = epochs * math.ceil(npair / batch)
    step = 0
    hist = [evaluate(net, data, ev)]
    t0 = time.time()
    for ep in range(epochs):
        perm = rng.permutation(npair)
        for b0 in range(0, npair, batch):
            for idx in perm[b0:b0 + batch]:
                net.set_diag(D[inst[idx]])
                r64.copy_(R[idx])
                t64.copy_(T[idx])
                net.train_sample(r64, t64)
            step += 1
            lr_t = 0.5 * lr * (1.0 + math.cos(math.pi * (step - 1) / nsteps))
            net.adam(lr_t, step)
        hist.append(evaluate(net, data, ev))
        if log:
            log(f"epoch {ep + 1}/{epochs}: loss {hist[-1]:.4f} ({time.time() - t0:.1f} s)")
    w = net.weights()
    net.free()
    return w, hist


def save(path, w, meta):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, w=w, **{k: np.asarray(v) for k, v in meta.items()})


def load(path=DEFAULT_WEIGHTS):
    z = np.load(path)
    w = z["w"].astype(np.float32)
    if w.size != NPARAM:
        raise ValueError(f"{path}: {w.size} weights, expected {NPARAM}")
    return w


def time_forward(grid, reps=20, sigma=1.5, seed=4, log=print):
    """Time the forward pass of the committed network bound to the grid^3 heat
    system (CUDA events on the library stream, after 3 warm-up calls)."""
    import torch
    ctx = bsg.Context(0)
    s = P.heat3d(grid, sigma=sigma, seed=seed)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    net = bsg.UNet(ctx, grid, grid, grid)
    net.set_weights(load())
    net.set_matrix(m)
    r = torch.as_tensor(np.random.default_rng(seed).standard_normal(s.n), device="cuda")
    y = torch.empty_like(r)
    for _ in range(3):
        net.forward(r, y)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        net.forward(r, y)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    log(f"U-Net forward at {grid}^3: {ms:.3f} ms ({reps} calls)")
    net.free()
    return ms


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--grid", type=int, default=64)
    ap.add_argument("--instances", type=int, default=100)
    ap.add_argument("--per", type=int, default=20)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--sigma", type=float, default=1.5)
    ap.add_argument("--nsweeps", type=int, default=6)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--time-forward", type=int, default=0, metavar="GRID",
                    help="only time the committed network's forward on the GRID^3 heat system")
    a = ap.parse_args()
    if a.time_forward:
        time_forward(a.time_forward)
        return
    ctx = bsg.Context(0)
    data = make_pairs(ctx, a.grid, a.instances, a.per, a.sigma, nsweeps=a.nsweeps)
    w, hist = train(ctx, data, a.grid, a.epochs, a.batch, a.lr, a.seed)
    save(a.out, w, dict(grid=a.grid, instances=a.instances, per=a.per, epochs=a.epochs, sigma=a.sigma,
                        nsweeps=a.nsweeps, loss=hist))
    print(f"saved {a.out}")


if __name__ == "__main__":
    main()
