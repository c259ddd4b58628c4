"""CPU oracle of the learned preconditioner stage -- TEST INFRASTRUCTURE ONLY.

The 4-level 3D convolutional U-Net that follows the ILU2 sweep inside FGMRES
has no counterpart in the reference (Bslib has no learned or reduced-precision
part), so this file is the definition the CUDA kernels (bcm-problems_b200/
csrc/unet.cu) are checked against: the same network, forward and backward, in
float64 numpy.  Only tests/ may import it.

Network (channels-last tensors [z, y, x, c]; R0 = the grid, Rl = R0 / 2^l):

    x0 = [r / |r|, (log diag(A) - mean) / std, 0 ... 0]      R0, 16 channels
    e0 = relu(conv(x0;  W0: 16 -> 16))                        R0
    e1 = relu(conv(pool(e0); W1: 16 -> 32))                   R1
    e2 = relu(conv(pool(e1); W2: 32 -> 64))                   R2
    e3 = relu(conv(pool(e2); W3: 64 -> 64))                   R3
    d2 = relu(conv(cat(up(e3), e2); W4: 128 -> 32))           R2
    d1 = relu(conv(cat(up(d2), e1); W5:  64 -> 16))           R1
    d0 = relu(conv(cat(up(d1), e0); W6:  32 -> 16))           R0
    y  = sum_c w7[c] d0[c]                                    R0
    correction = alpha * y,  alpha = (r . y) / (y . A y)      (energy-optimal)

conv: 3x3x3, zero padding, no bias, W[tap][cout][cin] with tap = 9 (dz+1) +
3 (dy+1) + (dx+1); pool: 2x2x2 mean; up: nearest (parent = coordinate // 2).
Training minimises 1 - cos^2(y, e) against the error e the ILU2 step left,
so only the direction of y is learned; the step length is the minimiser of
the A-norm of the remaining error.  The GPU stores activations in bfloat16 (round to nearest
even) after each relu / pool and accumulates in float32; `forward(...,
rounded=True)` reproduces those rounding points (accumulating in float64).
"""
import numpy as np

CH = {"W0": (16, 16), "W1": (16, 32), "W2": (32, 64), "W3": (64, 64),
      "W4": (128, 32), "W5": (64, 16), "W6": (32, 16)}
NAMES = ("W0", "W1", "W2", "W3", "W4", "W5", "W6")


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def init_weights(seed=0):
    """He-normal weights (bf16-rounded), W0's padded input channels zero."""
    rng = np.random.default_rng(seed)
    W = {}
    for k in NAMES:
        cin, cout = CH[k]
        fan = 27 * (2 if k == "W0" else cin)
        w = rng.standard_normal((27, cout, cin)) * np.sqrt(2.0 / fan)
        if k == "W0":
            w[:, :, 2:] = 0.0
        W[k] = bf16(w)
    W["w7"] = bf16(rng.standard_normal(16) * np.sqrt(1.0 / 16))
    return W


def _pad(x):
    return np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))


def conv(x, w):
    """3x3x3 zero-padded convolution, w [27, cout, cin]."""
    Z, Y, X, _ = x.shape
    xp = _pad(x)
    out = np.zeros((Z, Y, X, w.shape[1]))
    for t in range(27):
        dz, dy, dx = t // 9, (t // 3) % 3, t % 3
        out += xp[dz:dz + Z, dy:dy + Y, dx:dx + X, :] @ w[t].T
    return out


def conv_wgrad(x, g):
    """dW[t, co, ci] = sum_v g[v, co] x[v + off(t), ci]."""
    Z, Y, X, ci = x.shape
    xp = _pad(x)
    dw = np.zeros((27, g.shape[3], ci))
    gf = g.reshape(-1, g.shape[3])
    for t in range(27):
        dz, dy, dx = t // 9, (t // 3) % 3, t % 3
        dw[t] = gf.T @ xp[dz:dz + Z, dy:dy + Y, dx:dx + X, :].reshape(-1, ci)
    return dw


def conv_dgrad(g, w):
    """Gradient with respect to the convolution input: the convolution of g
    with the spatially flipped, channel-transposed kernel."""
    wt = w[::-1].transpose(0, 2, 1)
    return conv(g, wt)


def pool(x):
    Z, Y, X, C = x.shape
    return x.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(axis=(1, 3, 5))


def up(x):
    return x.repeat(2, axis=0).repeat(2, axis=1).repeat(2, axis=2)


def up_t(g):
    """Adjoint of up: sum over the 8 children."""
    Z, Y, X, C = g.shape
    return g.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(1, 3, 5))


def pool_t(g):
    """Adjoint of pool: each child gets its parent's gradient / 8."""
    return up(g) / 8.0


def make_input(r, logd):
    """x0 from a residual r and the normalised log-diagonal, both [Z, Y, X]."""
    nr = np.linalg.norm(r)
    x0 = np.zeros(r.shape + (16,))
    x0[..., 0] = r / nr if nr > 0 else 0.0
    x0[..., 1] = logd
    return x0, nr


def forward(x0, W, rounded=True):
    """Activations and the output y ([Z, Y, X]) of the network."""
    q = bf16 if rounded else (lambda a: a)
    relu = lambda a: np.maximum(a, 0.0)
    A = {"x0": q(x0)}
    A["e0"] = q(relu(conv(A["x0"], W["W0"])))
    A["p1"] = q(pool(A["e0"]))
    A["e1"] = q(relu(conv(A["p1"], W["W1"])))
    A["p2"] = q(pool(A["e1"]))
    A["e2"] = q(relu(conv(A["p2"], W["W2"])))
    A["p3"] = q(pool(A["e2"]))
    A["e3"] = q(relu(conv(A["p3"], W["W3"])))
    A["in4"] = np.concatenate([up(A["e3"]), A["e2"]], axis=3)
    A["d2"] = q(relu(conv(A["in4"], W["W4"])))
    A["in5"] = np.concatenate([up(A["d2"]), A["e1"]], axis=3)
    A["d1"] = q(relu(conv(A["in5"], W["W5"])))
    A["in6"] = np.concatenate([up(A["d1"]), A["e0"]], axis=3)
    A["d0"] = q(relu(conv(A["in6"], W["W6"])))
    A["y"] = A["d0"] @ W["w7"]
    return A


def loss(y, t):
    """Scale-free loss 1 - cos^2(y, t) and its gradient in y: the step length
    of the correction is chosen at apply time, so only the direction of the
    network output is trained."""
    a = float(np.sum(y * t))
    b = float(np.sum(y * y))
    c = float(np.sum(t * t))
    if b <= 0.0 or c <= 0.0:
        return 1.0, np.zeros_like(y)
    return 1.0 - a * a / (b * c), -2.0 * a / (b * c) * t + 2.0 * a * a / (b * b * c) * y


def backward(A, W, gy):
    """Gradients of all weights given dL/dy (float64, no rounding)."""
    G = {}
    G["w7"] = np.tensordot(A["d0"], gy, axes=([0, 1, 2], [0, 1, 2]))
    g = gy[..., None] * W["w7"] * (A["d0"] > 0)                 # d0 pre-activation
    G["W6"] = conv_wgrad(A["in6"], g)
    gi = conv_dgrad(g, W["W6"])
    g_d1 = up_t(gi[..., :16]) * (A["d1"] > 0)
    g_e0 = gi[..., 16:]
    G["W5"] = conv_wgrad(A["in5"], g_d1)
    gi = conv_dgrad(g_d1, W["W5"])
    g_d2 = up_t(gi[..., :32]) * (A["d2"] > 0)
    g_e1 = gi[..., 32:]
    G["W4"] = conv_wgrad(A["in4"], g_d2)
    gi = conv_dgrad(g_d2, W["W4"])
    g_e3 = up_t(gi[..., :64]) * (A["e3"] > 0)
    g_e2 = gi[..., 64:]
    G["W3"] = conv_wgrad(A["p3"], g_e3)
    g_e2 = (g_e2 + pool_t(conv_dgrad(g_e3, W["W3"]))) * (A["e2"] > 0)
    G["W2"] = conv_wgrad(A["p2"], g_e2)
    g_e1 = (g_e1 + pool_t(conv_dgrad(g_e2, W["W2"]))) * (A["e1"] > 0)
    G["W1"] = conv_wgrad(A["p1"], g_e1)
    g_e0 = (g_e0 + pool_t(conv_dgrad(g_e1, W["W1"]))) * (A["e0"] > 0)
    G["W0"] = conv_wgrad(A["x0"], g_e0)
    G["W0"][:, :, 2:] = 0.0
    return G
