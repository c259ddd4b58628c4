"""Triangular sweeps of several vectors at once (bsg_solve_multi_dev, the
batched PCG's preconditioner): the factor is read once per group of up to 8
vectors, and every vector must come out bit for bit as its own single-vector
solve -- point factors (FP64, FP32 tiled and untiled), factors with rows too
long for a slice, and 3x3 block factors (FP64 and FP32 values)."""
import numpy as np
import pytest

import problems as P
from test_gpu_sell_long import _bordered

pytestmark = pytest.mark.gpu


def _factor(ctx, case, precision):
    import bsg
    if case == "heat":
        s = P.heat3d(20, 18, 16, sigma=1.0, seed=12)
    elif case == "bordered":
        s = _bordered(17, 2, 40, 3)
    else:
        s = P.lame_periodic(8, rmin=1.5, rmax=2.5, seed=42)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, precision=precision)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    if case == "periodic_block" and precision == 1:
        f.to_fp32()
    return s.n * s.bs, m, f


@pytest.mark.parametrize("case", ["heat", "bordered", "periodic_block"])
@pytest.mark.parametrize("precision", [0, 1])
def test_multi_vector_sweeps_equal_single(ctx, case, precision):
    import torch
    n, m, f = _factor(ctx, case, precision)
    rng = np.random.default_rng(17)
    X = torch.as_tensor(rng.standard_normal((11, n)), device="cuda")
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    # one group of <= 4 or <= 8 vectors, two groups; even counts keep the
    # block iterates interleaved between passes
    for nr in (3, 4, 6, 10, 11):
        Y = torch.full((nr, n), np.nan, dtype=torch.float64, device="cuda")
        for lower in (True, False):
            for sw in (2, 3, 6):
                f.solve_multi(lower, X[:nr].contiguous(), Y, mode=1, nsweeps=sw)
                for q in range(nr):
                    (f.solve_l if lower else f.solve_u)(X[q].contiguous(), y, mode=1, nsweeps=sw)
                    assert torch.equal(Y[q], y), (nr, lower, sw, q)
    # exact solves go one vector at a time
    Y = torch.empty((3, n), dtype=torch.float64, device="cuda")
    f.solve_multi(True, X[:3].contiguous(), Y, mode=0)
    f.solve_l(X[1].contiguous(), y, mode=0)
    assert torch.equal(Y[1], y)
