"""IC(0) on the GPU (fcttyp = 1, CSMatrixR::Ich, Bslib/ich2r.cpp:1821):
the factor equals the oracle's (and so the reference's, tests/
test_oracle_pin.py) bit for bit, at the small golden system and at the
first benchmark configuration; PCG with it takes the reference's iteration
count +-1 and agrees with the reference's CG on its own IC(0) factor to 1e-8.

The reference's SolveSymm(CSMatrixR&) cannot itself run IC(0) (it hands CG
its empty block factor, Bslib/solvers.cpp:4692-4726), so the comparison is
against its CSVector::Cg with the IC(0) factor, which is what SolveSymm
means to run.
"""
import os

import numpy as np
import pytest
import torch

import problems as P

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "heat_8x8x6.npz")


def factor(ctx, s):
    import bsg
    p = bsg.default_param(ordtype=0, fcttyp=1, ittype=0, eps=1e-10, niter=2000)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    return p, m, bsg.Factor(ctx, m, "ich2", p)


def test_ic0_golden(ctx):
    import bsg
    g = np.load(GOLD)
    s = P.System(int(g["n"]), 1, g["ia"], g["ja"], g["a"], g["b"][None, :], np.array([0, int(g["n"])]), {})
    p, m, f = factor(ctx, s)
    iu, ju, _, u = f.export()
    assert np.array_equal(iu, g["ic0_iu"]) and np.array_equal(ju, g["ic0_ju"])
    assert np.array_equal(u, g["ic0_u"]), np.abs(u - g["ic0_u"]).max()
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    bsg.pcg(ctx, m, f, torch.as_tensor(g["b"], device="cuda"), x, p)
    assert abs(p.nitperf - int(g["symm_ic0_iters"])) <= 1
    xr = g["symm_ic0_x"]
    assert np.linalg.norm(x.cpu().numpy() - xr) <= 1e-8 * np.linalg.norm(xr)


def test_ic0_cfg1_matches_oracle_and_reference(ctx, oracle, reflib):
    import bsg
    s = P.config(1)
    u = s.upper()
    p, m, f = factor(ctx, s)
    iu, ju, _, gu = f.export()
    oiu, oju, ou = oracle.ich0(u.ia, u.ja, u.a)
    assert np.array_equal(iu, oiu) and np.array_equal(ju, oju) and np.array_equal(gu, ou)
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    bsg.pcg(ctx, m, f, torch.as_tensor(s.rhs[0], device="cuda"), x, p)
    xr, info = reflib.cg(u.ia, u.ja, u.a, oiu, oju, ou, s.rhs[0], ittype=0, eps=1e-10, niter=2000)
    err = np.linalg.norm(x.cpu().numpy() - xr) / np.linalg.norm(xr)
    print(f"IC(0) PCG at cfg1: {p.nitperf} iterations (reference {info['iters']}), rel. error {err:.2e}")
    assert abs(p.nitperf - info["iters"]) <= 1
    assert err <= 1e-8


def test_ic0_refuses_block_and_nonsymmetric(ctx):
    import bsg
    s = P.heat3d(4, 4, 4, sigma=1.0, seed=2)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=False)
    with pytest.raises(bsg.BsgError) as e:
        bsg.Factor(ctx, m, "ich2", bsg.default_param(ordtype=0, fcttyp=1))
    assert e.value.code == bsg.ERR_UNSUPPORTED
