"""Parity at the benchmark configurations, against the reference's own solves.

Fixtures (tests/golden/make_golden.py --cfg, made by running the reference
Bslib compiled from its sources):

* cfg1_heat32.npz -- the first benchmark configuration exactly: 3-D heat,
  7-point stencil, 32^3 (n = 32768), unit conductivity, RHS uniform[-1,1]
  from seed 0, CSVector::SolveSymm(CSMatrixR&) (Bslib/solvers.cpp:4615) with
  IC2 tau1 = tau2 = 1e-3 and PCG (Bslib/cg.cpp:31) to relative residual
  1e-10.
* cell12_lame_periodic.npz -- the homogenisation cell's shape (periodic Q1
  Lame, inclusions at 30 %, contrast 100, six unit macro-strain load cases)
  on 12^3 nodes, each load case solved by CSVector::SolveSymm(CSMatrixRS&)
  (Bslib/solvers.cpp:4452): block IC2 + PCG to relative residual 1e-8.

CPU tests pin the generators (hashes) and the oracle to the fixtures; GPU
tests state each GPU result's relative error against the reference's
solution.  Tolerances:

* cfg1, FP64 factor with exact solves (the reference's algorithm): the GPU
  IC2 factor equals the oracle's bit for bit, the iteration count is the
  reference's +-1 and ||x - x_ref|| / ||x_ref|| <= 1e-8;
* cfg1, FP32 factor with Jacobi sweeps inside the FP64 loop: true residual
  <= 1e-10 and ||x - x_ref|| / ||x_ref|| <= 1e-7 (the stopping test bounds
  the error only through the condition number, ~1e3 here);
* cell: each load case's relative error to the reference's solution is at
  most 10 x the reference's own error against a sparse direct solve (which
  the fixture records, 1e-8 .. 6e-8) -- both solutions stop at relative
  residual 1e-8, so neither is closer to the exact one than that.
"""
import hashlib
import os

import numpy as np
import pytest

import problems as P

HERE = os.path.join(os.path.dirname(__file__), "golden")
CFG1 = os.path.join(HERE, "cfg1_heat32.npz")
CELL = os.path.join(HERE, "cell12_lame_periodic.npz")
TAU = 1e-3


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def relerr(x, y):
    return float(np.linalg.norm(x - y) / np.linalg.norm(y))


@pytest.fixture(scope="module")
def cfg1():
    g = np.load(CFG1)
    s = P.config(1)
    return g, s, s.upper()


@pytest.fixture(scope="module")
def cell():
    g = np.load(CELL)
    c = P.lame_periodic(12, 0.3, 1.0, 2.0, 0.3, 100.0, 2)
    return g, c


# ---------------------------------------------------------------- CPU pins
def test_cfg1_generator_is_the_fixture_system(cfg1):
    g, s, u = cfg1
    assert s.n == 32768 and s.nnz == 223232 and u.nnz == 128000
    assert sha(s.ia, s.ja, s.a, s.rhs[0]) == str(g["system_sha"])
    assert sha(u.ia, u.ja, u.a) == str(g["upper_sha"])


def test_cfg1_oracle_factor_and_solve_match_reference(oracle, cfg1):
    g, s, u = cfg1
    iu, ju, uu, _, st = oracle.fact(0, u.ia, u.ja, u.a, tau1=TAU, tau2=TAU, theta=0.1)
    assert len(ju) == int(g["factor_nnz"])
    assert sha(iu, ju) == str(g["factor_pattern_sha"])
    assert abs(st[0] - float(g["density"])) < 1e-12
    probe = np.random.default_rng(101).standard_normal(s.n)
    idx = g["probe_idx"]
    for got, want in ((oracle.solve_l(iu, ju, uu, probe)[idx], g["probe_solve_l"]),
                      (oracle.solve_u(iu, ju, uu, probe)[idx], g["probe_solve_u"])):
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    xo, it, _ = oracle.pcg(u.ia, u.ja, u.a, iu, ju, uu, s.rhs[0], ittype=0, eps=1e-10, niter=3000)
    assert abs(it - int(g["iters"])) <= 1
    assert relerr(xo, g["x_ref"]) <= 1e-10


def test_cell_generator_is_the_fixture_system(cell):
    g, c = cell
    assert c.n == 1728 and c.bs == 3 and c.rhs.shape == (6, 5184)
    assert sha(c.ia, c.ja, c.a, c.rhs) == str(g["system_sha"])
    assert np.all(g["ref_err_vs_direct"] < 1e-7)


# ---------------------------------------------------------------- GPU parity
@pytest.mark.gpu
def test_cfg1_fp64_ic2_pcg_matches_reference(ctx, oracle, cfg1):
    """FP64 IC2 + PCG with exact solves at cfg1: the reference's algorithm."""
    import bsg
    import torch
    g, s, u = cfg1
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=TAU, tau2=TAU, theta=0.1, memory=20.0, ittype=0, eps=1e-10,
                          niter=3000, precision=0, trisolve=0)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    giu, gju, _, gu = f.export()
    iu, ju, uu, _, _ = oracle.fact(0, u.ia, u.ja, u.a, tau1=TAU, tau2=TAU, theta=0.1)
    assert np.array_equal(giu, iu) and np.array_equal(gju, ju), "IC2 pattern differs from the oracle"
    assert np.array_equal(gu, uu), "IC2 values differ from the oracle"
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    bsg.pcg(ctx, m, f, torch.as_tensor(s.rhs[0], device="cuda"), x, p)
    err = relerr(x.cpu().numpy(), g["x_ref"])
    print(f"cfg1 FP64: iterations {p.nitperf} (reference {int(g['iters'])}), rel. error vs reference {err:.2e}, "
          f"true residual {p.resfin:.2e}")
    assert abs(p.nitperf - int(g["iters"])) <= 1
    assert err <= 1e-8
    assert p.resfin <= 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("krylov", [0, 2])
def test_cfg1_mixed_precision_matches_reference(ctx, cfg1, krylov):
    """FP32 IC2 factor, Jacobi(6) sweeps, FP64 PCG / FGMRES(30) with the
    true-residual check: the mixed arms of the benchmark at cfg1."""
    import bsg
    import torch
    g, s, u = cfg1
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=TAU, tau2=TAU, theta=0.1, memory=20.0, ittype=0, eps=1e-10,
                          niter=3000, precision=1, trisolve=1, nsweeps=6, krylov=krylov, restart=30, sttype=1,
                          true_residual=1)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    b = torch.as_tensor(s.rhs[0], device="cuda")
    (bsg.pcg if krylov == 0 else bsg.gmres)(ctx, m, f, b, x, p)
    err = relerr(x.cpu().numpy(), g["x_ref"])
    print(f"cfg1 mixed krylov={krylov}: iterations {p.nitperf}, rel. error vs reference {err:.2e}, "
          f"true residual {p.resfin:.2e}")
    assert p.resfin <= 1e-10
    assert err <= 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("precision,trisolve", [(0, 0), (1, 1)])
def test_cell_load_cases_match_reference(ctx, cell, precision, trisolve):
    """The six load cases of the periodic cell as one batched block-IC2 PCG
    call, each against the reference's own SolveSymm(CSMatrixRS&) solution."""
    import bsg
    import torch
    g, c = cell
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=TAU, tau2=TAU, theta=0.1, memory=20.0, ittype=0, eps=1e-8,
                          niter=3000, precision=precision, trisolve=trisolve, nsweeps=6)
    m = bsg.Matrix.from_system(ctx, c, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    B = torch.as_tensor(c.rhs, device="cuda").contiguous()
    X = torch.zeros_like(B)
    its, res, _ = bsg.pcg_batch(ctx, m, f, B, X, p)
    X = X.cpu().numpy()
    for k in range(6):
        err = relerr(X[k], g["X_ref"][k])
        bound = max(10 * float(g["ref_err_vs_direct"][k]), 1e-10)
        print(f"cell load case {k}: iterations {its[k]} (reference {int(g['iters'][k])}), rel. error vs "
              f"reference {err:.2e} (bound {bound:.1e}), true residual {res[k]:.2e}")
        assert res[k] <= 1e-8
        assert err <= bound, (k, err, bound)
