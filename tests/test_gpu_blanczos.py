"""Block Lanczos on the GPU (bsg_block_lanczos_dev) against the reference's
CSVector::BlockLanczosCentral / Right / Left (Bslib/lanczos.cpp:2467 / :932 /
:1719), the iterations CSVector::Solver(CSMatrixRS&) runs for ittype 2 / 3 /
4, on one and on three right-hand sides at once.

The reference runs them with its block ILU2 of 1 x 1 blocks, the GPU with the
point ILU2 (the same preconditioner up to the scaling's rounding); both stop
when every right-hand side's true residual has fallen below eps = 1e-8 of its
start.  Checks: the GPU's true relative residual meets that test for every
right-hand side, and each GPU solution is as close to a sparse direct
solution as the reference's is (10x the reference's own error, plus 1e-9),
hence within 1e-7 of the reference's.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

import problems as P

pytestmark = pytest.mark.gpu
EPS = 1e-8


@pytest.fixture(scope="module")
def system():
    s = P.heat3d(12, 10, 9, sigma=1.0, seed=47)
    a = s.a.copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.ia))
    off = s.ja != rows
    a[off] *= 1.0 + 0.3 * np.sign(s.ja[off] - rows[off])
    A = sp.csr_matrix((a, s.ja, s.ia), shape=(s.n, s.n))
    B = np.random.default_rng(5).standard_normal((3, s.n))
    lu = spla.splu(A.tocsc())
    Xd = np.array([lu.solve(B[j]) for j in range(3)])
    return s, a, A, B, Xd


@pytest.mark.parametrize("ittype", [2, 3, 4])
@pytest.mark.parametrize("nrhs", [1, 3])
def test_block_lanczos_matches_reference(ctx, reflib, system, ittype, nrhs):
    import bsg
    s, a, A, B, Xd = system
    B, Xd = B[:nrhs], Xd[:nrhs]
    Xr = reflib.block_lanczos(s.ia, s.ja, a, 1, ittype, B, eps=EPS, niter=2000, ichk=1)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, eps=EPS, niter=2000,
                          ichk=1, ittype=ittype)
    m = bsg.Matrix(ctx, s.n, s.ia, s.ja, a)
    f = bsg.Factor(ctx, m, "ilu2", p)
    Bt = torch.as_tensor(B, device="cuda").contiguous()
    Xt = torch.zeros_like(Bt)
    res = bsg.block_lanczos(ctx, m, f, ittype, Bt, Xt, p)
    X = Xt.cpu().numpy()
    for j in range(nrhs):
        r = np.linalg.norm(B[j] - A @ X[j]) / np.linalg.norm(B[j])
        e_gpu = np.linalg.norm(X[j] - Xd[j]) / np.linalg.norm(Xd[j])
        e_ref = np.linalg.norm(Xr[j] - Xd[j]) / np.linalg.norm(Xd[j])
        e_gr = np.linalg.norm(X[j] - Xr[j]) / np.linalg.norm(Xr[j])
        print(f"ittype {ittype} rhs {j}/{nrhs}: {p.nitperf} steps, residual {r:.2e}, error vs direct GPU {e_gpu:.2e} "
              f"reference {e_ref:.2e}, GPU vs reference {e_gr:.2e}")
        assert abs(r - res[j]) <= 1e-6 * max(r, 1e-300) + 1e-15
        assert r < EPS * 1.0001
        assert e_gpu <= 10 * e_ref + 1e-9
        assert e_gr <= 1e-7
