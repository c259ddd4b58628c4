"""The GPU drop-ins for Bslib's AbstractSymmSolver / AbstractSolver
(libbsg_bslib.so, include/bsg_bslib.h) against the reference's own
AbstractSymmSolver / AbstractSolver (Bslib/solvers.cpp:5383, :5591), both
driven by the same generator object and the same seven callbacks
(oracle/ref/abstract_gen.cpp: block rows served in a shuffled column order,
pattern arrays allocated with new[] for the solver to delete[]).

Checks, per case:
* the callbacks are called as the reference calls them (once each for the
  sizes and the pattern, once per block row for the rows, right-hand side,
  initial guess and stored solution);
* the solution the GPU stores through the callback agrees with the one the
  reference stores: ||x_gpu - x_ref|| <= 1e-8 ||x_ref|| (both runs stop at
  relative residual 1e-10; the systems are small and well conditioned), and
  the GPU's FP64 true residual meets the tolerance;
* nitperf / resfin / density are filled.

Cases: 3x3 Lame blocks, symmetric (block IC2 + PCG) with the relative and
with the reference's default max-norm stop rule; variable block sizes
(1, 2, 3 repeating) cut from a heat matrix; a nonsymmetric Lame variant
through AbstractSolver (block ILU2 on the GPU, ILU2 + Lanczos in the
reference) and through AbstractParSolver on one process; a nonzero initial
guess; a matrix that is not positive definite.  Last, the reference's own
callback Krylov loops (CG and BlockGMRES on a one-processor CTree) run with
the GPU's SpMV and preconditioner behind their CMVM / CSOLVELU callbacks, the
role CParMvmA / CParSolveLU play in the reference's parallel driver.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import problems as P

pytestmark = pytest.mark.gpu


def block_csr_from_point(A, sizes, upper):
    """Block CSR (blocks column-major) of point matrix A cut into blocks of the
    given sizes; upper keeps block columns >= the block row."""
    A = sp.csr_matrix(A)
    sprnd = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    nb = len(sizes)
    owner = np.repeat(np.arange(nb), sizes)
    ia, ja, vals = [0], [], []
    for I in range(nb):
        r0, r1 = sprnd[I], sprnd[I + 1]
        cols = np.unique(owner[A[r0:r1].indices])
        if upper:
            cols = cols[cols >= I]
        for J in cols:
            blk = A[r0:r1, sprnd[J]:sprnd[J + 1]].toarray()
            ja.append(J)
            vals.append(blk.flatten(order="F"))
        ia.append(len(ja))
    return sprnd, np.array(ia, np.int32), np.array(ja, np.int32), np.concatenate(vals)


def skewed(s, skew=0.3):
    a = s.a.reshape(-1, s.bs, s.bs).copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.ia))
    off = s.ja != rows
    a[off] *= (1.0 + skew * np.sign(s.ja[off] - rows[off]))[:, None, None]
    return a.reshape(-1)


def run_both(reflib, symm, sprnd, ia, ja, a, b, x0, ittype=0, sttype=1, eps=1e-10, gpu_extra=None):
    import bsg
    n = int(sprnd[-1])
    nsup = len(sprnd) - 1
    fns = reflib.gen_fns()
    hr = reflib.gen_create(sprnd, ia, ja, a, b, x0, seed=11)
    info = reflib.abstract(symm, hr, ittype=ittype, sttype=sttype, eps=eps)
    x_ref = reflib.gen_solution(hr, n)
    reflib.gen_free(hr)
    hg = reflib.gen_create(sprnd, ia, ja, a, b, x0, seed=12)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, ittype=ittype,
                          sttype=sttype, eps=eps, niter=3000, **(gpu_extra or {}))
    rc = bsg.abstract_solve(symm, hg, fns, p)
    assert rc == bsg.OK, (rc, bsg.bslib().bsg_bslib_last_error())
    x_gpu = reflib.gen_solution(hg, n)
    calls = reflib.gen_calls(hg)
    reflib.gen_free(hg)
    assert list(calls) == [1, 1, 1, nsup, nsup, nsup, nsup], calls
    return x_ref, x_gpu, info, p


def relerr(x, y):
    return float(np.linalg.norm(x - y) / np.linalg.norm(y))


def test_symm_lame_blocks(reflib):
    s = P.lame3d(6, 0.3, 1.0, 5)
    u = s.upper()
    sprnd = np.arange(s.n + 1, dtype=np.int32) * 3
    b = s.rhs[0]
    x_ref, x_gpu, info, p = run_both(reflib, True, sprnd, u.ia, u.ja, u.a, b, np.zeros_like(b))
    A = s.to_scipy()
    err = relerr(x_gpu, x_ref)
    print(f"AbstractSymmSolver 3x3: GPU {p.nitperf} it, reference {info['iters']} it, rel. error {err:.2e}")
    assert err <= 1e-8
    assert np.linalg.norm(b - A @ x_gpu) <= 1e-9 * np.linalg.norm(b)
    assert p.nitperf > 0 and p.density > 1.0 and p.resfin <= 1e-9


def test_symm_default_max_norm_stop(reflib):
    """ittype 2, the reference's default: stop when max |r_i| <= eps."""
    s = P.lame3d(6, 0.3, 1.0, 6)
    u = s.upper()
    sprnd = np.arange(s.n + 1, dtype=np.int32) * 3
    b = s.rhs[0]
    x_ref, x_gpu, info, p = run_both(reflib, True, sprnd, u.ia, u.ja, u.a, b, np.zeros_like(b), ittype=2, eps=1e-11)
    A = s.to_scipy()
    r = b - A @ x_gpu
    print(f"ittype 2: GPU {p.nitperf} it, reference {info['iters']} it, max|r| {np.abs(r).max():.2e}")
    assert np.abs(r).max() <= 1e-11 * 1.001
    assert relerr(x_gpu, x_ref) <= 1e-8


def test_symm_variable_blocks(reflib):
    s = P.heat3d(8, 8, 8, sigma=1.0, seed=13)
    A = s.to_scipy()
    sizes = []
    left = s.n
    k = 0
    while left > 0:
        sz = min([1, 2, 3][k % 3], left)
        sizes.append(sz)
        left -= sz
        k += 1
    # upper block triangle, full (symmetric) diagonal blocks, as CSMatrixRS stores it
    sprnd, ia, ja, a = block_csr_from_point(A, sizes, upper=True)
    b = s.rhs[0]
    x_ref, x_gpu, info, p = run_both(reflib, True, sprnd, ia, ja, a, b, np.zeros_like(b))
    err = relerr(x_gpu, x_ref)
    print(f"variable blocks: GPU {p.nitperf} it, reference {info['iters']} it, rel. error {err:.2e}")
    assert err <= 1e-8


def test_nonsymmetric_lame_abstract_solver(reflib):
    s = P.lame3d(5, 0.3, 1.0, 7)
    a = skewed(s)
    sprnd = np.arange(s.n + 1, dtype=np.int32) * 3
    b = s.rhs[0]
    x_ref, x_gpu, info, p = run_both(reflib, False, sprnd, s.ia, s.ja, a, b, np.zeros_like(b), ittype=1, sttype=1)
    A = sp.bsr_matrix((a.reshape(-1, 3, 3).transpose(0, 2, 1), s.ja, s.ia), shape=(s.n * 3, s.n * 3)).tocsr()
    err = relerr(x_gpu, x_ref)
    print(f"AbstractSolver: GPU {p.nitperf} it, reference {info['iters']} it, rel. error {err:.2e}")
    assert np.linalg.norm(b - A @ x_gpu) <= 1e-9 * np.linalg.norm(b)
    assert err <= 1e-8


def test_initial_guess_is_used(reflib):
    s = P.lame3d(5, 0.3, 1.0, 8)
    u = s.upper()
    sprnd = np.arange(s.n + 1, dtype=np.int32) * 3
    b = s.rhs[0]
    x0 = np.random.default_rng(3).standard_normal(len(b))
    x_ref, x_gpu, info, p = run_both(reflib, True, sprnd, u.ia, u.ja, u.a, b, x0)
    assert relerr(x_gpu, x_ref) <= 1e-8


def test_not_positive_definite_raises(reflib):
    import bsg
    s = P.heat3d(4, 4, 4, sigma=0.0, seed=1)
    u = s.upper()
    a = u.a.copy()
    a[u.ia[10]] = -1.0  # a negative diagonal entry
    sprnd = np.arange(s.n + 1, dtype=np.int32)
    hg = reflib.gen_create(sprnd, u.ia, u.ja, a, s.rhs[0], np.zeros(s.n), seed=2)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, ittype=0, eps=1e-10)
    rc = bsg.abstract_solve(True, hg, reflib.gen_fns(), p)
    reflib.gen_free(hg)
    assert rc != bsg.OK
    assert bsg.bslib().bsg_bslib_last_error()


def test_abstract_par_solver_single_rank(reflib):
    """AbstractParSolver on one process: the GPU drop-in against the
    reference's AbstractSolver on the same generator (the reference's
    AbstractParSolver partitions with METIS even for one rank, which this
    build does not have)."""
    import bsg
    s = P.lame3d(5, 0.3, 1.0, 9)
    a = skewed(s)
    sprnd = np.arange(s.n + 1, dtype=np.int32) * 3
    b = s.rhs[0]
    n = s.n * 3
    hr = reflib.gen_create(sprnd, s.ia, s.ja, a, b, np.zeros(n), seed=21)
    reflib.abstract(False, hr, ittype=1, sttype=1, eps=1e-10)
    x_ref = reflib.gen_solution(hr, n)
    reflib.gen_free(hr)
    hg = reflib.gen_create(sprnd, s.ia, s.ja, a, b, np.zeros(n), seed=22)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, ittype=1, sttype=1,
                          eps=1e-10, niter=3000)
    rc = bsg.abstract_solve(2, hg, reflib.gen_fns(), p)
    assert rc == bsg.OK, bsg.bslib().bsg_bslib_last_error()
    x_gpu = reflib.gen_solution(hg, n)
    assert list(reflib.gen_calls(hg)) == [1, 1, 1, s.n, s.n, s.n, s.n]
    reflib.gen_free(hg)
    assert relerr(x_gpu, x_ref) <= 1e-8


def test_reference_cg_runs_on_gpu_operators(reflib):
    """The reference's own callback CG loop (Bslib/cg.cpp:355, one-rank CTree)
    with the GPU's SpMV and IC2 preconditioner behind CMVM / CSOLVELU, against
    the reference's SolveSymm with its own operators: the same iteration
    count +-1 and the same solution to 1e-8."""
    import bsg
    s = P.heat3d(12, 10, 8, sigma=1.0, seed=41)
    u = s.upper()
    b = s.rhs[0]
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0)
    op = bsg.GpuOperator(s.n, u.ia, u.ja, u.a, True, p)
    try:
        x, info = reflib.cg_tree(s.n, b, np.zeros(s.n), op, sttype=1, eps=1e-10, niter=1000)
    finally:
        op.free()
    xr, ir = reflib.solve_symm(u.ia, u.ja, u.a, b, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=-1.0, ittype=0, eps=1e-10)
    err = relerr(x, xr)
    print(f"reference Cg on GPU operators: {info['iters']} it (reference operators {ir['iters']}), rel. error {err:.2e}")
    assert abs(info["iters"] - ir["iters"]) <= 2
    assert err <= 1e-8


def test_reference_block_gmres_runs_on_gpu_operators(reflib):
    """The reference's callback BlockGMRES (Bslib/gmres.cpp:337, one-rank
    CTree) with the GPU's SpMV and ILU2 preconditioner, against the
    reference's Solver (ILU2 + Lanczos) with its own operators."""
    import bsg
    s = P.heat3d(10, 9, 8, sigma=1.0, seed=43)
    a = s.a.copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.ia))
    off = s.ja != rows
    a[off] *= 1.0 + 0.3 * np.sign(s.ja[off] - rows[off])
    b = s.rhs[0]
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0)
    op = bsg.GpuOperator(s.n, s.ia, s.ja, a, False, p)
    try:
        x, info = reflib.gmres_tree(s.n, b, np.zeros(s.n), op, sttype=1, eps=1e-10, niter=200)
    finally:
        op.free()
    xr, ir = reflib.solver(s.ia, s.ja, a, b, tau1=1e-3, tau2=1e-3, sttype=1, eps=1e-10)
    A = sp.csr_matrix((a, s.ja, s.ia), shape=(s.n, s.n))
    err = relerr(x, xr)
    print(f"reference BlockGMRES on GPU operators: {info['iters']} it, rel. error {err:.2e}")
    assert np.linalg.norm(b - A @ x) <= 1e-9 * np.linalg.norm(b)
    assert err <= 1e-8


@pytest.mark.parametrize("ittype", [2, 3, 4])
def test_abstract_solver_block_lanczos(reflib, ittype):
    """AbstractSolver with ittype 2 / 3 / 4 (the reference's default is 2):
    the reference's block ILU2 + block Lanczos variant against the GPU's block
    Lanczos on the point form of the same system."""
    s = P.lame3d(5, 0.3, 1.0, 10)
    a = skewed(s)
    sprnd = np.arange(s.n + 1, dtype=np.int32) * 3
    b = s.rhs[0]
    x_ref, x_gpu, info, p = run_both(reflib, False, sprnd, s.ia, s.ja, a, b, np.zeros_like(b), ittype=ittype,
                                     eps=1e-10)
    A = sp.bsr_matrix((a.reshape(-1, 3, 3).transpose(0, 2, 1), s.ja, s.ia), shape=(s.n * 3, s.n * 3)).tocsr()
    err = relerr(x_gpu, x_ref)
    print(f"AbstractSolver ittype {ittype}: GPU {p.nitperf} steps, rel. error {err:.2e}")
    assert np.linalg.norm(b - A @ x_gpu) <= 1e-9 * np.linalg.norm(b)
    assert err <= 1e-7
