"""GPU parity of the solver path against the CPU oracle (oracle/bsl_oracle.c).

Inputs are the seeded generators at sizes the oracle finishes in seconds.
Tolerances: integer/pattern work is compared exactly; the factorisation is
compared entry by entry (same arithmetic order and fma, so bit-exact unless a
product lands within rounding of a threshold); products and solves that sum
in a different order than the CPU loop are held to 1e-13 relative; Krylov
solutions to their stopping tolerance.
"""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def _t(x):
    import torch
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device="cuda")


def _nonsymmetric(s, skew=0.3):
    """Convection-like perturbation of a heat matrix: off-diagonal (i,j) scaled
    by 1 + skew*sign(j - i); stays diagonally dominant, loses symmetry."""
    a = s.a.copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.ia))
    off = s.ja != rows
    a[off] *= 1.0 + skew * np.sign(s.ja[off] - rows[off])
    return P.System(s.n, s.bs, s.ia, s.ja, a, s.rhs, s.parts)


@pytest.fixture(scope="module")
def heat():
    return P.heat3d(14, 12, 10, sigma=1.0, seed=11)


def test_spmv_csr_full_and_symmetric(ctx, oracle, heat):
    import bsg
    import torch
    s = heat
    u = s.upper()
    x = np.random.default_rng(1).standard_normal(s.n)
    ref = oracle.mvm(s.ia, s.ja, s.a, x)
    ref_s = oracle.mvm(u.ia, u.ja, u.a, x, symm=True)
    for sysm, symm, r in ((s, False, ref), (s, True, ref_s)):
        m = bsg.Matrix.from_system(ctx, sysm, symm_upper=symm)
        y = torch.empty(s.n, dtype=torch.float64, device="cuda")
        m.mvm(_t(x), y)
        got = y.cpu().numpy()
        assert np.abs(got - r).max() <= 1e-13 * np.abs(r).max()
        # host-buffer entry point
        assert np.abs(m.mvm_host(x) - r).max() <= 1e-13 * np.abs(r).max()


def test_spmm_multi_rhs(ctx, oracle, heat):
    import bsg
    import torch
    s = heat
    X = np.random.default_rng(2).standard_normal((5, s.n))
    m = bsg.Matrix.from_system(ctx, s)
    Y = torch.empty((5, s.n), dtype=torch.float64, device="cuda")
    m.mvm_multi(_t(X), Y)
    for r in range(5):
        ref = oracle.mvm(s.ia, s.ja, s.a, X[r])
        assert np.abs(Y[r].cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()


def test_spmv_bsr3(ctx, oracle):
    import bsg
    import torch
    s = P.lame3d(6, 0.3, 1.0, 5)
    x = np.random.default_rng(3).standard_normal(s.n * 3)
    ref = oracle.bsr_mvm(s.ia, s.ja, s.a, x, 3)
    m = bsg.Matrix.from_system(ctx, s)
    y = torch.empty(s.n * 3, dtype=torch.float64, device="cuda")
    m.mvm(_t(x), y)
    assert np.abs(y.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    # symmetric (upper block triangle) input
    u = s.upper()
    ms = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    ms.mvm(_t(x), y)
    assert np.abs(y.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    del u
    # several vectors in one pass over the blocks (groups of 1, 2, 4, 8, and
    # two groups): each vector bit for bit its own product
    X = np.random.default_rng(4).standard_normal((11, s.n * 3))
    for nr in (2, 3, 6, 11):
        Y = torch.full((nr, s.n * 3), np.nan, dtype=torch.float64, device="cuda")
        m.mvm_multi(_t(X[:nr]), Y)
        for q in range(nr):
            m.mvm(_t(X[q]), y)
            assert torch.equal(Y[q], y), (nr, q)
            r = oracle.bsr_mvm(s.ia, s.ja, s.a, X[q], 3)
            assert np.abs(y.cpu().numpy() - r).max() <= 1e-13 * np.abs(r).max()


def _factor_match(gpu, ora):
    giu, gju, gl, gu = gpu
    oiu, oju, ol, ou = ora[:4]
    assert np.array_equal(giu, oiu), "row pointers differ"
    assert np.array_equal(gju, oju), "column pattern differs"
    # same operations in the same order (fma, fixed-point compensation sums):
    # the factor must agree bit for bit
    assert np.array_equal(gl, ol), f"L values differ, max {np.abs(gl - ol).max():.3e}"
    assert np.array_equal(gu, ou), f"U values differ, max {np.abs(gu - ou).max():.3e}"


@pytest.mark.parametrize("tau1,tau2", [(1e-3, 1e-3), (1e-2, 1e-4)])
def test_ich2_matches_oracle(ctx, oracle, heat, tau1, tau2):
    import bsg
    u = heat.upper()
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=tau1, tau2=tau2, theta=0.1, memory=20.0)
    m = bsg.Matrix.from_system(ctx, heat, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    ora = oracle.fact(0, u.ia, u.ja, u.a, tau1=tau1, tau2=tau2, theta=0.1)
    _factor_match(f.export(), ora)
    assert abs(p.density - ora[4][0]) < 1e-12 and abs(p.density2 - ora[4][1]) < 1e-12


@pytest.mark.parametrize("tau1,tau2", [(1e-3, 1e-3), (1e-2, 1e-4)])
def test_ilu2_matches_oracle(ctx, oracle, heat, tau1, tau2):
    import bsg
    s = _nonsymmetric(heat)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=tau1, tau2=tau2, theta=0.1, memory=20.0)
    m = bsg.Matrix.from_system(ctx, s)
    f = bsg.Factor(ctx, m, "ilu2", p)
    sia, sja, al, au = oracle.combine_lu(s.ia, s.ja, s.a)
    ora = oracle.fact(1, sia, sja, al, au, tau1=tau1, tau2=tau2, theta=0.1)
    _factor_match(f.export(), ora)


@pytest.mark.parametrize("case,kind", [("lame", "ilu2"), ("lame", "ich2"), ("periodic", "ich2")])
def test_big_rows_match_oracle(ctx, oracle, case, kind):
    """Point-expanded elasticity rows have 300-1400 contributors, beyond the
    shared-memory workspace; they are retried in the global one and must
    still agree bit for bit."""
    import bsg
    if case == "lame":
        s = P.lame3d(10, 0.3, 1.0, 1).to_point()
    else:
        s = P.lame_periodic(8, 0.3, 1.5, 2.5, 0.3, 100.0, 2).to_point()
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0)
    if kind == "ich2":
        u = s.upper()
        m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
        f = bsg.Factor(ctx, m, "ich2", p)
        ora = oracle.fact(0, u.ia, u.ja, u.a, tau1=1e-3, tau2=1e-3, theta=0.1)
    else:
        m = bsg.Matrix.from_system(ctx, s)
        f = bsg.Factor(ctx, m, "ilu2", p)
        sia, sja, al, au = oracle.combine_lu(s.ia, s.ja, s.a)
        ora = oracle.fact(1, sia, sja, al, au, tau1=1e-3, tau2=1e-3, theta=0.1)
    assert bsg.fact_stats()["big_rows"] > 0
    _factor_match(f.export(), ora)


@pytest.mark.parametrize("kind", ["ilu2", "ich2"])
def test_block_matrix_factors_point_expansion(ctx, oracle, kind):
    """With blockfct = 0 a 3x3 block matrix is factored through its point
    expansion: the same factor as the point CSR copy of the same operator, bit
    for bit; the Krylov solve then runs with the block SpMV and the point
    factor.  (IC2 of a block matrix always takes this path.)"""
    import bsg
    import torch
    s = P.lame3d(6, 0.3, 1.0, 3)
    pt = s.to_point()
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, eps=1e-9,
                          ittype=0, sttype=1, restart=40, krylov=1, blockfct=0)
    if kind == "ich2":
        m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
        u = pt.upper()
        ora = oracle.fact(0, u.ia, u.ja, u.a, tau1=1e-3, tau2=1e-3, theta=0.1)
    else:
        m = bsg.Matrix.from_system(ctx, s)
        sia, sja, al, au = oracle.combine_lu(pt.ia, pt.ja, pt.a)
        ora = oracle.fact(1, sia, sja, al, au, tau1=1e-3, tau2=1e-3, theta=0.1)
    assert m.info()[:2] == (s.n, 3)
    f = bsg.Factor(ctx, m, kind, p)
    _factor_match(f.export(), ora)
    b = s.rhs[0]
    x = torch.zeros(pt.n, dtype=torch.float64, device="cuda")
    (bsg.pcg if kind == "ich2" else bsg.gmres)(ctx, m, f, _t(b), x, p)
    A = s.to_scipy()
    xh = x.cpu().numpy()
    assert np.linalg.norm(b - A @ xh) <= 1e-8 * np.linalg.norm(b)


def test_trisolve_exact_matches_oracle(ctx, oracle, heat):
    import bsg
    import torch
    u = heat.upper()
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0)
    m = bsg.Matrix.from_system(ctx, heat, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    iu, ju, l, uu = f.export()
    x = np.random.default_rng(4).standard_normal(heat.n)
    y = torch.empty(heat.n, dtype=torch.float64, device="cuda")
    f.solve_l(_t(x), y, mode=0)
    ref = oracle.solve_l(iu, ju, l, x)
    assert np.abs(y.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    f.solve_u(_t(x), y, mode=0)
    ref = oracle.solve_u(iu, ju, uu, x)
    assert np.abs(y.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()


def test_trisolve_jacobi_converges(ctx, oracle, heat):
    import bsg
    import torch
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-2, tau2=1e-4, memory=20.0)
    m = bsg.Matrix.from_system(ctx, heat, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    iu, ju, l, uu = f.export()
    x = np.random.default_rng(5).standard_normal(heat.n)
    ref = oracle.solve_u(iu, ju, uu, x)
    y = torch.empty(heat.n, dtype=torch.float64, device="cuda")
    errs = []
    for sw in (1, 4, 40):
        f.solve_u(_t(x), y, mode=1, nsweeps=sw)
        errs.append(np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref))
    assert errs[0] > errs[1] > errs[2] and errs[2] < 1e-10


def _sweeps_fp32(N, dinv, x, nsweeps):
    """The FP32-iterate Jacobi recurrence of a triangular solve: y0 =
    fl32(D^-1 x), y_k = D^-1 (x - N y_(k-1)) with FP32 values of N and FP64
    products, rounded to FP32 except the last of nsweeps iterates."""
    y = (x * dinv).astype(np.float32)
    for k in range(nsweeps - 1):
        v = (x - N @ y.astype(np.float64)) * dinv
        y = v if k == nsweeps - 2 else v.astype(np.float32)
    return y


def _strict_parts32(iu, ju, l, u):
    """Strict lower rows (from L's columns) and strict upper rows of a factor
    in the reference layout, values rounded to FP32; inverse pivots."""
    import scipy.sparse as sp
    n = len(iu) - 1
    rows = np.repeat(np.arange(n), np.diff(iu))
    off = ju != rows
    f32 = lambda v: v[off].astype(np.float32).astype(np.float64)
    NU = sp.csr_matrix((f32(u), (rows[off], ju[off])), shape=(n, n))
    NL = sp.csr_matrix((f32(l), (ju[off], rows[off])), shape=(n, n))
    return NL, NU, l[iu[:-1]], u[iu[:-1]]


def _random_graph(n, deg, seed):
    """SPD matrix on a random graph (each row joined to `deg` random rows, weak
    couplings): the columns a row tile reads are spread over the whole vector."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    i = np.repeat(np.arange(n), deg)
    j = rng.integers(0, n, n * deg)
    keep = i != j
    W = sp.coo_matrix((-rng.uniform(0.02, 0.05, keep.sum()), (i[keep], j[keep])), shape=(n, n)).tocsr()
    W = (W + W.T).tocsr()
    W.sum_duplicates()
    A = (W + sp.diags(np.asarray(abs(W).sum(axis=1)).ravel() + 1.0)).tocsr()
    A.sort_indices()
    ia, ja, a = [], [], []
    for r in range(n):  # each row's diagonal first
        c, v = A.indices[A.indptr[r]:A.indptr[r + 1]], A.data[A.indptr[r]:A.indptr[r + 1]]
        d = c == r
        ja.append(np.concatenate([c[d], c[~d]]))
        a.append(np.concatenate([v[d], v[~d]]))
    ia = np.concatenate([[0], np.cumsum([len(c) for c in ja])]).astype(np.int32)
    return P.System(n, 1, ia, np.concatenate(ja).astype(np.int32), np.concatenate(a), np.zeros((1, n)), None)


@pytest.mark.parametrize("case", ["heat", "heat_odd", "random"])
def test_fp32_sweeps_match_restated_recurrence(ctx, heat, case):
    """The FP32-factor sweeps (tiled, with x staged in shared memory, for the
    stencil factors; gathered from global memory where a tile would stage too
    many x blocks, for the random graph) equal the restated recurrence.  An
    odd row count puts the second FP32 iterate of the ping-pong pair off a
    16-byte boundary (staged with plain loads then)."""
    import bsg
    import torch
    s = {"heat": lambda: heat, "heat_odd": lambda: P.heat3d(13, 11, 9, sigma=1.0, seed=5),
         "random": lambda: _random_graph(60000, 4, 21)}[case]()
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, precision=1)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    st = f.sell_stats()
    if case != "random":
        assert st["tiles_l"] > 0 and st["tiles_u"] > 0
    else:
        assert st["tiles_l"] == 0 and st["tiles_u"] == 0
    NL, NU, dl, du = _strict_parts32(*f.export())
    x = np.random.default_rng(6).standard_normal(s.n)
    y = torch.empty(s.n, dtype=torch.float64, device="cuda")
    for sw in (2, 3, 6):
        f.solve_l(_t(x), y, mode=1, nsweeps=sw)
        ref = _sweeps_fp32(NL, dl, x, sw)
        assert np.abs(y.cpu().numpy() - ref).max() <= 1e-6 * np.abs(ref).max(), ("L", sw)
        f.solve_u(_t(x), y, mode=1, nsweeps=sw)
        ref = _sweeps_fp32(NU, du, x, sw)
        assert np.abs(y.cpu().numpy() - ref).max() <= 1e-6 * np.abs(ref).max(), ("U", sw)


def test_pcg_matches_oracle(ctx, oracle, heat):
    import bsg
    import torch
    u = heat.upper()
    b = heat.rhs[0]
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, ittype=0, eps=1e-10)
    m = bsg.Matrix.from_system(ctx, heat, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    x = torch.zeros(heat.n, dtype=torch.float64, device="cuda")
    bsg.pcg(ctx, m, f, _t(b), x, p)
    iu, ju, _, uu = f.export()
    xo, it, _ = oracle.pcg(u.ia, u.ja, u.a, iu, ju, uu, b, ittype=0, eps=1e-10)
    assert abs(p.nitperf - it) <= 1
    xg = x.cpu().numpy()
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) < 1e-8
    assert p.resfin < 1e-9


@pytest.mark.parametrize("precision,trisolve", [(0, 0), (1, 0), (1, 1)])
def test_gmres_nonsymmetric(ctx, oracle, heat, precision, trisolve):
    import bsg
    import torch
    s = _nonsymmetric(heat)
    b = s.rhs[0]
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, sttype=1, eps=1e-8,
                          restart=30, precision=precision, trisolve=trisolve, nsweeps=4, krylov=1)
    m = bsg.Matrix.from_system(ctx, s)
    f = bsg.Factor(ctx, m, "ilu2", p)
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    bsg.gmres(ctx, m, f, _t(b), x, p)
    assert p.resfin <= 1e-8
    sia, sja, al, au = oracle.combine_lu(s.ia, s.ja, s.a)
    oiu, oju, ol, ou, _ = oracle.fact(1, sia, sja, al, au, tau1=1e-3, tau2=1e-3)
    xo, it, _ = oracle.gmres(s.ia, s.ja, s.a, oiu, oju, ol, ou, b, m=30, eps=1e-10)
    assert np.linalg.norm(x.cpu().numpy() - xo) / np.linalg.norm(xo) < 1e-6
    if precision == 0 and trisolve == 0:
        xg, itg, _ = oracle.gmres(s.ia, s.ja, s.a, oiu, oju, ol, ou, b, m=30, eps=1e-8)
        assert abs(p.nitperf - itg) <= 1


def test_solve_symm_host_driver(ctx, oracle, heat):
    import bsg
    u = heat.upper()
    b = heat.rhs[0]
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, ittype=0, eps=1e-10)
    x = bsg.solve_symm(ctx, u.n, u.ia, u.ja, u.a, b, p)
    oiu, oju, ou, _, _ = oracle.fact(0, u.ia, u.ja, u.a, tau1=1e-3, tau2=1e-3)
    xo, it, _ = oracle.pcg(u.ia, u.ja, u.a, oiu, oju, ou, b, ittype=0, eps=1e-10)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8
    assert p.resfin < 1e-9 and p.timefct > 0 and p.timeitr > 0


def test_nonpositive_pivot_reports_reference_error(ctx):
    import bsg
    # 3x3 symmetric indefinite matrix, upper storage
    ia = np.array([0, 2, 4, 5], np.int32)
    ja = np.array([0, 1, 1, 2, 2], np.int32)
    a = np.array([1.0, 2.0, 1.0, 0.5, 1.0])
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0)
    m = bsg.Matrix(ctx, 3, ia, ja, a, symm_upper=True)
    with pytest.raises(bsg.BsgError) as e:
        bsg.Factor(ctx, m, "ich2", p)
    assert e.value.code == bsg.ERR_PIVOT and "Diagonal pivot is nonpositive" in str(e.value)
    # the context stays usable after the reported error
    m2 = bsg.Matrix(ctx, 3, np.array([0, 1, 2, 3], np.int32), np.array([0, 1, 2], np.int32), np.ones(3),
                    symm_upper=True)
    bsg.Factor(ctx, m2, "ich2", p)


def test_bad_csr_rejected(ctx):
    """Host-buffer input is checked (on device copies) with the messages and
    in the order of the checks: row pointers, then columns, then the upper
    storage rule, the first failing row deciding between its two messages."""
    import bsg

    def bad(n, ia, ja, upper=False, bs=1):
        with pytest.raises(bsg.BsgError) as e:
            bsg.Matrix(ctx, n, np.array(ia, np.int32), np.array(ja, np.int32), np.ones(bs * bs * len(ja)), bs=bs,
                       symm_upper=upper)
        assert e.value.code == bsg.ERR_ARG
        return str(e.value)

    assert "ia not monotone" in bad(2, [0, 2, 1], [0, 1])
    assert "ia not monotone" in bad(2, [0, 1, -1], [0])
    assert "ia[0] != 0" in bad(2, [1, 2, 3], [0, 1])
    assert "out of range" in bad(2, [0, 1, 2], [0, 5])
    assert "out of range" in bad(3, [0, 1, 2, 3], [0, 7, 1], upper=True)  # before the upper rule
    assert "start with its diagonal" in bad(2, [0, 1, 2], [1, 1], upper=True)
    assert "below the diagonal" in bad(2, [0, 1, 3], [0, 1, 0], upper=True)
    # the first failing row decides: row 1 below / row 2 without its diagonal
    assert "below the diagonal" in bad(3, [0, 1, 3, 4], [0, 1, 0, 1], upper=True)
    assert "start with its diagonal" in bad(3, [0, 1, 2, 4], [0, 2, 2, 1], upper=True)
    # 3x3 blocks: the same checks on the block pattern
    assert "ia not monotone" in bad(2, [0, 2, 1], [0, 1], bs=3)
    assert "out of range" in bad(2, [0, 1, 2], [0, 2], bs=3)
    assert "start with its diagonal" in bad(2, [0, 2, 3], [1, 0, 1], upper=True, bs=3)
    # the context stays usable
    m = bsg.Matrix(ctx, 2, np.array([0, 1, 2], np.int32), np.array([0, 1], np.int32), np.ones(2), symm_upper=True)
    assert m.info()[0] == 2


@pytest.mark.parametrize("precision,trisolve", [(0, 0), (1, 1)])
def test_lanczos_matches_oracle(ctx, oracle, heat, precision, trisolve):
    """CSVector::Lanczos on the GPU: with the FP64 factor and exact solves it
    follows the oracle's recurrence (iterations +-1, same solution); with the
    FP32 factor and Jacobi sweeps it still reaches the tolerance."""
    import bsg
    import torch
    s = _nonsymmetric(heat, skew=0.4)
    b = s.rhs[0]
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, sttype=1, eps=1e-9, niter=500,
                          precision=precision, trisolve=trisolve, nsweeps=6)
    m = bsg.Matrix.from_system(ctx, s)
    f = bsg.Factor(ctx, m, "ilu2", p)
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    bsg.lanczos(ctx, m, f, _t(b), x, p)
    A = s.to_scipy()
    xg = x.cpu().numpy()
    r = b - A @ xg
    assert np.all(np.isfinite(xg))
    assert abs(p.resfin - np.linalg.norm(r) / np.linalg.norm(b)) <= 1e-12
    # the returned iterate is the one of least max-norm residual (the
    # reference's goodsol), recorded in resrec
    assert abs(np.abs(r).max() - p.resrec) <= 1e-12 * np.abs(b).max()
    sia, sja, al, au = oracle.combine_lu(s.ia, s.ja, s.a)
    oiu, oju, ol, ou, _ = oracle.fact(1, sia, sja, al, au, tau1=1e-3, tau2=1e-3)
    xo, it, _ = oracle.lanczos(s.ia, s.ja, s.a, oiu, oju, ol, ou, b, eps=1e-9, sttype=1)
    if precision == 0:
        assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(b)
        assert np.linalg.norm(xg - xo) <= 1e-6 * np.linalg.norm(xo)
        assert abs(p.nitperf - it) <= 1, (p.nitperf, it)
    else:
        # FP32 factor applied by sweeps: the recurrence is less smooth, and the
        # least-max-norm iterate can sit a little above the 2-norm target
        assert np.linalg.norm(r) <= 1e-7 * np.linalg.norm(b)
        assert np.linalg.norm(xg - xo) <= 1e-5 * np.linalg.norm(xo)


def test_solver_driver_runs_lanczos(ctx, oracle, heat):
    """bsg_solver_csr (CSVector::Solver): CombineLU + ILU2 + Lanczos by default."""
    import bsg
    s = _nonsymmetric(heat, skew=0.2)
    b = s.rhs[0]
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, sttype=1, eps=1e-9)
    x = bsg.solver(ctx, s.n, s.ia, s.ja, s.a, b, p)
    sia, sja, al, au = oracle.combine_lu(s.ia, s.ja, s.a)
    oiu, oju, ol, ou, _ = oracle.fact(1, sia, sja, al, au, tau1=1e-3, tau2=1e-3)
    xo, it, _ = oracle.lanczos(s.ia, s.ja, s.a, oiu, oju, ol, ou, b, eps=1e-9, sttype=1)
    assert abs(p.nitperf - it) <= 1 and p.resfin <= 1e-8
    assert np.linalg.norm(x - xo) <= 1e-6 * np.linalg.norm(xo)


@pytest.mark.parametrize("precision,mode", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_transposed_solves_are_adjoint(ctx, oracle, heat, precision, mode):
    """<y, U^{-1} x> = <U^{-T} y, x> and likewise for L, for exact solves and
    sweeps, FP64 and FP32 factors; the exact FP64 transposed solves equal the
    oracle's SolveL on U / SolveU on L."""
    import bsg
    import torch
    s = _nonsymmetric(heat, skew=0.4)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, precision=precision)
    m = bsg.Matrix.from_system(ctx, s)
    f = bsg.Factor(ctx, m, "ilu2", p)
    rng = np.random.default_rng(8)
    x, yv = rng.standard_normal(s.n), rng.standard_normal(s.n)
    out = torch.empty(s.n, dtype=torch.float64, device="cuda")
    tol = 1e-12 if precision == 0 else 1e-5
    for fwd, adj in ((f.solve_u, f.solve_ut), (f.solve_l, f.solve_lt)):
        fwd(_t(x), out, mode=mode, nsweeps=4)
        a = float(np.dot(yv, out.cpu().numpy()))
        adj(_t(yv), out, mode=mode, nsweeps=4)
        b = float(np.dot(out.cpu().numpy(), x))
        assert abs(a - b) <= tol * max(abs(a), 1.0), (a, b)
    if precision == 0 and mode == 0:
        iu, ju, l, u = f.export()
        f.solve_ut(_t(x), out, mode=0)
        ref = oracle.solve_l(iu, ju, u, x)
        assert np.abs(out.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
        f.solve_lt(_t(x), out, mode=0)
        ref = oracle.solve_u(iu, ju, l, x)
        assert np.abs(out.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()


def test_time_kernel_kinds(ctx):
    """bsg_time_kernel, the benchmark's event timer: the point and block
    products (kind 0), the product of several vectors (kind 3, 1..64 of them)
    and a sweep of a factor (kind 2); bad kinds and vector counts are refused."""
    import ctypes as C
    import bsg
    L = bsg.lib()
    tk = L.bsg_time_kernel
    tk.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    s = P.lame3d(5, 0.3, 1.0, 7)
    mb = bsg.Matrix.from_system(ctx, s)
    h = P.heat3d(10, 9, 8, sigma=1.0, seed=13)
    mp = bsg.Matrix.from_system(ctx, h, symm_upper=True)
    f = bsg.Factor(ctx, mp, "ich2", bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, precision=1))
    t = C.c_double()
    for m in (mb, mp):
        assert tk(ctx.h, 0, m.h, None, 0, 0, 3, C.byref(t)) == bsg.OK and t.value > 0
        for nv in (1, 6, 64):
            assert tk(ctx.h, 3, m.h, None, 0, nv, 3, C.byref(t)) == bsg.OK and t.value > 0
        for nv in (0, 65):
            assert tk(ctx.h, 3, m.h, None, 0, nv, 3, C.byref(t)) == bsg.ERR_ARG
    assert tk(ctx.h, 2, None, f.h, 1, 1, 3, C.byref(t)) == bsg.OK and t.value > 0
    assert tk(ctx.h, 4, mb.h, None, 0, 1, 3, C.byref(t)) == bsg.ERR_ARG
    assert tk(ctx.h, 3, None, None, 0, 1, 3, C.byref(t)) == bsg.ERR_ARG
