"""The CPU oracle against the reference Bslib (CPU only).

* against tests/golden/heat_8x8x6.npz -- outputs of the reference itself,
  made by tests/golden/make_golden.py (runs everywhere);
* against the live reference library oracle/_ref (runs where it was built).

The oracle applies factorisation updates in ascending row order and sums the
theta compensations in fixed point, the reference in its linked-list order:
the factors agree in pattern exactly and in value to rounding (1e-13
relative here); products and solves agree to 1e-14.
"""
import os

import numpy as np
import pytest

import problems as P

GOLD = os.path.join(os.path.dirname(__file__), "golden", "heat_8x8x6.npz")
GOLD_BLOCK = os.path.join(os.path.dirname(__file__), "golden", "lame_block.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_mvm_matches_reference(oracle, gold):
    g = gold
    assert rel(oracle.mvm(g["ia"], g["ja"], g["a"], g["x"]), g["mvm"]) < 1e-15
    assert rel(oracle.mvm(g["ua_ia"], g["ua_ja"], g["ua_a"], g["x"], symm=True), g["mvm_symm"]) < 1e-15


@pytest.mark.parametrize("tag,t1,t2", [("ic2_a", 1e-3, 1e-3), ("ic2_b", 1e-2, 1e-4)])
def test_ich2_matches_reference(oracle, gold, tag, t1, t2):
    g = gold
    iu, ju, uu, _, st = oracle.fact(0, g["ua_ia"], g["ua_ja"], g["ua_a"], tau1=t1, tau2=t2, theta=0.1)
    assert np.array_equal(iu, g[f"{tag}_iu"]) and np.array_equal(ju, g[f"{tag}_ju"])
    assert rel(uu, g[f"{tag}_u"]) < 1e-13
    assert np.allclose(st, g[f"{tag}_density"], rtol=0, atol=1e-12)
    # triangular solves with the reference's own factor
    assert rel(oracle.solve_l(g[f"{tag}_iu"], g[f"{tag}_ju"], g[f"{tag}_u"], g["x"]), g[f"{tag}_solve_l"]) < 1e-14
    assert rel(oracle.solve_u(g[f"{tag}_iu"], g[f"{tag}_ju"], g[f"{tag}_u"], g["x"]), g[f"{tag}_solve_u"]) < 1e-14


@pytest.mark.parametrize("tag,t1,t2", [("ilu2_a", 1e-3, 1e-3), ("ilu2_b", 1e-2, 1e-4)])
def test_ilu2_matches_reference(oracle, gold, tag, t1, t2):
    g = gold
    sia, sja, al, au = oracle.combine_lu(g["ia"], g["ja"], g["ns_a"])
    iu, ju, lv, uv, st = oracle.fact(1, sia, sja, al, au, tau1=t1, tau2=t2, theta=0.1)
    assert np.array_equal(iu, g[f"{tag}_iu"]) and np.array_equal(ju, g[f"{tag}_ju"])
    assert rel(lv, g[f"{tag}_l"]) < 1e-13
    assert rel(uv, g[f"{tag}_u"]) < 1e-13
    assert np.allclose(st, g[f"{tag}_density"], rtol=0, atol=1e-12)


def test_pcg_solution_matches_reference(oracle, gold):
    g = gold
    iu, ju, uu, _, _ = oracle.fact(0, g["ua_ia"], g["ua_ja"], g["ua_a"], tau1=1e-3, tau2=1e-3)
    x, it, _ = oracle.pcg(g["ua_ia"], g["ua_ja"], g["ua_a"], iu, ju, uu, g["b"], ittype=0, eps=1e-10)
    assert abs(it - int(g["symm_iters"])) <= 1
    assert rel(x, g["symm_x"]) < 1e-9


def test_gmres_solution_matches_reference_solver(oracle, gold):
    """The reference's nonsymmetric driver runs Lanczos, the GPU path GMRES:
    only the converged solutions are compared."""
    g = gold
    sia, sja, al, au = oracle.combine_lu(g["ia"], g["ja"], g["ns_a"])
    iu, ju, lv, uv, _ = oracle.fact(1, sia, sja, al, au, tau1=1e-3, tau2=1e-3)
    x, it, res = oracle.gmres(g["ia"], g["ja"], g["ns_a"], iu, ju, lv, uv, g["b"], m=30, eps=1e-11)
    assert res < 1e-11
    assert rel(x, g["nonsymm_x"]) < 1e-8


def test_compensation_sum_is_order_independent(oracle):
    """Factors of a symmetric-permutation-free problem do not depend on how
    many rows drop into the same diagonal: rerunning gives identical bits."""
    s = P.heat3d(9, 7, 5, sigma=1.2, seed=5).upper()
    a = oracle.fact(0, s.ia, s.ja, s.a, tau1=1e-2, tau2=1e-4)
    b = oracle.fact(0, s.ia, s.ja, s.a, tau1=1e-2, tau2=1e-4)
    assert all(np.array_equal(x, y) for x, y in zip(a[:4], b[:4]))


def test_live_reference_larger_case(oracle, reflib):
    s = P.heat3d(12, 11, 10, sigma=1.0, seed=23)
    u = s.upper()
    iu, ju, uu, _ = reflib.ich2(u.ia, u.ja, u.a, tau1=1e-3, tau2=1e-3)
    oiu, oju, ouu, _, _ = oracle.fact(0, u.ia, u.ja, u.a, tau1=1e-3, tau2=1e-3)
    assert np.array_equal(iu, oiu) and np.array_equal(ju, oju)
    assert rel(ouu, uu) < 1e-13
    x, info = reflib.solve_symm(u.ia, u.ja, u.a, s.rhs[0], memory=-1.0, eps=1e-10)
    xo, it, _ = oracle.pcg(u.ia, u.ja, u.a, oiu, oju, ouu, s.rhs[0], eps=1e-10)
    assert abs(it - info["iters"]) <= 1 and rel(xo, x) < 1e-9


def test_lanczos_matches_reference_solver(oracle, gold):
    """The oracle's restatement of CSVector::Lanczos against the reference's
    own Solver (CombineLU + ILU2 + Lanczos) recorded in the fixture."""
    g = gold
    sia, sja, al, au = oracle.combine_lu(g["ia"], g["ja"], g["ns_a"])
    iu, ju, lv, uv, _ = oracle.fact(1, sia, sja, al, au, tau1=1e-3, tau2=1e-3)
    x, it, _ = oracle.lanczos(g["ia"], g["ja"], g["ns_a"], iu, ju, lv, uv, g["b"], eps=1e-10, sttype=1)
    assert abs(it - int(g["nonsymm_iters"])) <= 1
    assert rel(x, g["nonsymm_x"]) < 1e-9


def test_live_reference_lanczos_larger_case(oracle, reflib):
    s = P.heat3d(12, 11, 10, sigma=1.0, seed=23)
    rows = np.repeat(np.arange(s.n), np.diff(s.ia))
    a = s.a.copy()
    off = s.ja != rows
    a[off] *= 1.0 + 0.4 * np.sign(s.ja[off] - rows[off])
    x, info = reflib.solver(s.ia, s.ja, a, s.rhs[0], tau1=1e-3, tau2=1e-3, sttype=1, eps=1e-9)
    sia, sja, al, au = oracle.combine_lu(s.ia, s.ja, a)
    iu, ju, lv, uv, _ = oracle.fact(1, sia, sja, al, au, tau1=1e-3, tau2=1e-3)
    xo, it, _ = oracle.lanczos(s.ia, s.ja, a, iu, ju, lv, uv, s.rhs[0], eps=1e-9, sttype=1)
    assert abs(it - info["iters"]) <= 1
    assert rel(xo, x) < 1e-7


# ---- block (CSMatrixRS) ILU2: the oracle replays the reference's own update
#      order and calls the same LAPACK dgesvd, so it agrees bit for bit ----

@pytest.fixture(scope="module")
def gold_block():
    return np.load(GOLD_BLOCK)


def test_block_combine_lu_matches_reference(oracle, gold_block):
    g = gold_block
    ia_s, ja_s, al, au = oracle.combine_lu_block(g["ia"], g["ja"], g["a"], int(g["bs"]))
    assert np.array_equal(ia_s, g["clu_ia"]) and np.array_equal(ja_s, g["clu_ja"])
    assert np.array_equal(al, g["clu_l"]) and np.array_equal(au, g["clu_u"])


@pytest.mark.parametrize("tag,vals,t1,t2", [("bilu_a", "a", 1e-3, 1e-3), ("bilu_b", "a", 1e-2, 1e-5),
                                            ("bilu_ns", "ns_a", 1e-3, 1e-4)])
def test_block_ilu2_matches_reference(oracle, gold_block, tag, vals, t1, t2):
    g = gold_block
    bs = int(g["bs"])
    clu = oracle.combine_lu_block(g["ia"], g["ja"], g[vals], bs)
    ia_f, ja_f, l, u, st = oracle.ilu2_block(*clu, bs, tau1=t1, tau2=t2, theta=0.1)
    assert np.array_equal(ia_f, g[f"{tag}_ia"]) and np.array_equal(ja_f, g[f"{tag}_ja"])
    assert np.array_equal(l, g[f"{tag}_l"]) and np.array_equal(u, g[f"{tag}_u"])
    assert np.allclose(st, g[f"{tag}_density"], rtol=0, atol=1e-14)
    x = g["x"]
    assert np.array_equal(oracle.solve_l_block(ia_f, ja_f, l, bs, x), g[f"{tag}_solve_l"])
    assert np.array_equal(oracle.solve_u_block(ia_f, ja_f, u, bs, x), g[f"{tag}_solve_u"])


def test_live_reference_block_ilu2_larger_cases(oracle, reflib):
    cases = [(P.lame3d(9, sigma=1.0, seed=33), 1e-3, 1e-3),
             (P.lame_periodic(10, rmin=1.5, rmax=3.0, seed=34), 1e-2, 1e-4)]
    for s, t1, t2 in cases:
        ia_f, ja_f, l, u, st = reflib.ilu2_block(s.ia, s.ja, s.a, 3, tau1=t1, tau2=t2)
        o = oracle.ilu2_block(*oracle.combine_lu_block(s.ia, s.ja, s.a, 3), 3, tau1=t1, tau2=t2)
        assert np.array_equal(o[0], ia_f) and np.array_equal(o[1], ja_f)
        assert np.array_equal(o[2], l) and np.array_equal(o[3], u)


@pytest.mark.parametrize("tag,t1,t2", [("bic_a", 1e-3, 1e-3), ("bic_b", 1e-2, 1e-5)])
def test_block_ich2_matches_reference(oracle, gold_block, tag, t1, t2):
    g = gold_block
    bs = int(g["bs"])
    ia_f, ja_f, u, st = oracle.ich2_block(g["ua_ia"], g["ua_ja"], g["ua_a"], bs, tau1=t1, tau2=t2, theta=0.1)
    assert np.array_equal(ia_f, g[f"{tag}_ia"]) and np.array_equal(ja_f, g[f"{tag}_ja"])
    assert np.array_equal(u, g[f"{tag}_u"])
    x = g["x"]
    assert np.array_equal(oracle.solve_l_block(ia_f, ja_f, u, bs, x), g[f"{tag}_solve_l"])
    assert np.array_equal(oracle.solve_u_block(ia_f, ja_f, u, bs, x), g[f"{tag}_solve_u"])


def test_live_reference_block_ich2_larger_cases(oracle, reflib):
    for s, t1, t2 in [(P.lame3d(9, sigma=1.0, seed=35), 1e-3, 1e-3),
                      (P.lame_periodic(10, rmin=1.5, rmax=3.0, seed=36), 1e-2, 1e-4)]:
        u = s.upper()
        ia_f, ja_f, uf, _ = reflib.ich2_block(u.ia, u.ja, u.a, 3, tau1=t1, tau2=t2)
        o = oracle.ich2_block(u.ia, u.ja, u.a, 3, tau1=t1, tau2=t2)
        assert np.array_equal(o[0], ia_f) and np.array_equal(o[1], ja_f) and np.array_equal(o[2], uf)


def test_ich0_matches_reference(oracle, gold):
    """IC(0) (CSMatrixR::Ich): the oracle's factor is the reference's bit for
    bit (the same products and subtractions, no fused multiply-add)."""
    g = gold
    iu, ju, u = oracle.ich0(g["ua_ia"], g["ua_ja"], g["ua_a"])
    assert np.array_equal(iu, g["ic0_iu"]) and np.array_equal(ju, g["ic0_ju"])
    assert np.array_equal(u, g["ic0_u"])


def test_ich0_matches_live_reference_at_cfg1(oracle, reflib):
    s = P.config(1)
    u = s.upper()
    a = oracle.ich0(u.ia, u.ja, u.a)
    b = reflib.ich0(u.ia, u.ja, u.a)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
