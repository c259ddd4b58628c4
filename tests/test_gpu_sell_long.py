"""Rows too long for a SELL slice (k_sell.cu): rows of more than 256 entries
leave the slices and are summed by a warp, beyond 4096 by a whole block, in
the same kernel as the slices.  The products and sweeps of a matrix with both
kinds of rows, in L and U, must equal plain CSR arithmetic.

Tolerances: the long rows sum in a tree, not in the CPU loop's order, so FP64
products and sweeps are held to 1e-13 / 1e-12 relative; FP32-factor sweeps to
the restated FP32 recurrence at 1e-6, as for the short-row factors.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import problems as P

pytestmark = pytest.mark.gpu


def _t(x):
    import torch
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device="cuda")


def _bordered(m, border, medium, seed):
    """SPD heat matrix on an m^3 grid bordered by `border` nodes joined to
    every grid node and `medium` nodes joined to 300..2000 random grid nodes.
    Order: half the medium nodes, the grid, the other medium half, the border
    -- so that the strict upper rows of the first ones and the strict lower
    rows of the last ones are long.  (Border nodes first would make every grid
    row merge a 5000-entry row tail in the factorisation.)"""
    rng = np.random.default_rng(seed)
    h = P.heat3d(m, sigma=0.5, seed=seed)
    n0, nx = h.n, border + medium
    rows = np.repeat(np.arange(n0), np.diff(h.ia))
    A = sp.csr_matrix((h.a, (rows, h.ja)), shape=(n0, n0))
    ei, ej, ev = [], [], []
    for k in range(nx):
        cols = np.arange(n0) if k < border else rng.choice(n0, rng.integers(300, 2000), replace=False)
        ei.append(np.full(len(cols), n0 + k))
        ej.append(cols)
        ev.append(-rng.uniform(0.2, 0.4, len(cols)))
    N = n0 + nx
    B = sp.coo_matrix((np.concatenate(ev), (np.concatenate(ei), np.concatenate(ej))), shape=(N, N)).tocsr()
    A = sp.bmat([[A, None], [None, sp.csr_matrix((nx, nx))]]).tocsr() + B + B.T
    d = np.asarray(abs(A).sum(axis=1)).ravel()
    A = A + sp.diags(np.where(np.arange(N) >= n0, d + 1.0, np.asarray(abs(B.T).sum(axis=1)).ravel()))
    mh = medium // 2
    order = np.concatenate([n0 + border + np.arange(mh), np.arange(n0), n0 + border + np.arange(mh, medium),
                            n0 + np.arange(border)])
    A = A.tocsr()[order][:, order].tocsr()
    A.sort_indices()
    ja, a = [], []
    for r in range(N):  # each row's diagonal first
        c, v = A.indices[A.indptr[r]:A.indptr[r + 1]], A.data[A.indptr[r]:A.indptr[r + 1]]
        dg = c == r
        ja.append(np.concatenate([c[dg], c[~dg]]))
        a.append(np.concatenate([v[dg], v[~dg]]))
    ia = np.concatenate([[0], np.cumsum([len(c) for c in ja])]).astype(np.int32)
    return P.System(N, 1, ia, np.concatenate(ja).astype(np.int32), np.concatenate(a), np.zeros((1, N)), None)


@pytest.fixture(scope="module")
def bordered():
    return _bordered(17, 2, 40, 3)


@pytest.mark.parametrize("symm", [False, True])
def test_spmv_long_rows(ctx, bordered, symm):
    import bsg
    import torch
    s = bordered
    m = bsg.Matrix.from_system(ctx, s, symm_upper=symm)
    assert m.sell_stats()["long"] == int((np.diff(s.ia) > 256).sum()) == 42
    rows = np.repeat(np.arange(s.n), np.diff(s.ia))
    A = sp.csr_matrix((s.a, (rows, s.ja)), shape=(s.n, s.n))
    x = np.random.default_rng(4).standard_normal(s.n)
    y = torch.empty(s.n, dtype=torch.float64, device="cuda")
    m.mvm(_t(x), y)
    ref = A @ x
    scale = abs(A) @ abs(x)
    assert np.all(np.abs(y.cpu().numpy() - ref) <= 1e-13 * scale)


def _strict(iu, ju, l, u, fp32):
    n = len(iu) - 1
    rows = np.repeat(np.arange(n), np.diff(iu))
    off = ju != rows
    cast = (lambda v: v[off].astype(np.float32).astype(np.float64)) if fp32 else (lambda v: v[off])
    NU = sp.csr_matrix((cast(u), (rows[off], ju[off])), shape=(n, n))
    NL = sp.csr_matrix((cast(l), (ju[off], rows[off])), shape=(n, n))
    return NL, NU, l[iu[:-1]], u[iu[:-1]]


def _sweeps(N, dinv, x, nsweeps, fp32):
    """y0 = D^-1 x, y_k = D^-1 (x - N y_(k-1)); with fp32 the iterates but the
    last are rounded to FP32 (products and sums stay FP64)."""
    y = x * dinv
    if fp32:
        y = y.astype(np.float32)
    for k in range(nsweeps - 1):
        v = (x - N @ y.astype(np.float64)) * dinv
        y = v if (k == nsweeps - 2 or not fp32) else v.astype(np.float32)
    return y


@pytest.mark.parametrize("precision", [0, 1])
def test_sweeps_long_rows(ctx, bordered, precision):
    import bsg
    import torch
    s = bordered
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, precision=precision)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    iu, ju, l, u = f.export()
    rows = np.repeat(np.arange(s.n), np.diff(iu))
    lenu = np.diff(iu) - 1
    lenl = np.bincount(ju[ju != rows], minlength=s.n)
    # rows for a block (L) and for a warp (both sides)
    assert (lenl > 4096).sum() >= 1
    for ln in (lenl, lenu):
        assert ((ln > 256) & (ln <= 4096)).sum() >= 10
    st = f.sell_stats()
    assert st["long_l"] == (lenl > 256).sum() and st["long_u"] == (lenu > 256).sum()
    assert st["tiles_l"] == 0 and st["tiles_u"] == 0
    NL, NU, dl, du = _strict(iu, ju, l, u, precision == 1)
    x = np.random.default_rng(6).standard_normal(s.n)
    y = torch.empty(s.n, dtype=torch.float64, device="cuda")
    tol = 1e-6 if precision == 1 else 1e-12
    for sw in (2, 3, 6):
        f.solve_l(_t(x), y, mode=1, nsweeps=sw)
        ref = _sweeps(NL, dl, x, sw, precision == 1)
        assert np.abs(y.cpu().numpy() - ref).max() <= tol * np.abs(ref).max(), ("L", sw)
        f.solve_u(_t(x), y, mode=1, nsweeps=sw)
        ref = _sweeps(NU, du, x, sw, precision == 1)
        assert np.abs(y.cpu().numpy() - ref).max() <= tol * np.abs(ref).max(), ("U", sw)
