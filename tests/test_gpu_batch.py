"""Batched PCG (bsg_pcg_batch_dev) on the GPU: many independent problems as
segments of one block-diagonal matrix, and several load cases of one
matrix, each system with its own scalars and stopping test.

Checks: every system reaches the FP64 true relative residual 1e-8; its
solution agrees with a sparse direct solve to 1e-6 relative; its iteration
count is the single-system PCG's (the same recurrence; the segmented sums
round differently, so +-1); a matrix that couples two segments is refused.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import problems as P

pytestmark = pytest.mark.gpu


def _sub(s, a, b):
    """Rows / columns [a, b) of a point CSR system (a diagonal block)."""
    A = s.to_scipy()[a:b, a:b].tocsr()
    A.sort_indices()
    rhs = s.rhs[:, a:b] if s.rhs.ndim == 2 else s.rhs[a:b]
    return P.System(b - a, 1, A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.copy(), rhs,
                    np.array([0, b - a]), s.info)


@pytest.mark.parametrize("precision,trisolve", [(0, 0), (1, 1)])
def test_batch_of_independent_problems(ctx, precision, trisolve):
    import bsg
    import torch
    s = P.heat2d_batch(24, 8, 40, sigma=1.0, seed=3)
    parts = s.parts
    assert len(parts) == 25
    prm = dict(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, ittype=0, eps=1e-8, niter=2000,
               precision=precision, trisolve=trisolve, nsweeps=6)
    p = bsg.default_param(**prm)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    b = s.rhs[0]
    B = torch.as_tensor(b, device="cuda").reshape(1, -1).contiguous()
    X = torch.zeros_like(B)
    it, rs, tuned = bsg.pcg_batch(ctx, m, f, B, X, p, seg_off=parts)
    x = X.cpu().numpy()[0]
    assert rs.max() <= 1e-8, rs.max()
    assert tuned[0] in (4096, 16384, 65536) and tuned[3] >= 1
    A = s.to_scipy().tocsc()
    for g in range(len(parts) - 1):
        a, e = parts[g], parts[g + 1]
        xe = spla.spsolve(A[a:e, a:e], b[a:e])
        assert np.linalg.norm(x[a:e] - xe) <= 1e-6 * np.linalg.norm(xe), g
    # the single-system PCG on a few of the segments takes the same iterations
    for g in (0, 7, 23):
        a, e = parts[g], parts[g + 1]
        ss = _sub(s, a, e)
        ms = bsg.Matrix.from_system(ctx, ss, symm_upper=True)
        ps = bsg.default_param(**prm)
        fs = bsg.Factor(ctx, ms, "ich2", ps)
        xs = torch.zeros(e - a, dtype=torch.float64, device="cuda")
        bsg.pcg(ctx, ms, fs, torch.as_tensor(b[a:e], device="cuda"), xs, ps)
        assert abs(int(it[g]) - ps.nitperf) <= 1, (g, it[g], ps.nitperf)


def test_multiple_load_cases(ctx):
    import bsg
    import torch
    s = P.lame_periodic(8, 0.3, 1.5, 2.5, 0.3, 100.0, 2)
    assert s.rhs.shape[0] == 6
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, ittype=0, eps=1e-8, niter=3000,
                          precision=1, trisolve=1, nsweeps=6)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)  # 3x3 blocks
    f = bsg.Factor(ctx, m, "ich2", p)
    B = torch.as_tensor(np.ascontiguousarray(s.rhs), device="cuda")
    X = torch.zeros_like(B)
    it, rs, _ = bsg.pcg_batch(ctx, m, f, B, X, p)
    assert len(it) == 6 and rs.max() <= 1e-8
    A = s.to_scipy().tocsc()
    lu = spla.splu(A)
    x = X.cpu().numpy()
    for k in range(6):
        xe = lu.solve(s.rhs[k])
        assert np.linalg.norm(x[k] - xe) <= 1e-6 * np.linalg.norm(xe), k
    # one right-hand side alone through the single-system PCG
    x1 = torch.zeros(s.n * 3, dtype=torch.float64, device="cuda")
    p1 = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, ittype=0, eps=1e-8,
                           niter=3000, precision=1, trisolve=1, nsweeps=6)
    bsg.pcg(ctx, m, f, B[2].contiguous(), x1, p1)
    assert abs(int(it[2]) - p1.nitperf) <= 1


def test_coupled_segments_are_refused(ctx):
    import bsg
    import torch
    s = P.heat3d(8, 8, 8, sigma=0.5, seed=1)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, ittype=0, eps=1e-8)
    f = bsg.Factor(ctx, m, "ich2", p)
    B = torch.ones((1, s.n), dtype=torch.float64, device="cuda")
    X = torch.zeros_like(B)
    with pytest.raises(bsg.BsgError) as e:
        bsg.pcg_batch(ctx, m, f, B, X, p, seg_off=[0, 256, 512])
    assert e.value.code == bsg.ERR_ARG and "couples" in str(e.value)
