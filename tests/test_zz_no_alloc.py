"""The allocation-free sweep solve (bsg_solve_sweep_static) against the
allocating entry points bsg_solve_l_dev / bsg_solve_u_dev in sweep mode.

Both run the same kernels in the same order, so the results agree to the
last bit; the test allows 1e-14 relative.  Two calls in a row check that the
shared static work array carries nothing from one call to the next.  The
library allocates from the device's default stream-ordered memory pool; the
pool's high-water mark, reset before each call, shows that the static entry
point takes nothing from it while the allocating entry point does.
"""
import ctypes as C

import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu

TOL = 1e-14


def _pool_marks(device=0):
    """(used bytes now, high-water mark) of the device's default memory pool."""
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(device)
    assert err == rt.cudaError_t.cudaSuccess
    err, cur = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    assert err == rt.cudaError_t.cudaSuccess
    err, high = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh)
    assert err == rt.cudaError_t.cudaSuccess
    return int(cur), int(high)


def _reset_high_mark(device=0):
    from cuda.bindings import driver as dr
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(device)
    assert err == rt.cudaError_t.cudaSuccess
    (err,) = rt.cudaMemPoolSetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh, dr.cuuint64_t(0))
    assert err == rt.cudaError_t.cudaSuccess


def _static_solve(ctx, f, lower, nsweeps, x, y):
    import bsg
    L = bsg.lib()
    fn = L.bsg_solve_sweep_static
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    return fn(ctx.h, f.h, lower, nsweeps, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()))


@pytest.mark.parametrize("precision", [0, 1])
def test_static_sweep_matches_allocating_solve(ctx, precision):
    import bsg
    import torch
    s = P.heat3d(20, 18, 16, sigma=1.0, seed=21)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, precision=precision)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    rng = np.random.default_rng(7)
    for lower in (1, 0):
        for nsweeps in (2, 5):
            for call in range(2):
                x = torch.as_tensor(rng.standard_normal(s.n), device="cuda")
                want = torch.empty_like(x)
                got = torch.full_like(x, np.nan)
                ctx.sync()
                _reset_high_mark()
                base, _ = _pool_marks()
                (f.solve_l if lower else f.solve_u)(x, want, mode=1, nsweeps=nsweeps)
                ctx.sync()
                _, high_alloc = _pool_marks()
                assert high_alloc > base, "the allocating solve should draw its work vector from the pool"
                _reset_high_mark()
                assert _static_solve(ctx, f, lower, nsweeps, x, got) == bsg.OK, bsg.lib().bsg_last_error()
                ctx.sync()
                cur, high = _pool_marks()
                assert cur == base and high == base, ("the static solve took pool memory", base, cur, high)
                w, g = want.cpu().numpy(), got.cpu().numpy()
                assert np.all(np.isfinite(g))
                assert np.abs(g - w).max() <= TOL * np.abs(w).max(), (lower, nsweeps, call)


def test_static_sweep_rejects_too_many_rows(ctx):
    import bsg
    import torch
    n = (1 << 21) + 1
    ia = np.arange(n + 1, dtype=np.int32)
    ja = np.arange(n, dtype=np.int32)
    m = bsg.Matrix(ctx, n, ia, ja, np.full(n, 4.0), symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", bsg.default_param(ordtype=0, fcttyp=2))
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    rc = _static_solve(ctx, f, 1, 3, x, y)
    assert rc == bsg.ERR_ARG
    assert "exceed the static scratch" in bsg.lib().bsg_last_error().decode()
