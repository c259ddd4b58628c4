"""Failure detection on the GPU without a fault: every device spin-wait has a
time limit (bsg_set_spin_limit_ns), after which the kernel records
BSG_ERR_TIMEOUT in the context's status word and returns, and the context
stays usable.

The waits are made to run out by a limit far below their legitimate length:
on a 1-D chain (the tridiagonal 1-D heat matrix) every row of the factor
depends on the one before, so a warp that claims row i waits for thousands
of rows to be solved or factored ahead of it, milliseconds, against a limit
of 10 microseconds.  Nothing is left waiting: a warp whose wait runs out
stops waiting, and every other warp leaves as soon as it sees the status.
After the timeout the limit goes back to its default and the same call, in
the same context, succeeds and agrees with the oracle.
"""
import numpy as np
import pytest
import torch

import problems as P

pytestmark = pytest.mark.gpu

DEFAULT_NS = 2_000_000_000
SHORT_NS = 10_000


def chain(n):
    return P.heat3d(n, 1, 1, sigma=1.0, seed=5)


def test_spin_limit_range(ctx):
    import bsg
    L = bsg.lib()
    assert L.bsg_set_spin_limit_ns(ctx.h, 999) == bsg.ERR_ARG
    assert L.bsg_set_spin_limit_ns(ctx.h, 601_000_000_000) == bsg.ERR_ARG
    assert L.bsg_set_spin_limit_ns(ctx.h, DEFAULT_NS) == bsg.OK


def test_sync_free_solve_wait_runs_out(ctx, oracle):
    import bsg
    L = bsg.lib()
    s = chain(200_000)
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    f = bsg.Factor(ctx, m, "ich2", p)
    x = torch.as_tensor(np.random.default_rng(1).standard_normal(s.n), device="cuda")
    y = torch.empty_like(x)
    try:
        assert L.bsg_set_spin_limit_ns(ctx.h, SHORT_NS) == bsg.OK
        rc = L.bsg_solve_l_dev(ctx.h, f.h, 0, 1, bsg._ptr(x), bsg._ptr(y))
        assert rc == bsg.ERR_TIMEOUT, (rc, L.bsg_last_error())
    finally:
        assert L.bsg_set_spin_limit_ns(ctx.h, DEFAULT_NS) == bsg.OK
    # the context still works: the same solve, now to completion
    f.solve_l(x, y, mode=0)
    ctx.sync()
    giu, gju, _, gu = f.export()
    want = oracle.solve_l(giu, gju, gu, x.cpu().numpy())
    got = y.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


def test_factorisation_scheduler_wait_runs_out(ctx, oracle):
    import bsg
    L = bsg.lib()
    s = chain(100_000)
    u = s.upper()
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0)
    m = bsg.Matrix.from_system(ctx, s, symm_upper=True)
    try:
        assert L.bsg_set_spin_limit_ns(ctx.h, SHORT_NS) == bsg.OK
        with pytest.raises(bsg.BsgError) as e:
            bsg.Factor(ctx, m, "ich2", p)
        assert e.value.code == bsg.ERR_TIMEOUT, str(e.value)
    finally:
        assert L.bsg_set_spin_limit_ns(ctx.h, DEFAULT_NS) == bsg.OK
    f = bsg.Factor(ctx, m, "ich2", p)
    giu, gju, _, gu = f.export()
    iu, ju, uu, _, _ = oracle.fact(0, u.ia, u.ja, u.a, tau1=1e-3, tau2=1e-3)
    assert np.array_equal(giu, iu) and np.array_equal(gju, ju) and np.array_equal(gu, uu)
