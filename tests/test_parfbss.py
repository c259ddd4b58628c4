"""Bslib's ParFBSS_* interface on one GPU (include/bsg_parfbss.h).

The reference's own ParFBSS (Bslib/parfbss.cpp) partitions the rows over MPI
ranks with METIS (it sets ordtype = 1, :447); neither exists here, so the
reference side of the comparison is its serial driver on the same system:
CSVector::SolveSymm (IC2 + PCG) for ParFBSS_SolveSymm and CSVector::Solver
(ILU2 + Lanczos) for ParFBSS_Solve, natural order.  The solution must agree
with it to 1e-8 relative (both stop at relative residual 1e-10 on small,
well-conditioned systems).

CPU tests: the object registry (20 objects, -1 when full or for a bad number),
the data arrays handed out, the data checks of ParFBSS_Solve_Ini
(Bslib/parfbss.cpp:712-790: ia[0] == 0, no empty row, columns in range) and
the rule of one process (LIST numbers every row once), and the reference's
C++ names exported.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import problems as P

IP = C.POINTER(C.c_int)
DP = C.POINTER(C.c_double)


def lib():
    import bsg
    L = bsg.lib()
    sig = {
        "bsg_parfbss_create": [C.c_void_p, C.c_int, C.c_int, IP],
        "bsg_parfbss_recreate": [C.c_int, C.c_int, C.c_int],
        "bsg_parfbss_linear_equations_data": [C.c_int, C.POINTER(IP), C.POINTER(IP), C.POINTER(IP), C.POINTER(DP),
                                              C.POINTER(DP), C.POINTER(DP)],
        "bsg_parfbss_normalization_data": [C.c_int, C.POINTER(DP)],
        "bsg_parfbss_nonlinear_equations_data": [C.c_int, C.POINTER(DP)],
        "bsg_parfbss_set_solver_parameters": [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                              C.c_double],
        "bsg_parfbss_set_msglev_and_filename": [C.c_int, C.c_int, C.c_char_p],
        "bsg_parfbss_set_schurtype": [C.c_int, C.c_int, C.c_int],
        "bsg_parfbss_set_ncpuext": [C.c_int, C.c_int],
        "bsg_parfbss_solve_symm": [C.c_int, C.c_int, IP],
        "bsg_parfbss_solve": [C.c_int, C.c_int, IP],
        "bsg_parfbss_solution": [C.c_int, C.POINTER(DP)],
        "bsg_parfbss_distribution": [C.c_int, IP, C.POINTER(IP)],
        "bsg_parfbss_destroy": [C.c_int],
    }
    for nm, at in sig.items():
        f = getattr(L, nm)
        f.argtypes = at
        f.restype = C.c_int
    return L


class Obj:
    """One ParFBSS object filled with a CSR system given row by row in the
    order `order` (LIST[i] = order[i]) with each row's columns shuffled."""

    def __init__(self, ia, ja, a, b, order, seed=0):
        self.L = lib()
        n = len(ia) - 1
        self.n = n
        oid = C.c_int(-1)
        assert self.L.bsg_parfbss_create(None, n, int(ia[-1]), C.byref(oid)) == 0
        self.id = oid.value
        pl, pia, pja = IP(), IP(), IP()
        pa, pb, px = DP(), DP(), DP()
        assert self.L.bsg_parfbss_linear_equations_data(self.id, C.byref(pl), C.byref(pia), C.byref(pja),
                                                        C.byref(pa), C.byref(pb), C.byref(px)) == 0
        rng = np.random.default_rng(seed)
        lst = np.ctypeslib.as_array(pl, (n,))
        lia = np.ctypeslib.as_array(pia, (n + 1,))
        lja = np.ctypeslib.as_array(pja, (int(ia[-1]),))
        la = np.ctypeslib.as_array(pa, (int(ia[-1]),))
        lb = np.ctypeslib.as_array(pb, (n,))
        lx = np.ctypeslib.as_array(px, (n,))
        lia[0] = 0
        for i, g in enumerate(order):
            lst[i] = g
            cols = np.arange(ia[g], ia[g + 1])
            rng.shuffle(cols)
            k0 = lia[i]
            lja[k0:k0 + len(cols)] = ja[cols]
            la[k0:k0 + len(cols)] = a[cols]
            lia[i + 1] = k0 + len(cols)
            lb[i] = b[g]
            lx[i] = 0.0
        self.views = (lst, lia, lja, la, lb, lx)

    def solution(self):
        ps = DP()
        assert self.L.bsg_parfbss_solution(self.id, C.byref(ps)) == 0
        return np.ctypeslib.as_array(ps, (self.n,)).copy()

    def destroy(self):
        assert self.L.bsg_parfbss_destroy(self.id) == 0


# ------------------------------------------------------------------ CPU
def test_registry_holds_twenty_objects():
    L = lib()
    ids = []
    for _ in range(20):
        oid = C.c_int(-1)
        assert L.bsg_parfbss_create(None, 4, 8, C.byref(oid)) == 0
        ids.append(oid.value)
    assert sorted(ids) == list(range(20))
    oid = C.c_int(-1)
    assert L.bsg_parfbss_create(None, 4, 8, C.byref(oid)) == -1
    assert L.bsg_parfbss_destroy(5) == 0
    assert L.bsg_parfbss_create(None, 4, 8, C.byref(oid)) == 0 and oid.value == 5
    for i in ids:
        assert L.bsg_parfbss_destroy(i) == 0
    assert L.bsg_parfbss_destroy(3) == -1
    n = C.c_int()
    for bad in (-1, 20, 7):
        assert L.bsg_parfbss_solve_symm(bad, 1, C.byref(n)) == -1
        assert L.bsg_parfbss_set_solver_parameters(bad, 1, 1e-3, 1e-3, 0.1, 10, 1e-8) == -1
        assert L.bsg_parfbss_recreate(bad, 4, 4) == -1


def test_data_arrays_and_recreate():
    L = lib()
    oid = C.c_int(-1)
    assert L.bsg_parfbss_create(None, 3, 5, C.byref(oid)) == 0
    pn = DP()
    assert L.bsg_parfbss_normalization_data(oid.value, C.byref(pn)) == 0
    assert np.array_equal(np.ctypeslib.as_array(pn, (3,)), np.ones(3))
    pp = DP()
    assert L.bsg_parfbss_nonlinear_equations_data(oid.value, C.byref(pp)) == 0
    assert np.array_equal(np.ctypeslib.as_array(pp, (3,)), np.zeros(3))
    assert L.bsg_parfbss_recreate(oid.value, 6, 10) == 0
    assert L.bsg_parfbss_normalization_data(oid.value, C.byref(pn)) == 0
    assert np.array_equal(np.ctypeslib.as_array(pn, (6,)), np.ones(6))
    assert L.bsg_parfbss_set_msglev_and_filename(oid.value, 1, b"log.txt") == 0
    assert L.bsg_parfbss_set_schurtype(oid.value, 1, 2) == 0
    assert L.bsg_parfbss_set_ncpuext(oid.value, 2) == 0
    assert L.bsg_parfbss_destroy(oid.value) == 0


def _heat(n=5):
    s = P.heat3d(n, n, n, sigma=1.0, seed=23)
    return s


@pytest.mark.parametrize("what", ["ia0", "empty_row", "column", "list_repeat", "list_range"])
def test_malformed_data_is_refused_before_any_device_use(what):
    s = _heat(4)
    order = np.arange(s.n)
    o = Obj(s.ia, s.ja, s.a, s.rhs[0], order)
    lst, lia, lja, la, lb, lx = o.views
    if what == "ia0":
        lia[0] = 1
    elif what == "empty_row":
        lia[3] = lia[2]
    elif what == "column":
        lja[5] = s.n
    elif what == "list_repeat":
        lst[1] = lst[0]
    else:
        lst[2] = s.n + 3
    n = C.c_int(-7)
    assert o.L.bsg_parfbss_solve_symm(o.id, 1, C.byref(n)) == -1
    assert o.L.bsg_parfbss_solve(o.id, 1, C.byref(n)) == -1
    o.destroy()


def test_reference_names_are_exported():
    import bsg
    syms = subprocess.run(["nm", "-DC", bsg.LIB_SO], capture_output=True, text=True, check=True).stdout
    for sig in ("ParFBSS_Create(void*, int, int, int*)", "ParFBSS_ReCreate(int, int, int)",
                "ParFBSS_LinearEquationsData(int, int**, int**, int**, double**, double**, double**)",
                "ParFBSS_NormalizationData(int, double**)", "ParFBSS_NonLinearEquationsData(int, double**)",
                "ParFBSS_SetSolverParameters(int, int, double, double, double, int, double)",
                "ParFBSS_SetMsglevAndFilename(int, int, char*)", "ParFBSS_SetSchurtype(int, int, int)",
                "ParFBSS_SetNcpuext(int, int)", "ParFBSS_SolveSymm(int, int, int*)", "ParFBSS_Solve(int, int, int*)",
                "ParFBSS_Solution(int, double**)", "ParFBSS_Distribution(int, int*, int**)",
                "ParFBSS_Destroy(int)"):
        assert sig in syms, sig


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("eps", [1e-10, -1e-9])
def test_solve_symm_matches_reference(ctx, reflib, eps):
    s = P.heat3d(10, 9, 8, sigma=1.0, seed=29)
    order = np.random.default_rng(4).permutation(s.n)
    o = Obj(s.ia, s.ja, s.a, s.rhs[0], order, seed=5)
    assert o.L.bsg_parfbss_set_solver_parameters(o.id, 1, 1e-3, 1e-3, 0.1, 2000, eps) == 0
    nit = C.c_int(-1)
    rc = o.L.bsg_parfbss_solve_symm(o.id, 1, C.byref(nit))
    assert rc == 0, o.L.bsg_last_error()
    x = np.empty(s.n)
    x[order] = o.solution()
    b = s.rhs[0]
    A = s.to_scipy()
    r = np.linalg.norm(b - A @ x)
    if eps > 0:
        assert r <= 1e-9 * np.linalg.norm(b)
    else:
        assert r <= abs(eps) * 1.001
    u = s.upper()
    xr, info = reflib.solve_symm(u.ia, u.ja, u.a, b, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=-1.0,
                                 ittype=0 if eps > 0 else 1, eps=abs(eps))
    err = np.linalg.norm(x - xr) / np.linalg.norm(xr)
    print(f"ParFBSS_SolveSymm eps={eps}: {nit.value} iterations (reference {info['iters']}), rel. error {err:.2e}")
    assert nit.value > 0 and err <= 1e-8
    ni, pl = C.c_int(), IP()
    assert o.L.bsg_parfbss_distribution(o.id, C.byref(ni), C.byref(pl)) == 0
    assert ni.value == s.n and np.array_equal(np.ctypeslib.as_array(pl, (s.n,)), order)
    o.destroy()


@pytest.mark.gpu
def test_solve_nonsymmetric_matches_reference(ctx, reflib):
    s = P.heat3d(9, 8, 7, sigma=1.0, seed=31)
    a = s.a.copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.ia))
    off = s.ja != rows
    a[off] *= 1.0 + 0.3 * np.sign(s.ja[off] - rows[off])
    order = np.random.default_rng(6).permutation(s.n)
    o = Obj(s.ia, s.ja, a, s.rhs[0], order, seed=7)
    assert o.L.bsg_parfbss_set_solver_parameters(o.id, 1, 1e-3, 1e-3, 0.1, 2000, 1e-10) == 0
    nit = C.c_int(-1)
    assert o.L.bsg_parfbss_solve(o.id, 1, C.byref(nit)) == 0, o.L.bsg_last_error()
    x = np.empty(s.n)
    x[order] = o.solution()
    xr, info = reflib.solver(s.ia, s.ja, a, s.rhs[0], tau1=1e-3, tau2=1e-3, sttype=1, eps=1e-10)
    err = np.linalg.norm(x - xr) / np.linalg.norm(xr)
    print(f"ParFBSS_Solve: {nit.value} iterations (reference Solver {info['iters']}), rel. error {err:.2e}")
    assert err <= 1e-8
    o.destroy()
