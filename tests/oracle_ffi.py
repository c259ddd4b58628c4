"""ctypes access to the two CPU checkers (test infrastructure only).

* ``Oracle`` -- the C restatement in ``oracle/bsl_oracle.c`` (``oracle/_build``).
* ``RefLib`` -- the reference Bslib compiled from its own sources into
  ``oracle/_ref/libbslib_ref.so`` by ``oracle/Makefile``.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use this module; the product never imports it.
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libbslib_ref.so")

_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


def _i(x):
    return np.ascontiguousarray(x, dtype=np.int32).ctypes.data_as(_ip)


def _d(x):
    return np.ascontiguousarray(x, dtype=np.float64).ctypes.data_as(_dp)


def _take_csr(lib, n, pia, pja, pa, pb=None):
    ia = np.ctypeslib.as_array(pia, (n + 1,)).copy()
    nz = int(ia[-1])
    ja = np.ctypeslib.as_array(pja, (max(nz, 1),))[:nz].copy()
    a = np.ctypeslib.as_array(pa, (max(nz, 1),))[:nz].copy()
    b = None
    if pb is not None:
        b = np.ctypeslib.as_array(pb, (max(nz, 1),))[:nz].copy()
    return ia, ja, a, b


def _take_bsr(nb, bs, pia, pja, *pvals):
    """Block CSR arrays handed back by the C side (malloc'ed): copies."""
    ia = np.ctypeslib.as_array(pia, (nb + 1,)).copy()
    nz = int(ia[-1])
    ja = np.ctypeslib.as_array(pja, (max(nz, 1),))[:nz].copy()
    vals = [np.ctypeslib.as_array(p, (max(nz, 1) * bs * bs,))[:nz * bs * bs].copy() for p in pvals]
    return ia, ja, vals


class Oracle:
    def __init__(self, path=ORACLE_SO):
        self.lib = C.CDLL(path)
        L = self.lib
        L.orc_fact.restype = C.c_int
        L.orc_combine_lu.restype = C.c_int
        L.orc_pcg.restype = C.c_int
        L.orc_gmres.restype = C.c_int

    def mvm(self, ia, ja, a, x, symm=False):
        n = len(ia) - 1
        y = np.zeros(n)
        f = self.lib.orc_mvm_symm if symm else self.lib.orc_mvm
        f(n, _i(ia), _i(ja), _d(a), _d(x), _d(y))
        return y

    def bsr_mvm(self, ia, ja, a, x, bs):
        nb = len(ia) - 1
        y = np.zeros(nb * bs)
        self.lib.orc_bsr_mvm(nb, bs, _i(ia), _i(ja), _d(a), _d(x), _d(y))
        return y

    def solve_l(self, iu, ju, u, x):
        n = len(iu) - 1
        y = np.zeros(n)
        self.lib.orc_solve_l(n, _i(iu), _i(ju), _d(u), _d(x), _d(y))
        return y

    def solve_u(self, iu, ju, u, x):
        n = len(iu) - 1
        y = np.zeros(n)
        self.lib.orc_solve_u(n, _i(iu), _i(ju), _d(u), _d(x), _d(y))
        return y

    def combine_lu(self, ia, ja, a):
        n = len(ia) - 1
        pia, pja, pl, pu = _ip(), _ip(), _dp(), _dp()
        ia, ja, a = [np.ascontiguousarray(v) for v in (ia, ja, a)]
        rc = self.lib.orc_combine_lu(n, _i(ia), _i(ja), _d(a), C.byref(pia), C.byref(pja), C.byref(pl), C.byref(pu))
        if rc < 0:
            raise ValueError("combine_lu failed")
        sia, sja, al, au = _take_csr(self.lib, n, pia, pja, pl, pu)
        for p in (pia, pja, pl, pu):
            self.lib.orc_free(p)
        return sia, sja, al, au

    def fact(self, kind, ia, ja, al, au=None, tau1=1e-3, tau2=1e-3, theta=0.1, sclmin=1e-8, pivmin=1e-8):
        n = len(ia) - 1
        if au is None:
            au = al
        piu, pju, pl, pu = _ip(), _ip(), _dp(), _dp()
        st = (C.c_double * 4)()
        keep = [np.ascontiguousarray(v) for v in (ia, ja, al, au)]
        rc = self.lib.orc_fact(kind, n, _i(keep[0]), _i(keep[1]), _d(keep[2]), _d(keep[3]), C.c_double(tau1),
                               C.c_double(tau2), C.c_double(theta), C.c_double(sclmin), C.c_double(pivmin),
                               C.byref(piu), C.byref(pju), C.byref(pl), C.byref(pu), st)
        if rc == -2:
            raise ArithmeticError(f"Ich2: Diagonal pivot is nonpositive (row {int(st[2])})")
        if rc != 0:
            raise RuntimeError(f"orc_fact failed rc={rc}")
        iu, ju, lv, uv = _take_csr(self.lib, n, piu, pju, pl, pu if kind == 1 else None)
        self.lib.orc_free(piu)
        self.lib.orc_free(pju)
        self.lib.orc_free(pl)
        if kind == 1:
            self.lib.orc_free(pu)
        else:
            uv = lv
        return iu, ju, lv, uv, (st[0], st[1])

    def ich0(self, ia, ja, a):
        """IC(0) (CSMatrixR::Ich) of an upper-stored matrix: (iu, ju, u)."""
        n = len(ia) - 1
        piu, pju, pu = _ip(), _ip(), _dp()
        keep = [np.ascontiguousarray(v) for v in (ia, ja, a)]
        if self.lib.orc_ich0(n, _i(keep[0]), _i(keep[1]), _d(keep[2]), C.byref(piu), C.byref(pju), C.byref(pu)) != 0:
            raise RuntimeError("orc_ich0 failed")
        iu, ju, u, _ = _take_csr(self.lib, n, piu, pju, pu)
        for p in (piu, pju, pu):
            self.lib.orc_free(p)
        return iu, ju, u

    def pcg(self, ia, ja, a, iu, ju, u, b, ittype=0, eps=1e-10, niter=1000):
        n = len(ia) - 1
        x = np.zeros(n)
        res = C.c_double()
        it = self.lib.orc_pcg(n, _i(ia), _i(ja), _d(a), _i(iu), _i(ju), _d(u), _d(b), _d(x), ittype,
                              C.c_double(eps), niter, C.byref(res))
        return x, it, res.value

    def gmres(self, ia, ja, a, iu, ju, l, u, b, m=50, eps=1e-8, sttype=1, niter=2000):
        n = len(ia) - 1
        x = np.zeros(n)
        res = C.c_double()
        it = self.lib.orc_gmres(n, _i(ia), _i(ja), _d(a), _i(iu), _i(ju), _d(l), _d(u), _d(b), _d(x), m,
                                C.c_double(eps), sttype, niter, C.byref(res))
        return x, it, res.value


    def lanczos(self, ia, ja, a, iu, ju, l, u, b, eps=1e-8, sttype=1, niter=2000):
        n = len(ia) - 1
        x = np.zeros(n)
        em = C.c_double()
        it = self.lib.orc_lanczos(n, _i(ia), _i(ja), _d(a), _i(iu), _i(ju), _d(l), _d(u), _d(b), _d(x),
                                  C.c_double(eps), sttype, niter, C.byref(em))
        return x, it, em.value


    # ---- block (CSMatrixRS) part ----
    def combine_lu_block(self, ia, ja, a, bs):
        nb = len(ia) - 1
        pia, pja, pl, pu = _ip(), _ip(), _dp(), _dp()
        if self.lib.orc_combine_lu_block(nb, bs, _i(ia), _i(ja), _d(a), C.byref(pia), C.byref(pja), C.byref(pl),
                                         C.byref(pu)) != 0:
            raise MemoryError("combine_lu_block")
        ia_s, ja_s, (al, au) = _take_bsr(nb, bs, pia, pja, pl, pu)
        for p in (pia, pja, pl, pu):
            self.lib.orc_free(p)
        return ia_s, ja_s, al, au

    def ilu2_block(self, ia_s, ja_s, al, au, bs, tau1=1e-3, tau2=1e-3, theta=0.1, sclmin=1e-8, pivmin=1e-8,
                   jacobi_svd=False):
        """Block ILU2 of a CombineLU'd block matrix: (ia, ja, l, u, (density, density2)).
        jacobi_svd: the GPU path's one-sided Jacobi SVD instead of LAPACK's dgesvd."""
        nb = len(ia_s) - 1
        pia, pja, pl, pu = _ip(), _ip(), _dp(), _dp()
        st = (C.c_double * 3)()
        f = self.lib.orc_ilu2_block_jacobi if jacobi_svd else self.lib.orc_ilu2_block
        rc = f(nb, bs, _i(ia_s), _i(ja_s), _d(al), _d(au), C.c_double(tau1), C.c_double(tau2),
                                     C.c_double(theta), C.c_double(sclmin), C.c_double(pivmin), C.byref(pia),
                                     C.byref(pja), C.byref(pl), C.byref(pu), st)
        if rc != 0:
            raise RuntimeError(f"orc_ilu2_block failed ({rc})")
        ia_f, ja_f, (l, u) = _take_bsr(nb, bs, pia, pja, pl, pu)
        for p in (pia, pja, pl, pu):
            self.lib.orc_free(p)
        return ia_f, ja_f, l, u, (st[0], st[1])

    def ich2_block(self, ia, ja, a, bs, tau1=1e-3, tau2=1e-3, theta=0.1, jacobi_eig=False):
        """Block IC2 of an upper-stored symmetric block matrix: (ia, ja, u, (density, density2)).
        jacobi_eig: the GPU path's Jacobi eigenpairs instead of LAPACK's dsyev."""
        nb = len(ia) - 1
        pia, pja, pu = _ip(), _ip(), _dp()
        st = (C.c_double * 3)()
        f = self.lib.orc_ich2_block_jacobi if jacobi_eig else self.lib.orc_ich2_block
        rc = f(nb, bs, _i(ia), _i(ja), _d(a), C.c_double(tau1), C.c_double(tau2),
                                     C.c_double(theta), C.byref(pia), C.byref(pja), C.byref(pu), st)
        if rc == -2:
            raise ArithmeticError("negative pivot in block IC2")
        if rc != 0:
            raise RuntimeError(f"orc_ich2_block failed ({rc})")
        ia_f, ja_f, (u,) = _take_bsr(nb, bs, pia, pja, pu)
        for p in (pia, pja, pu):
            self.lib.orc_free(p)
        return ia_f, ja_f, u, (st[0], st[1])

    def solve_l_block(self, ia, ja, a, bs, x):
        nb = len(ia) - 1
        y = np.zeros(nb * bs)
        self.lib.orc_solve_l_block(nb, bs, _i(ia), _i(ja), _d(a), _d(x), _d(y))
        return y

    def solve_u_block(self, ia, ja, a, bs, x):
        nb = len(ia) - 1
        y = np.zeros(nb * bs)
        self.lib.orc_solve_u_block(nb, bs, _i(ia), _i(ja), _d(a), _d(x), _d(y))
        return y


class RefLib:
    """The reference Bslib, compiled here from its sources (oracle/Makefile)."""

    def __init__(self, path=REF_SO):
        self.lib = C.CDLL(path)
        self.lib.ref_last_error.restype = C.c_char_p

    def _err(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def mvm(self, ia, ja, a, x, symm=False):
        n = len(ia) - 1
        y = np.zeros(n)
        self._err(self.lib.ref_mvm(n, _i(ia), _i(ja), _d(a), _d(x), _d(y), int(symm)))
        return y

    def solve_l(self, iu, ju, u, x):
        n = len(iu) - 1
        y = np.zeros(n)
        self._err(self.lib.ref_solve_l(n, _i(iu), _i(ju), _d(u), _d(x), _d(y)))
        return y

    def solve_u(self, iu, ju, u, x):
        n = len(iu) - 1
        y = np.zeros(n)
        self._err(self.lib.ref_solve_u(n, _i(iu), _i(ju), _d(u), _d(x), _d(y)))
        return y

    def ich0(self, ia, ja, a):
        """CSMatrixR::Ich (IC(0)) of an upper-stored matrix: (iu, ju, u)."""
        n = len(ia) - 1
        piu, pju, pu = _ip(), _ip(), _dp()
        self._err(self.lib.ref_ich0(n, _i(ia), _i(ja), _d(a), C.byref(piu), C.byref(pju), C.byref(pu)))
        iu, ju, u, _ = _take_csr(self.lib, n, piu, pju, pu)
        for p in (piu, pju, pu):
            self.lib.ref_free(p)
        return iu, ju, u

    def ich2(self, ia, ja, a, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0):
        n = len(ia) - 1
        piu, pju, pu = _ip(), _ip(), _dp()
        st = (C.c_double * 3)()
        self._err(self.lib.ref_ich2(n, _i(ia), _i(ja), _d(a), C.c_double(tau1), C.c_double(tau2),
                                    C.c_double(theta), C.c_double(memory), C.byref(piu), C.byref(pju),
                                    C.byref(pu), st))
        iu, ju, u, _ = _take_csr(self.lib, n, piu, pju, pu)
        for p in (piu, pju, pu):
            self.lib.ref_free(p)
        return iu, ju, u, (st[0], st[1], st[2])

    def ilu2(self, ia, ja, a, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, sclmin=1e-8, pivmin=1e-8):
        n = len(ia) - 1
        pil, pjl, pl, piu, pju, pu = _ip(), _ip(), _dp(), _ip(), _ip(), _dp()
        st = (C.c_double * 3)()
        self._err(self.lib.ref_ilu2(n, _i(ia), _i(ja), _d(a), C.c_double(tau1), C.c_double(tau2),
                                    C.c_double(theta), C.c_double(memory), C.c_double(sclmin), C.c_double(pivmin),
                                    C.byref(pil), C.byref(pjl), C.byref(pl), C.byref(piu), C.byref(pju),
                                    C.byref(pu), st))
        il, jl, lv, _ = _take_csr(self.lib, n, pil, pjl, pl)
        iu, ju, uv, _ = _take_csr(self.lib, n, piu, pju, pu)
        for p in (pil, pjl, pl, piu, pju, pu):
            self.lib.ref_free(p)
        return (il, jl, lv), (iu, ju, uv), (st[0], st[1], st[2])

    def solve_symm(self, ia, ja, a, b, fcttyp=2, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, ittype=0,
                   eps=1e-10, niter=1000, ichk=1):
        n = len(ia) - 1
        x = np.zeros(n)
        st = (C.c_double * 8)()
        self._err(self.lib.ref_solve_symm(n, _i(ia), _i(ja), _d(a), _d(b), _d(x), fcttyp, C.c_double(tau1),
                                          C.c_double(tau2), C.c_double(theta), C.c_double(memory), ittype,
                                          C.c_double(eps), niter, ichk, st))
        return x, dict(iters=int(st[0]), resfin=st[1], tfct=st[2], titr=st[3], density=st[4], density2=st[5],
                       wall=st[6])

    def cg(self, ia, ja, a, iu, ju, u, b, ittype=0, eps=1e-10, niter=1000, ichk=1):
        n = len(ia) - 1
        x = np.zeros(n)
        st = (C.c_double * 3)()
        self._err(self.lib.ref_cg(n, _i(ia), _i(ja), _d(a), _i(iu), _i(ju), _d(u), _d(b), _d(x), ittype,
                                  C.c_double(eps), niter, ichk, st))
        return x, dict(iters=int(st[0]), resfin=st[1], wall=st[2])

    def solver(self, ia, ja, a, b, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, sclmin=1e-8, pivmin=1e-8,
               sttype=1, eps=1e-8, niter=1000, ichk=1):
        n = len(ia) - 1
        x = np.zeros(n)
        st = (C.c_double * 8)()
        self._err(self.lib.ref_solver(n, _i(ia), _i(ja), _d(a), _d(b), _d(x), C.c_double(tau1), C.c_double(tau2),
                                      C.c_double(theta), C.c_double(memory), C.c_double(sclmin),
                                      C.c_double(pivmin), sttype, C.c_double(eps), niter, ichk, st))
        return x, dict(iters=int(st[0]), resfin=st[1], tfct=st[2], titr=st[3], density=st[4], density2=st[5],
                       wall=st[6])

    # ---- block (CSMatrixRS) part ----
    def combine_lu_block(self, ia, ja, a, bs):
        nb = len(ia) - 1
        pia, pja, pl, pu = _ip(), _ip(), _dp(), _dp()
        self._err(self.lib.ref_combine_lu_block(nb, bs, _i(ia), _i(ja), _d(a), C.byref(pia), C.byref(pja),
                                                C.byref(pl), C.byref(pu)))
        ia_s, ja_s, (al, au) = _take_bsr(nb, bs, pia, pja, pl, pu)
        for p in (pia, pja, pl, pu):
            self.lib.ref_free(p)
        return ia_s, ja_s, al, au

    def ilu2_block(self, ia, ja, a, bs, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, sclmin=1e-8, pivmin=1e-8):
        """CombineLU + CSMatrixRS::Ilu2: (ia, ja, l, u, (density, density2, seconds))."""
        nb = len(ia) - 1
        pia, pja, pl, pu = _ip(), _ip(), _dp(), _dp()
        st = (C.c_double * 3)()
        self._err(self.lib.ref_ilu2_block(nb, bs, _i(ia), _i(ja), _d(a), C.c_double(tau1), C.c_double(tau2),
                                          C.c_double(theta), C.c_double(memory), C.c_double(sclmin),
                                          C.c_double(pivmin), C.byref(pia), C.byref(pja), C.byref(pl),
                                          C.byref(pu), st))
        ia_f, ja_f, (l, u) = _take_bsr(nb, bs, pia, pja, pl, pu)
        for p in (pia, pja, pl, pu):
            self.lib.ref_free(p)
        return ia_f, ja_f, l, u, (st[0], st[1], st[2])

    def solve_l_block(self, ia, ja, a, bs, x):
        nb = len(ia) - 1
        y = np.zeros(nb * bs)
        self._err(self.lib.ref_solve_l_block(nb, bs, _i(ia), _i(ja), _d(a), _d(x), _d(y)))
        return y

    def solve_u_block(self, ia, ja, a, bs, x):
        nb = len(ia) - 1
        y = np.zeros(nb * bs)
        self._err(self.lib.ref_solve_u_block(nb, bs, _i(ia), _i(ja), _d(a), _d(x), _d(y)))
        return y

    def ich2_block(self, ia, ja, a, bs, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0):
        """CSMatrixRS::Ich2 of an upper-stored block matrix: (ia, ja, u, (density, density2, seconds))."""
        nb = len(ia) - 1
        pia, pja, pu = _ip(), _ip(), _dp()
        st = (C.c_double * 3)()
        self._err(self.lib.ref_ich2_block(nb, bs, _i(ia), _i(ja), _d(a), C.c_double(tau1), C.c_double(tau2),
                                          C.c_double(theta), C.c_double(memory), C.byref(pia), C.byref(pja),
                                          C.byref(pu), st))
        ia_f, ja_f, (u,) = _take_bsr(nb, bs, pia, pja, pu)
        for p in (pia, pja, pu):
            self.lib.ref_free(p)
        return ia_f, ja_f, u, (st[0], st[1], st[2])

    def solve_symm_block(self, ia, ja, a, bs, B, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, ittype=0, eps=1e-8,
                         niter=1000):
        """CSVector::SolveSymm(CSMatrixRS&) (block IC2 + PCG) for each row of B
        (load cases), x0 = 0: (X, [dict(iters, resfin, wall, density)])."""
        nb = len(ia) - 1
        B = np.ascontiguousarray(np.atleast_2d(B), dtype=np.float64)
        nrhs = B.shape[0]
        X = np.zeros_like(B)
        st = (C.c_double * (4 * nrhs))()
        self._err(self.lib.ref_solve_symm_block(nb, bs, _i(ia), _i(ja), _d(a), nrhs, _d(B), _d(X),
                                                C.c_double(tau1), C.c_double(tau2), C.c_double(theta),
                                                C.c_double(memory), ittype, C.c_double(eps), niter, st))
        info = [dict(iters=int(st[4 * k]), resfin=st[4 * k + 1], wall=st[4 * k + 2], density=st[4 * k + 3])
                for k in range(nrhs)]
        return X, info

    # ---- generator behind the abstract-interface callbacks (oracle/ref/abstract_gen.cpp) ----
    def gen_create(self, sprnd, ia, ja, a, b, x0, seed=1):
        """A generator serving block CSR (blocks column-major, sizes from
        sprnd) through Bslib's seven callbacks, each block row's blocks in a
        shuffled order.  Returns an opaque handle (free with gen_free)."""
        self.lib.ref_gen_create.restype = C.c_void_p
        self._gen_keep = [np.ascontiguousarray(v, dt) for v, dt in
                          ((sprnd, np.int32), (ia, np.int32), (ja, np.int32), (a, np.float64), (b, np.float64),
                           (x0, np.float64))]
        sp_, ia_, ja_, a_, b_, x_ = self._gen_keep
        h = self.lib.ref_gen_create(len(ia_) - 1, _i(sp_), _i(ia_), _i(ja_), _d(a_), _d(b_), _d(x_),
                                    C.c_uint(seed))
        return C.c_void_p(h)

    def gen_free(self, h):
        self.lib.ref_gen_free(h)

    def gen_solution(self, h, n):
        x = np.zeros(n)
        self.lib.ref_gen_solution(h, _d(x))
        return x

    def gen_calls(self, h):
        c = np.zeros(7, np.int32)
        self.lib.ref_gen_calls(h, _i(c))
        return c

    def gen_fns(self):
        fns = (C.c_void_p * 7)()
        self.lib.ref_gen_fns(fns)
        return fns

    def abstract(self, symm, h, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0, ittype=0, sttype=1, eps=1e-10,
                 niter=3000):
        """The reference's AbstractSymmSolver (symm) / AbstractSolver on generator h."""
        out = (C.c_double * 4)()
        rc = self.lib.ref_abstract(int(symm), h, C.c_double(tau1), C.c_double(tau2), C.c_double(theta),
                                   C.c_double(memory), ittype, sttype, C.c_double(eps), niter, out)
        if rc != 0:
            self.lib.ref_abstract_error.restype = C.c_char_p
            raise RuntimeError(self.lib.ref_abstract_error().decode())
        return dict(iters=int(out[0]), resfin=out[1], density=out[2], wall=out[3])

    # ---- the reference's own file readers / writers ----
    def write_system_bin(self, path, ia, ja, a, vecs=()):
        """CSMatrixR::WriteMtrBin, then CSVector::WriteVectBin per vector."""
        n = len(ia) - 1
        pb = os.fsencode(path)
        self._err(self.lib.ref_write_mtr_bin(pb, n, _i(ia), _i(ja), _d(a)))
        for v in vecs:
            self._err(self.lib.ref_write_vect_bin(pb, 1, len(v), _d(v)))

    def read_system_bin(self, path, nvec, n):
        """CSMatrixR::ReadMtrBin then nvec CSVector::ReadVectBin: (ia, ja, a, vecs)."""
        pia, pja, pa = _ip(), _ip(), _dp()
        nn = C.c_int()
        vecs = np.zeros(max(nvec * n, 1))
        self._err(self.lib.ref_read_system_bin(os.fsencode(path), nvec, C.byref(nn), C.byref(pia), C.byref(pja),
                                               C.byref(pa), _d(vecs)))
        ia, ja, a, _ = _take_csr(self.lib, nn.value, pia, pja, pa)
        for p in (pia, pja, pa):
            self.lib.ref_free(p)
        return ia, ja, a, [vecs[k * n:(k + 1) * n].copy() for k in range(nvec)]

    def convert_to_binary(self, text_path, bin_path):
        """CSMatrixR::ConvertToBinary (text matrix + rhs + norm -> binary), run
        as the separate program oracle/_ref/ref_convert (the reference's text
        streams crash inside a Python process)."""
        import subprocess
        tool = os.path.join(os.path.dirname(REF_SO), "ref_convert")
        r = subprocess.run([tool, text_path, bin_path], capture_output=True, text=True, timeout=120)
        if r.returncode != 0:
            raise RuntimeError(f"ref_convert failed: {r.stderr.strip()}")

    def _krylov_tree(self, fn, n, b, x0, op, *args):
        x = np.array(x0, dtype=np.float64, copy=True)
        st = (C.c_double * 2)()
        rc = fn(n, _d(b), x.ctypes.data_as(_dp), op.h, C.c_void_p(op.fns[0]), op.h, C.c_void_p(op.fns[1]), *args, st)
        if rc != 0:
            self.lib.ref_abstract_error.restype = C.c_char_p
            raise RuntimeError(self.lib.ref_abstract_error().decode())
        return x, dict(iters=int(st[0]), wall=st[1])

    def cg_tree(self, n, b, x0, op, sttype=1, eps=1e-10, niter=1000):
        """The reference's callback CSVector::Cg on a one-processor CTree, with
        the matrix / preconditioner operators of `op` (.h object, .fns[0..1]
        CMVM / CSOLVELU pointers); it stops on sttype (0 absolute, 1 relative)."""
        return self._krylov_tree(self.lib.ref_cg_tree, n, b, x0, op, sttype, C.c_double(eps), niter)

    def gmres_tree(self, n, b, x0, op, sttype=1, eps=1e-10, niter=300):
        """The reference's callback CSVector::BlockGMRES on a one-processor CTree."""
        return self._krylov_tree(self.lib.ref_gmres_tree, n, b, x0, op, sttype, C.c_double(eps), niter)

    def block_lanczos(self, ia, ja, a, bs, ittype, B, tau1=1e-3, tau2=1e-3, theta=0.1, eps=1e-8, niter=1000, ichk=1):
        """CombineLU + block ILU2 + CSVector::BlockLanczos{Central,Right,Left}
        (ittype 2 / 3 / 4) on the columns of B (rows of the array), x0 = 0."""
        nb = len(ia) - 1
        B = np.ascontiguousarray(np.atleast_2d(B), dtype=np.float64)
        X = np.zeros_like(B)
        st = (C.c_double * 1)()
        self._err(self.lib.ref_block_lanczos(nb, bs, _i(ia), _i(ja), _d(a), ittype, B.shape[0], _d(B), _d(X),
                                             C.c_double(tau1), C.c_double(tau2), C.c_double(theta),
                                             C.c_double(eps), niter, ichk, st))
        return X
