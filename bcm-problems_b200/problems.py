"""Seeded synthetic systems for the solver path (ctypes over libbsg_problems.so).

The generators are written in C++ (``csrc/problems.cpp``) so that every
consumer -- the GPU tests, the CPU oracles and the benchmark -- sees the
identical matrix and right-hand side for a given seed.
"""
import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PROBLEMS_SO = os.path.join(HERE, "libbsg_problems.so")

_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(PROBLEMS_SO):
            raise RuntimeError(f"{PROBLEMS_SO} is not built; run __graft_entry__.build()")
        L = C.CDLL(PROBLEMS_SO)
        vp = C.c_void_p
        for name, args in (("bsgp_heat3d", [C.c_int, C.c_int, C.c_int, C.c_double, C.c_ulonglong]),
                           ("bsgp_heat2d_batch", [C.c_int, C.c_int, C.c_int, C.c_double, C.c_ulonglong]),
                           ("bsgp_lame3d", [C.c_int, C.c_double, C.c_double, C.c_ulonglong]),
                           ("bsgp_lame_periodic", [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                                   C.c_double, C.c_ulonglong])):
            f = getattr(L, name)
            f.restype = vp
            f.argtypes = args
        for name, rt in (("bsgp_ia", C.POINTER(C.c_int)), ("bsgp_ja", C.POINTER(C.c_int)),
                         ("bsgp_a", C.POINTER(C.c_double)), ("bsgp_rhs", C.POINTER(C.c_double)),
                         ("bsgp_parts", C.POINTER(C.c_int))):
            f = getattr(L, name)
            f.restype = rt
            f.argtypes = [vp]
        L.bsgp_info.restype = C.c_double
        L.bsgp_info.argtypes = [vp, C.c_int]
        L.bsgp_sizes.argtypes = [vp] + [C.POINTER(C.c_int)] * 5
        L.bsgp_free.argtypes = [vp]
        _lib = L
    return _lib


@dataclass
class System:
    """A linear system in Bslib storage: CSR (bs == 1) or 3x3 block CSR with
    column-major blocks (bs == 3).  ``rhs`` has shape (nrhs, n*bs)."""
    n: int
    bs: int
    ia: np.ndarray
    ja: np.ndarray
    a: np.ndarray
    rhs: np.ndarray
    parts: np.ndarray
    info: dict = field(default_factory=dict)

    @property
    def nnz(self):
        return int(self.ia[-1])

    def upper(self):
        """Upper block triangle (diagonal first), the symmetric-solver input."""
        rows = np.repeat(np.arange(self.n, dtype=np.int32), np.diff(self.ia))
        keep = self.ja >= rows
        ia = np.zeros(self.n + 1, np.int32)
        np.cumsum(np.bincount(rows[keep], minlength=self.n), out=ia[1:])
        bs2 = self.bs * self.bs
        a = self.a.reshape(-1, bs2)[keep].reshape(-1)
        return System(self.n, self.bs, ia, self.ja[keep].copy(), a.copy(), self.rhs, self.parts, self.info)

    def to_point(self):
        """The same matrix as a point (bs == 1) CSR system: every entry of every
        block is kept (zeros included); point row bs*i + r holds columns
        bs*j + c of the blocks of block row i, sorted ascending."""
        if self.bs == 1:
            return self
        bs, n = self.bs, self.n
        nb = np.diff(self.ia).astype(np.int64)
        B = self.a.reshape(-1, bs, bs).transpose(0, 2, 1)  # [k, r, c]
        ia = np.zeros(n * bs + 1, np.int64)
        ia[1:] = np.cumsum(np.repeat(nb * bs, bs))
        rowb = np.repeat(np.arange(n), nb)
        k = np.arange(len(self.ja))[:, None, None]
        r = np.arange(bs)[None, :, None]
        c = np.arange(bs)[None, None, :]
        pos = ia[bs * rowb[k] + r] + (k - self.ia[rowb[k]]) * bs + c
        ja = np.empty(ia[-1], np.int32)
        a = np.empty(ia[-1])
        ja[pos] = bs * self.ja[k] + c
        a[pos] = B
        rows = np.repeat(np.arange(n * bs), np.diff(ia))
        order = np.lexsort((ja, rows))
        ja, a = ja[order], a[order]
        return System(n * bs, 1, ia.astype(np.int32), ja, a, self.rhs, self.parts * bs, self.info)

    def to_scipy(self):
        import scipy.sparse as sp
        if self.bs == 1:
            return sp.csr_matrix((self.a, self.ja, self.ia), shape=(self.n, self.n))
        blocks = self.a.reshape(-1, self.bs, self.bs).transpose(0, 2, 1)  # column-major -> row-major
        return sp.bsr_matrix((blocks, self.ja, self.ia), shape=(self.n * self.bs, self.n * self.bs)).tocsr()


def _wrap(h):
    L = _load()
    if not h:
        raise MemoryError("problem generation failed")
    try:
        n, bs, nnz, nrhs, nparts = (C.c_int() for _ in range(5))
        L.bsgp_sizes(h, C.byref(n), C.byref(bs), C.byref(nnz), C.byref(nrhs), C.byref(nparts))
        n, bs, nnz, nrhs, nparts = n.value, bs.value, nnz.value, nrhs.value, nparts.value
        ia = np.ctypeslib.as_array(L.bsgp_ia(h), (n + 1,)).copy()
        ja = np.ctypeslib.as_array(L.bsgp_ja(h), (nnz,)).copy()
        a = np.ctypeslib.as_array(L.bsgp_a(h), (nnz * bs * bs,)).copy()
        rhs = np.ctypeslib.as_array(L.bsgp_rhs(h), (nrhs * n * bs,)).copy().reshape(nrhs, n * bs)
        parts = np.ctypeslib.as_array(L.bsgp_parts(h), (nparts + 1,)).copy()
        info = {"frac": L.bsgp_info(h, 0), "count": L.bsgp_info(h, 1)}
    finally:
        L.bsgp_free(h)
    return System(n, bs, ia, ja, a, rhs, parts, info)


def heat3d(nx, ny=None, nz=None, sigma=0.0, seed=0):
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    return _wrap(_load().bsgp_heat3d(nx, ny, nz, sigma, seed))


def heat2d_batch(nprob=256, smin=32, smax=256, sigma=1.0, seed=3):
    return _wrap(_load().bsgp_heat2d_batch(nprob, smin, smax, sigma, seed))


def lame3d(nn=64, nu=0.3, sigma=1.0, seed=1):
    return _wrap(_load().bsgp_lame3d(nn, nu, sigma, seed))


def lame_periodic(nn=48, nu=0.3, rmin=4.0, rmax=8.0, volfrac=0.3, contrast=100.0, seed=2):
    return _wrap(_load().bsgp_lame_periodic(nn, nu, rmin, rmax, volfrac, contrast, seed))


# The five benchmark workloads (full size).
def config(k):
    if k == 1:
        return heat3d(32, sigma=0.0, seed=0)
    if k == 2:
        return lame3d(64, 0.3, 1.0, 1)
    if k == 3:
        return lame_periodic(48, 0.3, 4.0, 8.0, 0.3, 100.0, 2)
    if k == 4:
        return heat2d_batch(256, 32, 256, 1.0, 3)
    if k == 5:
        return heat3d(128, sigma=1.5, seed=4)
    raise ValueError(k)
