"""Python binding of libbsg.so, the B200 solver library (C ABI in include/bslib_gpu.h).

This module is a thin ctypes layer: PyTorch provides device buffers and the
CUDA stream, every computation runs in the library's own sm_100a kernels.
There is no CPU fallback -- if the library or a GPU is missing, the calls
raise.

Naming follows Bslib: ``Matrix`` is a device CSMatrixR / CSMatrixRS,
``Factor`` an IC2 / ILU2 factor, ``Param`` the CSlvParam fields of the path.
"""
import ctypes as C
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_SO = os.path.join(HERE, "libbsg.so")

OK = 0
ERR_ARG, ERR_PIVOT, ERR_WORKSPACE, ERR_BREAKDOWN, ERR_CUDA, ERR_TIMEOUT, ERR_NOCONV, ERR_UNSUPPORTED, ERR_NOMEM = \
    -1, -2, -3, -4, -5, -6, -7, -8, -9


class BsgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Param(C.Structure):
    """Mirror of ``bsg_param`` (CSlvParam fields of the path + GPU extensions)."""
    _fields_ = [
        ("msglev", C.c_int), ("fcttyp", C.c_int), ("ordtype", C.c_int), ("memory", C.c_double),
        ("tau1", C.c_double), ("tau2", C.c_double), ("theta", C.c_double), ("sclmin", C.c_double),
        ("pivmin", C.c_double), ("ittype", C.c_int), ("sttype", C.c_int), ("niter", C.c_int),
        ("eps", C.c_double), ("ichk", C.c_int), ("nitperf", C.c_int), ("resfin", C.c_double),
        ("density", C.c_double), ("density2", C.c_double), ("timefct", C.c_double), ("timeitr", C.c_double),
        ("precision", C.c_int), ("trisolve", C.c_int), ("nsweeps", C.c_int), ("krylov", C.c_int),
        ("restart", C.c_int), ("true_residual", C.c_int), ("learned", C.c_void_p), ("resrec", C.c_double),
        ("blockfct", C.c_int), ("pad", C.c_int * 3),
    ]


_lib = None


def lib():
    """Load libbsg.so (raises when it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_SO):
        raise RuntimeError(f"{LIB_SO} is not built; run __graft_entry__.build()")
    L = C.CDLL(LIB_SO)
    vp, ip, dp, i_ = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int
    pp = C.POINTER(C.c_void_p)
    sig = {
        "bsg_param_default": (None, [C.POINTER(Param)]),
        "bsg_last_error": (C.c_char_p, []),
        "bsg_version": (C.c_char_p, []),
        "bsg_create": (i_, [pp, i_, vp]),
        "bsg_destroy": (i_, [vp]),
        "bsg_sync": (i_, [vp]),
        "bsg_mat_csr": (i_, [vp, i_, ip, ip, dp, i_, pp]),
        "bsg_mat_csr_dev": (i_, [vp, i_, vp, vp, vp, i_, pp]),
        "bsg_mat_bsr": (i_, [vp, i_, i_, ip, ip, dp, i_, pp]),
        "bsg_mat_free": (i_, [vp]),
        "bsg_mat_info": (i_, [vp, ip, ip, ip]),
        "bsg_mvm_dev": (i_, [vp, vp, vp, vp]),
        "bsg_mvm": (i_, [vp, vp, dp, dp]),
        "bsg_mvm_multi_dev": (i_, [vp, vp, i_, vp, vp]),
        "bsg_fct_ich2": (i_, [vp, vp, C.POINTER(Param), pp]),
        "bsg_fct_ilu2": (i_, [vp, vp, C.POINTER(Param), pp]),
        "bsg_fct_to_fp32": (i_, [vp]),
        "bsg_fct_export": (i_, [vp, ip, ip, ip, dp, dp]),
        "bsg_fct_info": (i_, [vp, ip, ip, ip, ip, dp, dp]),
        "bsg_fct_free": (i_, [vp]),
        "bsg_solve_l_dev": (i_, [vp, vp, i_, i_, vp, vp]),
        "bsg_solve_u_dev": (i_, [vp, vp, i_, i_, vp, vp]),
        "bsg_pcg_dev": (i_, [vp, vp, vp, vp, vp, C.POINTER(Param)]),
        "bsg_gmres_dev": (i_, [vp, vp, vp, vp, vp, C.POINTER(Param)]),
        "bsg_solve_symm_csr": (i_, [vp, i_, ip, ip, dp, dp, dp, C.POINTER(Param)]),
        "bsg_solver_csr": (i_, [vp, i_, ip, ip, dp, dp, dp, C.POINTER(Param)]),
        "bsg_fact_stats": (i_, [C.POINTER(C.c_ulonglong), i_]),
        "bsg_unet_create": (i_, [vp, i_, i_, i_, i_, pp]),
        "bsg_unet_free": (i_, [vp]),
        "bsg_unet_nparam": (i_, [vp]),
        "bsg_unet_set_weights": (i_, [vp, C.POINTER(C.c_float)]),
        "bsg_unet_get_weights": (i_, [vp, C.POINTER(C.c_float)]),
        "bsg_unet_get_grads": (i_, [vp, C.POINTER(C.c_float)]),
        "bsg_unet_set_matrix": (i_, [vp, vp]),
        "bsg_unet_set_diag": (i_, [vp, vp]),
        "bsg_unet_forward_dev": (i_, [vp, vp, vp]),
        "bsg_unet_train_sample": (i_, [vp, vp, vp, C.POINTER(C.c_double)]),
        "bsg_unet_adam": (i_, [vp, C.c_float, C.c_float, C.c_float, C.c_float, i_]),
        "bsg_unet_zero_grads": (i_, [vp]),
        "bsg_launch_count": (C.c_ulonglong, []),
        "bsg_pcg_batch_dev": (i_, [vp, vp, vp, i_, i_, ip, vp, vp, C.POINTER(Param), ip, dp, ip]),
        "bsg_lanczos_dev": (i_, [vp, vp, vp, vp, vp, C.POINTER(Param)]),
        "bsg_solve_t_dev": (i_, [vp, vp, i_, i_, i_, vp, vp]),
        "bsg_sell_stats": (i_, [vp, vp, C.POINTER(C.c_longlong)]),
        "bsg_solve_multi_dev": (i_, [vp, vp, i_, i_, i_, i_, vp, vp]),
        "bsg_fct_export_block": (i_, [vp, ip, ip, ip, ip, dp, dp]),
        "bsg_mat_vbsr": (i_, [vp, i_, ip, ip, ip, dp, i_, pp]),
        "bsg_read_mtr_bin": (i_, [C.c_char_p, C.POINTER(C.c_longlong), ip, ip, ip, ip, ip, ip, ip, dp]),
        "bsg_write_mtr_bin": (i_, [C.c_char_p, i_, i_, i_, i_, ip, ip, ip, dp]),
        "bsg_read_mtr": (i_, [C.c_char_p, C.POINTER(C.c_longlong), ip, ip, ip, ip, dp]),
        "bsg_read_vect": (i_, [C.c_char_p, C.POINTER(C.c_longlong), i_, dp]),
        "bsg_write_vect_bin": (i_, [C.c_char_p, i_, i_, i_, i_, dp, ip, ip]),
        "bsg_read_vect_bin": (i_, [C.c_char_p, C.POINTER(C.c_longlong), ip, ip, ip, dp, ip, ip]),
        "bsg_solve": (i_, [vp, vp, vp, dp, dp, C.POINTER(Param)]),
        "bsg_solve_lu": (i_, [vp, vp, i_, i_, i_, dp, dp]),
        "bsg_set_spin_limit_ns": (i_, [vp, C.c_ulonglong]),
        "bsg_block_lanczos_dev": (i_, [vp, vp, vp, i_, i_, vp, vp, C.POINTER(Param), dp]),
    }
    for name, (rt, at) in sig.items():
        f = getattr(L, name)
        f.restype = rt
        f.argtypes = at
    _lib = L
    return L


def _check(rc):
    if rc != OK:
        raise BsgError(rc, lib().bsg_last_error().decode(errors="replace"))


def _ip(a):
    return np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(C.POINTER(C.c_int))


def _dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def default_param(**kw):
    p = Param()
    lib().bsg_param_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def _ptr(t):
    """Device pointer of a contiguous CUDA tensor."""
    import torch
    assert isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


class Context:
    """A device + stream.  By default it runs on PyTorch's current stream, so
    library kernels are ordered with the tensors the caller hands in."""

    def __init__(self, device=0, stream=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("bsg needs a CUDA device (no CPU fallback)")
        torch.cuda.set_device(device)
        if stream is None:
            stream = torch.cuda.current_stream(device).cuda_stream
        self.h = C.c_void_p()
        _check(lib().bsg_create(C.byref(self.h), device, C.c_void_p(stream)))
        self.device = device
        self._children = weakref.WeakSet()

    def _adopt(self, obj):
        self._children.add(obj)

    def sync(self):
        _check(lib().bsg_sync(self.h))

    def close(self):
        """Free every matrix / factor still alive on this context, then the context."""
        if self.h:
            for obj in list(self._children):
                obj.free()
            lib().bsg_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Matrix:
    """Device copy of a CSMatrixR (bs == 1) or 3x3 CSMatrixRS (bs == 3)."""

    def __init__(self, ctx, n, ia, ja, a, bs=1, symm_upper=False):
        self.ctx = ctx
        self.h = C.c_void_p()
        self.n, self.bs = n, bs
        self._keep = (np.ascontiguousarray(ia, np.int32), np.ascontiguousarray(ja, np.int32),
                      np.ascontiguousarray(a, np.float64))
        ia_, ja_, a_ = self._keep
        if bs == 1:
            _check(lib().bsg_mat_csr(ctx.h, n, _ip(ia_), _ip(ja_), _dp(a_), int(symm_upper), C.byref(self.h)))
        else:
            _check(lib().bsg_mat_bsr(ctx.h, n, bs, _ip(ia_), _ip(ja_), _dp(a_), int(symm_upper), C.byref(self.h)))
        self._keep = None
        ctx._adopt(self)

    @classmethod
    def from_system(cls, ctx, sysm, symm_upper=False):
        s = sysm.upper() if symm_upper else sysm
        return cls(ctx, s.n, s.ia, s.ja, s.a, s.bs, symm_upper)

    def info(self):
        n, bs, nnz = C.c_int(), C.c_int(), C.c_int()
        _check(lib().bsg_mat_info(self.h, C.byref(n), C.byref(bs), C.byref(nnz)))
        return n.value, bs.value, nnz.value

    def sell_stats(self):
        """Sliced copy of a point matrix: stored entries (padding included)
        and rows summed outside the slices (more than 256 entries)."""
        out = (C.c_longlong * 9)()
        _check(lib().bsg_sell_stats(self.h, None, out))
        return dict(entries=out[0], long=out[6])

    def mvm(self, x, y):
        """y = A x, both CUDA float64 tensors of length n*bs."""
        _check(lib().bsg_mvm_dev(self.ctx.h, self.h, _ptr(x), _ptr(y)))

    def mvm_multi(self, X, Y):
        """Y = A X for X of shape (nrhs, n*bs)."""
        _check(lib().bsg_mvm_multi_dev(self.ctx.h, self.h, X.shape[0], _ptr(X), _ptr(Y)))

    def mvm_host(self, x):
        y = np.zeros(self.n * self.bs)
        _check(lib().bsg_mvm(self.ctx.h, self.h, _dp(x), _dp(y)))
        return y

    def free(self):
        if self.h:
            lib().bsg_mat_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Factor:
    """IC2 (kind 'ich2') or ILU2 (kind 'ilu2') factor of a Matrix, on the device."""

    def __init__(self, ctx, mat, kind="ich2", param=None):
        self.ctx = ctx
        self.param = param if param is not None else default_param(ordtype=0, fcttyp=2)
        self.h = C.c_void_p()
        f = lib().bsg_fct_ich2 if kind == "ich2" else lib().bsg_fct_ilu2
        _check(f(ctx.h, mat.h, C.byref(self.param), C.byref(self.h)))
        self.kind = kind
        ctx._adopt(self)

    def info(self):
        n, nnz, ll, lu = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        d1, d2 = C.c_double(), C.c_double()
        _check(lib().bsg_fct_info(self.h, C.byref(n), C.byref(nnz), C.byref(ll), C.byref(lu), C.byref(d1),
                                  C.byref(d2)))
        return dict(n=n.value, nnz=nnz.value, levels_l=ll.value, levels_u=lu.value, density=d1.value,
                    density2=d2.value)

    def export(self):
        """Factor in the reference layout: (iu, ju, l, u), inverse pivots first."""
        info = self.info()
        n, nnz = info["n"], info["nnz"]
        iu = np.zeros(n + 1, np.int32)
        ju = np.zeros(nnz, np.int32)
        l = np.zeros(nnz)
        u = np.zeros(nnz)
        _check(lib().bsg_fct_export(self.h, None, iu.ctypes.data_as(C.POINTER(C.c_int)),
                                    ju.ctypes.data_as(C.POINTER(C.c_int)), l.ctypes.data_as(C.POINTER(C.c_double)),
                                    u.ctypes.data_as(C.POINTER(C.c_double))))
        return iu, ju, l, u

    def to_fp32(self):
        _check(lib().bsg_fct_to_fp32(self.h))

    def export_block(self):
        """Block factor of a block ILU2: (ia, ja, l, u), 3x3 column-major blocks."""
        nb, nz = C.c_int(), C.c_int()
        _check(lib().bsg_fct_export_block(self.h, C.byref(nb), C.byref(nz), None, None, None, None))
        ia = np.zeros(nb.value + 1, np.int32)
        ja = np.zeros(nz.value, np.int32)
        l = np.zeros(9 * nz.value)
        u = np.zeros(9 * nz.value)
        _check(lib().bsg_fct_export_block(self.h, None, None, ia.ctypes.data_as(C.POINTER(C.c_int)),
                                          ja.ctypes.data_as(C.POINTER(C.c_int)),
                                          l.ctypes.data_as(C.POINTER(C.c_double)),
                                          u.ctypes.data_as(C.POINTER(C.c_double))))
        return ia, ja, l, u

    def sell_stats(self):
        """Sliced copies of the factor: stored entries of the strict L / U
        rows, tiles of their tiled FP32 form (0: untiled), the most x
        blocks one tile stages and the rows of L / U summed outside the
        slices (more than 256 entries)."""
        out = (C.c_longlong * 9)()
        _check(lib().bsg_sell_stats(None, self.h, out))
        return dict(entries_l=out[1], entries_u=out[2], tiles_l=out[3], tiles_u=out[4], tile_blocks=out[5],
                    long_l=out[7], long_u=out[8])

    def solve_l(self, x, y, mode=0, nsweeps=3):
        _check(lib().bsg_solve_l_dev(self.ctx.h, self.h, mode, nsweeps, _ptr(x), _ptr(y)))

    def solve_u(self, x, y, mode=0, nsweeps=3):
        _check(lib().bsg_solve_u_dev(self.ctx.h, self.h, mode, nsweeps, _ptr(x), _ptr(y)))

    def solve_multi(self, lower, X, Y, mode=0, nsweeps=3):
        """Solves with L (lower) or U for the rows of X (nrhs, n) into Y."""
        _check(lib().bsg_solve_multi_dev(self.ctx.h, self.h, int(lower), mode, nsweeps, X.shape[0], _ptr(X),
                                         _ptr(Y)))

    def solve_ut(self, x, y, mode=0, nsweeps=3):
        """y = U^{-T} x (SolveL on U's storage)."""
        _check(lib().bsg_solve_t_dev(self.ctx.h, self.h, 0, mode, nsweeps, _ptr(x), _ptr(y)))

    def solve_lt(self, x, y, mode=0, nsweeps=3):
        """y = L^{-T} x (SolveU on L's storage)."""
        _check(lib().bsg_solve_t_dev(self.ctx.h, self.h, 1, mode, nsweeps, _ptr(x), _ptr(y)))

    def free(self):
        if self.h:
            lib().bsg_fct_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class UNet:
    """The learned FGMRES stage (bsg_unet_*): a 4-level 3D conv U-Net on an
    nx x ny x nz grid, bf16 weights, FP32 accumulation, trained by the
    library's own forward / backward kernels."""

    def __init__(self, ctx, nx, ny, nz, train=False):
        self.ctx = ctx
        self.h = C.c_void_p()
        self.grid = (nx, ny, nz)
        _check(lib().bsg_unet_create(ctx.h, nx, ny, nz, int(train), C.byref(self.h)))
        self.nparam = lib().bsg_unet_nparam(self.h)
        ctx._adopt(self)

    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.size == self.nparam
        _check(lib().bsg_unet_set_weights(self.h, w.ctypes.data_as(C.POINTER(C.c_float))))

    def weights(self):
        w = np.zeros(self.nparam, np.float32)
        _check(lib().bsg_unet_get_weights(self.h, w.ctypes.data_as(C.POINTER(C.c_float))))
        return w

    def grads(self):
        g = np.zeros(self.nparam, np.float32)
        _check(lib().bsg_unet_get_grads(self.h, g.ctypes.data_as(C.POINTER(C.c_float))))
        return g

    def set_matrix(self, mat):
        _check(lib().bsg_unet_set_matrix(self.h, mat.h))
        self._mat = mat

    def set_diag(self, d):
        """Second input channel from a CUDA float64 tensor of diagonal values."""
        _check(lib().bsg_unet_set_diag(self.h, _ptr(d)))

    def forward(self, r, y):
        _check(lib().bsg_unet_forward_dev(self.h, _ptr(r), _ptr(y)))

    def train_sample(self, r, t, want_loss=False):
        loss = C.c_double(0.0)
        _check(lib().bsg_unet_train_sample(self.h, _ptr(r), _ptr(t), C.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def adam(self, lr, step, beta1=0.9, beta2=0.999, eps=1e-8):
        _check(lib().bsg_unet_adam(self.h, lr, beta1, beta2, eps, step))

    def zero_grads(self):
        _check(lib().bsg_unet_zero_grads(self.h))

    def free(self):
        if self.h:
            lib().bsg_unet_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


FACT_STAT_NAMES = ("tries", "parks", "cyc_pop", "cyc_close", "cyc_blocked", "cyc_tail", "cyc_upd", "cyc_fin",
                   "members", "mask", "rounds", "cyc_pf", "cyc_pa", "cyc_pb", "big_rows", "warps",
                   "cyc_pass_load", "cyc_pass_close", "cyc_to_publish", "cyc_post_publish", "batches", "closed",
                   "cyc_tail_close", "cyc_fin_prepub")


def fact_stats():
    """Scheduler counters of the last factorisation in this process."""
    out = (C.c_ulonglong * 24)()
    _check(lib().bsg_fact_stats(out, 24))
    return dict(zip(FACT_STAT_NAMES, list(out)))


def pcg(ctx, mat, fct, b, x, param):
    """PCG on device tensors (x holds the initial guess, overwritten)."""
    _check(lib().bsg_pcg_dev(ctx.h, mat.h, fct.h, _ptr(b), _ptr(x), C.byref(param)))
    return param


def pcg_batch(ctx, mat, fct, B, X, param, seg_off=None):
    """Batched PCG: B, X CUDA float64 tensors [nrhs, n]; seg_off (optional)
    the point-row offsets of independent diagonal blocks.  Returns per-system
    iterations, FP64 true relative residuals ([nrhs * nseg], right-hand side
    major) and the tuned shapes (chunk, group, iterations per graph, replays)."""
    nrhs = B.shape[0]
    if seg_off is None:
        nseg, so = 1, None
    else:
        so = np.ascontiguousarray(seg_off, dtype=np.int32)
        nseg = len(so) - 1
    it = np.zeros(nrhs * nseg, np.int32)
    rs = np.zeros(nrhs * nseg)
    tn = np.zeros(4, np.int32)
    _check(lib().bsg_pcg_batch_dev(ctx.h, mat.h, fct.h, nrhs, nseg, None if so is None else _ip(so), _ptr(B), _ptr(X),
                                   C.byref(param), it.ctypes.data_as(C.POINTER(C.c_int)),
                                   rs.ctypes.data_as(C.POINTER(C.c_double)), tn.ctypes.data_as(C.POINTER(C.c_int))))
    return it, rs, tn


def lanczos(ctx, mat, fct, b, x, param):
    """Two-sided Lanczos (CSVector::Lanczos) on device tensors (x holds x0)."""
    _check(lib().bsg_lanczos_dev(ctx.h, mat.h, fct.h, _ptr(b), _ptr(x), C.byref(param)))
    return param


def block_lanczos(ctx, mat, fct, ittype, B, X, param):
    """Block Lanczos (ittype 2 central, 3 right, 4 left) on device tensors
    B, X [nrhs, n] (X holds x0); returns the final relative true residuals."""
    nrhs = B.shape[0]
    res = np.zeros(nrhs)
    _check(lib().bsg_block_lanczos_dev(ctx.h, mat.h, fct.h, ittype, nrhs, _ptr(B), _ptr(X), C.byref(param),
                                       res.ctypes.data_as(C.POINTER(C.c_double))))
    return res


def gmres(ctx, mat, fct, b, x, param):
    """GMRES(restart) / FGMRES(restart) (param.krylov == 2) on device tensors."""
    _check(lib().bsg_gmres_dev(ctx.h, mat.h, fct.h, _ptr(b), _ptr(x), C.byref(param)))
    return param


def solve_symm(ctx, n, ia, ja, a, b, param):
    """CSVector::SolveSymm(CSMatrixR&) counterpart: upper-stored SPD CSR, host buffers."""
    x = np.zeros(n)
    _check(lib().bsg_solve_symm_csr(ctx.h, n, _ip(ia), _ip(ja), _dp(a), _dp(b), _dp(x), C.byref(param)))
    return x


def solve(ctx, mat, fct, b, x0, param):
    """The Krylov solve of bsg_solve with host buffers: x0 the initial guess;
    returns the solution (also when the iteration limit stopped the loop,
    which then raises after the copy is taken)."""
    x = np.array(x0, dtype=np.float64, copy=True)
    _check(lib().bsg_solve(ctx.h, mat.h, fct.h, _dp(b), x.ctypes.data_as(C.POINTER(C.c_double)), C.byref(param)))
    return x


# ---- files in the reference's formats (CSMatrixR::ReadMtrBin / WriteMtrBin /
#      ReadMtr, CSVector::ReadVect / WriteVectBin / ReadVectBin)

def _ni(n):
    return np.zeros(max(n, 0), np.int32)


def read_system_bin(path, nvec=0):
    """A CSMatrixR in binary form followed by nvec CSVectors in binary form
    (the layout of CSMatrixR::ConvertToBinary): returns (m, n, list, ia, ja,
    a, [vectors])."""
    L = lib()
    pb = os.fsencode(path)
    off = C.c_longlong(0)
    m, n, nl, nz = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    _check(L.bsg_read_mtr_bin(pb, C.byref(off), C.byref(m), C.byref(n), C.byref(nl), C.byref(nz), None, None, None,
                              None))
    lst, ia, ja, a = _ni(nl.value), _ni(nl.value + 1), _ni(nz.value), np.zeros(nz.value)
    ptr = lambda v: v.ctypes.data_as(C.POINTER(C.c_int if v.dtype == np.int32 else C.c_double))  # noqa: E731
    _check(L.bsg_read_mtr_bin(pb, C.byref(off), None, None, None, None, ptr(lst), ptr(ia), ptr(ja), ptr(a)))
    vecs = []
    for _ in range(nvec):
        nv, nr, npart = C.c_int(), C.c_int(), C.c_int()
        _check(L.bsg_read_vect_bin(pb, C.byref(off), C.byref(nv), C.byref(nr), C.byref(npart), None, None, None))
        v, bl, ind = np.zeros(nv.value * nr.value), _ni(npart.value + 1), _ni(npart.value)
        _check(L.bsg_read_vect_bin(pb, C.byref(off), None, None, None, ptr(v), ptr(bl), ptr(ind)))
        vecs.append(v)
    return m.value, n.value, lst, ia, ja, a, vecs


def write_system_bin(path, ia, ja, a, vecs=(), lst=None):
    """Write a CSMatrixR (binary form) and then the vectors (CSVector binary
    form, one part each), as CSMatrixR::ConvertToBinary lays a system out."""
    L = lib()
    pb = os.fsencode(path)
    n = len(ia) - 1
    lst = np.arange(n, dtype=np.int32) if lst is None else lst
    _check(L.bsg_write_mtr_bin(pb, 0, n, n, n, _ip(lst), _ip(ia), _ip(ja), _dp(a)))
    for v in vecs:
        v = np.ascontiguousarray(v, np.float64)
        _check(L.bsg_write_vect_bin(pb, 1, len(v), 1, 1, _dp(v), _ip(np.array([0, len(v)])), _ip(np.array([0]))))


def read_system_text(path, nvec=0):
    """The text form CSMatrixR::ReadMtr reads, then nvec vectors as
    CSVector::ReadVect reads them: returns (n, ia, ja, a, [vectors])."""
    L = lib()
    pb = os.fsencode(path)
    off = C.c_longlong(0)
    n, nz = C.c_int(), C.c_int()
    _check(L.bsg_read_mtr(pb, C.byref(off), C.byref(n), C.byref(nz), None, None, None))
    ia, ja, a = _ni(n.value + 1), _ni(nz.value), np.zeros(nz.value)
    _check(L.bsg_read_mtr(pb, C.byref(off), None, None, ia.ctypes.data_as(C.POINTER(C.c_int)),
                          ja.ctypes.data_as(C.POINTER(C.c_int)), a.ctypes.data_as(C.POINTER(C.c_double))))
    vecs = []
    for _ in range(nvec):
        v = np.zeros(n.value)
        _check(L.bsg_read_vect(pb, C.byref(off), n.value, v.ctypes.data_as(C.POINTER(C.c_double))))
        vecs.append(v)
    return n.value, ia, ja, a, vecs


_bslib = None


def bslib():
    """Load libbsg_bslib.so, the drop-ins for Bslib's AbstractSymmSolver /
    AbstractSolver (built against the reference's headers)."""
    global _bslib
    if _bslib is None:
        lib()
        path = os.path.join(os.path.dirname(LIB_SO), "libbsg_bslib.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is not built; build with BSLIB_INCLUDE (or BSG_REFERENCE) set")
        L = C.CDLL(path)
        L.bsg_bslib_abstract.restype = C.c_int
        L.bsg_bslib_abstract.argtypes = [C.c_int, C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(Param)]
        L.bsg_bslib_last_error.restype = C.c_char_p
        L.bsg_bslib_operator_create.restype = C.c_int
        L.bsg_bslib_operator_create.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                                C.POINTER(C.c_double), C.c_int, C.POINTER(Param),
                                                C.POINTER(C.c_void_p)]
        L.bsg_bslib_operator_free.argtypes = [C.c_void_p]
        L.bsg_bslib_operator_fns.argtypes = [C.POINTER(C.c_void_p)]
        _bslib = L
    return _bslib


def abstract_solve(symm, gener, fns, param):
    """bsg_bslib_abstract: the GPU AbstractSymmSolver (symm) / AbstractSolver
    on a generator object and its seven callbacks; returns the status code
    (the solution goes through the generator's store callback)."""
    return bslib().bsg_bslib_abstract(int(symm), gener, fns, C.byref(param))


class GpuOperator:
    """The matrix and its IC2 / ILU2 factor on the GPU behind the reference's
    CMVM / CSOLVELU callbacks (bsg_bslib::MvmA / SolveLU / SolveL / SolveU):
    .h is the operator object, .fns the four function pointers."""

    def __init__(self, n, ia, ja, a, symm_upper, param):
        L = bslib()
        self.h = C.c_void_p()
        rc = L.bsg_bslib_operator_create(n, _ip(ia), _ip(ja), _dp(a), int(symm_upper), C.byref(param),
                                         C.byref(self.h))
        if rc != OK:
            raise BsgError(rc, L.bsg_bslib_last_error().decode(errors="replace"))
        self.fns = (C.c_void_p * 4)()
        L.bsg_bslib_operator_fns(self.fns)

    def free(self):
        if self.h:
            bslib().bsg_bslib_operator_free(self.h)
            self.h = C.c_void_p()


def solver(ctx, n, ia, ja, a, b, param):
    """CSVector::Solver(CSMatrixR&) counterpart: full CSR, ILU2 + GMRES, host buffers."""
    x = np.zeros(n)
    _check(lib().bsg_solver_csr(ctx.h, n, _ip(ia), _ip(ja), _dp(a), _dp(b), _dp(x), C.byref(param)))
    return x
