"""The C ABI library without a GPU: it loads, exports every function that
include/bslib_gpu.h declares, and its host-side logic answers as documented."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bslib_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_ ]+\**\s*\**(bsg_[a-z0-9_]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_path():
    names = declared_functions()
    for must in ("bsg_create", "bsg_mat_csr", "bsg_mat_bsr", "bsg_mvm_dev", "bsg_fct_ich2", "bsg_fct_ilu2",
                 "bsg_solve_l_dev", "bsg_solve_u_dev", "bsg_pcg_dev", "bsg_gmres_dev", "bsg_solve_symm_csr",
                 "bsg_solver_csr"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import bsg
    L = C.CDLL(bsg.LIB_SO)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_param_defaults_mirror_cslvparam():
    """bsg_param_default == CSlvParam() for the fields of the path
    (Bslib/slvparam.h:121-214)."""
    import bsg
    p = bsg.default_param()
    assert (p.msglev, p.fcttyp, p.ordtype) == (0, 1, 1)
    assert (p.memory, p.tau1, p.tau2, p.theta) == (1.0, 1e-2, 1e-4, 1e-1)
    assert (p.sclmin, p.pivmin) == (1e-8, 1e-8)
    assert (p.ittype, p.sttype, p.niter, p.eps, p.ichk) == (2, 2, 1000, 1e-9, 5)
    assert p.resfin == 1e10
    assert (p.precision, p.trisolve, p.restart) == (0, 0, 50)


def test_argument_checks_need_no_device():
    import bsg
    L = bsg.lib()
    h = C.c_void_p()
    # null context
    assert L.bsg_mat_csr(None, 1, None, None, None, 0, C.byref(h)) == bsg.ERR_ARG
    assert L.bsg_fct_ich2(None, None, None, C.byref(h)) == bsg.ERR_ARG
    assert L.bsg_version().startswith(b"bsg")


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import bsg
    with pytest.raises(RuntimeError):
        bsg.Context(0)
    h = C.c_void_p()
    assert bsg.lib().bsg_create(C.byref(h), 0, None) == bsg.ERR_CUDA
