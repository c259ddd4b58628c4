"""The C ABI library without a GPU: it loads, exports every function that
include/bslib_gpu.h declares, and its host-side logic answers as documented."""
import ctypes as C
import os
import re
import sys

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


_NULL_SWEEP = r'''
import ctypes as C, re, sys
sys.path.insert(0, sys.argv[1])
import bsg
L = bsg.lib()
hdr = open(sys.argv[2]).read()
names = re.findall(r"^(?:int|unsigned long long|const char \*|void) \*?(bsg_\w+)\(", hdr, re.M)
skip = {"bsg_create", "bsg_param_default", "bsg_last_error", "bsg_version", "bsg_launch_count"}
extra = {  # entry points the Python binding does not declare
    "bsg_solve_sweep_static": [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p],
    "bsg_time_kernel": [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p],
}
def dflt(t):
    if t in (C.c_int, C.c_long, C.c_longlong, C.c_uint, C.c_ulonglong, C.c_size_t):
        return 0
    if t in (C.c_float, C.c_double):
        return 0.0
    return None
for nm in names:
    if nm in skip:
        continue
    f = getattr(L, nm)
    if f.argtypes is None:
        f.argtypes = extra[nm]
    f.restype = C.c_int
    print(nm, f(*[dflt(t) for t in f.argtypes]), flush=True)
# a null output with a positive count
f = L.bsg_fact_stats
print("bsg_fact_stats/24", f(None, 24), flush=True)
'''


def test_every_entry_point_rejects_null_handles():
    """Every declared entry point, called with null handles and buffers and
    zero sizes, returns BSG_ERR_ARG (the release functions: BSG_OK, as free()
    of NULL), touches no device and does not crash -- run in a child process
    so that a crash is reported, not fatal to the test run."""
    import subprocess
    import bsg
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _NULL_SWEEP, os.path.join(root, "bcm-problems_b200"),
                        os.path.join(root, "include", "bslib_gpu.h")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    got = dict(line.split() for line in r.stdout.splitlines())
    releases = {"bsg_destroy", "bsg_mat_free", "bsg_fct_free", "bsg_unet_free"}
    ok_when_empty = {"bsg_fact_stats"}  # nothing requested, nothing written
    assert len(got) >= 35
    for nm, v in got.items():
        want = bsg.OK if nm in releases | ok_when_empty else bsg.ERR_ARG
        assert int(v) == want, (nm, v)


def test_bslib_dropins_export_the_reference_signatures():
    """libbsg_bslib.so exports the C form of the Abstract*Solver drop-ins and
    the C++ drop-ins with the reference's parameter types
    (Bslib/smatrix.h:27-34: void *, ofstream &, CSlvParam &, then the seven
    callback types)."""
    import subprocess
    import bsg
    L = bsg.bslib()
    for nm in ("bsg_bslib_abstract", "bsg_bslib_last_error"):
        assert hasattr(L, nm)
    path = os.path.join(os.path.dirname(bsg.LIB_SO), "libbsg_bslib.so")
    syms = subprocess.run(["nm", "-DC", path], capture_output=True, text=True, check=True).stdout
    cb = ("void (*)(void*, int&), void (*)(void*, int*), void (*)(void*, int*&, int*&), "
          "void (*)(void*, int, double*), void (*)(void*, int, double*), void (*)(void*, int, double*), "
          "void (*)(void*, int, double*)")
    for fn in ("AbstractSymmSolver", "AbstractSolver"):
        sig = f"bsg_bslib::{fn}(void*, std::basic_ofstream<char, std::char_traits<char> >&, CSlvParam&, {cb})"
        assert sig in syms, fn


def test_bslib_dropin_rejects_null_arguments_without_a_device():
    import bsg
    p = bsg.default_param()
    assert bsg.abstract_solve(True, None, None, p) == bsg.ERR_ARG
    fns = (C.c_void_p * 7)()
    assert bsg.abstract_solve(True, None, fns, p) == bsg.ERR_ARG
    assert b"callback 1 is null" in bsg.bslib().bsg_bslib_last_error()


def test_parfbss_header_symbols_are_exported():
    """Every bsg_parfbss_* function include/bsg_parfbss.h declares is exported
    by libbsg.so."""
    import bsg
    src = open(os.path.join(ROOT, "include", "bsg_parfbss.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = sorted(set(re.findall(r"\b(bsg_parfbss_[a-z_]+)\s*\(", src)))
    assert len(names) == 15
    L = C.CDLL(bsg.LIB_SO)
    assert not [n for n in names if not hasattr(L, n)]
