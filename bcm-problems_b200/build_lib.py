"""Build the native libraries of the package in-tree.

* ``libbsg.so``          -- the sm_100a solver library (csrc/*.cu), nvcc.
* ``libbsg_problems.so`` -- the host-side problem generators (csrc/problems.cpp).
* ``libbsg_bslib.so``    -- the drop-ins for Bslib's AbstractSymmSolver /
  AbstractSolver (csrc/bsg_bslib.cpp), compiled against the reference's own
  headers (slvparam.h, smatrix.h): built only when BSLIB_INCLUDE names the
  directory that holds them (or BSG_REFERENCE the reference source tree, whose
  Bslib/ it is); a library built earlier is kept otherwise.

Objects are compiled in parallel into ``_build/`` and linked next to this
file, so the shared objects travel with a copy of the repository.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def bslib_include():
    """Directory of the reference's Bslib headers, from BSLIB_INCLUDE or
    BSG_REFERENCE (the reference source tree); None when neither is set."""
    inc = os.environ.get("BSLIB_INCLUDE")
    if not inc and os.environ.get("BSG_REFERENCE"):
        inc = os.path.join(os.environ["BSG_REFERENCE"], "Bslib")
    if inc and not os.path.isfile(os.path.join(inc, "slvparam.h")):
        raise RuntimeError(f"BSLIB_INCLUDE / BSG_REFERENCE: no slvparam.h in {inc}")
    return inc


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "bslib_gpu.h"))
    cus = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    jobs = []
    for src in cus:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        if _stale(obj, [src] + headers) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append((src, [NVCC] + NVFLAGS + extra + ["-c", src, "-o", obj]))
    logs = {}
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        futs = {ex.submit(_run, cmd): src for src, cmd in jobs}
        for f in cf.as_completed(futs):
            logs[futs[f]] = f.result()
    objs = [os.path.join(BUILD, os.path.basename(s)[:-3] + ".o") for s in cus]
    lib = os.path.join(HERE, "libbsg.so")
    if _stale(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"])
    gen_src = os.path.join(CSRC, "problems.cpp")
    gen_lib = os.path.join(HERE, "libbsg_problems.so")
    if _stale(gen_lib, [gen_src]):
        _run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-o", gen_lib, gen_src])
    inc = bslib_include()
    shim_src = os.path.join(CSRC, "bsg_bslib.cpp")
    shim_lib = os.path.join(HERE, "libbsg_bslib.so")
    if inc and _stale(shim_lib, [shim_src, lib, os.path.join(os.path.dirname(HERE), "include", "bsg_bslib.h")]):
        _run(["g++", "-O2", "-fPIC", "-shared", "-std=gnu++14", "-fpermissive", "-w", "-I", inc, "-I",
              os.path.join(os.path.dirname(HERE), "include"), "-o", shim_lib, shim_src, "-L", HERE, "-lbsg",
              "-Wl,-rpath,$ORIGIN"])
    if verbose or ptxas_info:
        for k, v in logs.items():
            if v.strip():
                print(f"== {os.path.basename(k)}\n{v}", file=sys.stderr)
    return lib


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
