"""Build the native libraries of the package in-tree.

* ``libbsg.so``          -- the sm_100a solver library (csrc/*.cu), nvcc.
* ``libbsg_problems.so`` -- the host-side problem generators (csrc/problems.cpp).

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
    if verbose or ptxas_info:
        for k, v in logs.items():
            if v.strip():
                print(f"== {os.path.basename(k)}\n{v}", file=sys.stderr)
    return lib


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
