"""Generate tests/golden/*.npz from the reference Bslib itself.

The reference ships no golden vectors or known-answer tests, so its own
solver, compiled from its sources into oracle/_ref/libbslib_ref.so
(``make -C oracle ref``), is run here on small seeded systems and the outputs
are stored as fixtures.  The GPU box has no reference sources; the fixtures
let every machine check the oracle against the reference.

    python tests/golden/make_golden.py            (all fixtures)
    python tests/golden/make_golden.py --block    (lame_block.npz only)
    python tests/golden/make_golden.py --cfg      (the benchmark-configuration
                                                  fixtures cfg1_heat32.npz and
                                                  cell12_lame_periodic.npz only)
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "bcm-problems_b200"), os.path.join(ROOT, "tests")]

import problems as P  # noqa: E402
from oracle_ffi import RefLib  # noqa: E402


def nonsymmetric(s, skew=0.3):
    a = s.a.copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.ia))
    off = s.ja != rows
    a[off] *= 1.0 + skew * np.sign(s.ja[off] - rows[off])
    return a


def main():
    ref = RefLib()
    out = {}
    s = P.heat3d(8, 8, 6, sigma=1.0, seed=21)
    u = s.upper()
    x = np.random.default_rng(22).standard_normal(s.n)
    out["n"] = s.n
    out["ia"], out["ja"], out["a"] = s.ia, s.ja, s.a
    out["ua_ia"], out["ua_ja"], out["ua_a"] = u.ia, u.ja, u.a
    out["b"] = s.rhs[0]
    out["x"] = x
    out["mvm"] = ref.mvm(s.ia, s.ja, s.a, x)
    out["mvm_symm"] = ref.mvm(u.ia, u.ja, u.a, x, symm=True)
    for tag, t1, t2 in (("ic2_a", 1e-3, 1e-3), ("ic2_b", 1e-2, 1e-4)):
        iu, ju, uu, st = ref.ich2(u.ia, u.ja, u.a, tau1=t1, tau2=t2, theta=0.1)
        out[f"{tag}_iu"], out[f"{tag}_ju"], out[f"{tag}_u"] = iu, ju, uu
        out[f"{tag}_density"] = np.array(st[:2])
        out[f"{tag}_solve_l"] = ref.solve_l(iu, ju, uu, x)
        out[f"{tag}_solve_u"] = ref.solve_u(iu, ju, uu, x)
    iu, ju, uu = ref.ich0(u.ia, u.ja, u.a)
    out["ic0_iu"], out["ic0_ju"], out["ic0_u"] = iu, ju, uu
    # SolveSymm(CSMatrixR&) itself cannot run IC(0): it hands Cg the (empty)
    # block factor whenever memory >= 0 and Ich fills only the plain one
    # (Bslib/solvers.cpp:4690-4730), so Cg runs on the IC(0) factor directly
    xs0, info0 = ref.cg(u.ia, u.ja, u.a, iu, ju, uu, s.rhs[0], ittype=0, eps=1e-10)
    out["symm_ic0_x"], out["symm_ic0_iters"] = xs0, np.array(info0["iters"])
    an = nonsymmetric(s)
    out["ns_a"] = an
    for tag, t1, t2 in (("ilu2_a", 1e-3, 1e-3), ("ilu2_b", 1e-2, 1e-4)):
        (il, jl, lv), (iu, ju, uv), st = ref.ilu2(s.ia, s.ja, an, tau1=t1, tau2=t2, theta=0.1)
        out[f"{tag}_iu"], out[f"{tag}_ju"], out[f"{tag}_l"], out[f"{tag}_u"] = iu, ju, lv, uv
        out[f"{tag}_density"] = np.array(st[:2])
    xs, info = ref.solve_symm(u.ia, u.ja, u.a, s.rhs[0], fcttyp=2, tau1=1e-3, tau2=1e-3, memory=-1.0, ittype=0,
                              eps=1e-10)
    out["symm_x"] = xs
    out["symm_iters"] = np.array(info["iters"])
    xn, info = ref.solver(s.ia, s.ja, an, s.rhs[0], tau1=1e-3, tau2=1e-3, sttype=1, eps=1e-10)
    out["nonsymm_x"] = xn
    out["nonsymm_iters"] = np.array(info["iters"])
    path = os.path.join(HERE, "heat_8x8x6.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def nonsymmetric_blocks(s, skew=0.3):
    a = s.a.reshape(-1, s.bs, s.bs).copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.ia))
    off = s.ja != rows
    a[off] *= (1.0 + skew * np.sign(s.ja[off] - rows[off]))[:, None, None]
    return a.reshape(-1)


def main_block():
    """Block (CSMatrixRS) fixtures: CombineLU, block ILU2 with its SVD scaling,
    block IC2 with its eigenvector scaling, block SolveL / SolveU, on a small
    Lame block matrix and a nonsymmetric variant of it."""
    ref = RefLib()
    out = {}
    s = P.lame3d(4, sigma=1.0, seed=31)
    bs = s.bs
    x = np.random.default_rng(32).standard_normal(s.n * bs)
    out["nb"], out["bs"] = s.n, bs
    out["ia"], out["ja"], out["a"] = s.ia, s.ja, s.a
    out["ns_a"] = nonsymmetric_blocks(s)
    out["x"] = x
    ia_s, ja_s, al, au = ref.combine_lu_block(s.ia, s.ja, s.a, bs)
    out["clu_ia"], out["clu_ja"], out["clu_l"], out["clu_u"] = ia_s, ja_s, al, au
    for tag, vals, t1, t2 in (("bilu_a", "a", 1e-3, 1e-3), ("bilu_b", "a", 1e-2, 1e-5), ("bilu_ns", "ns_a", 1e-3, 1e-4)):
        ia_f, ja_f, l, u, st = ref.ilu2_block(s.ia, s.ja, out[vals], bs, tau1=t1, tau2=t2, theta=0.1)
        out[f"{tag}_ia"], out[f"{tag}_ja"], out[f"{tag}_l"], out[f"{tag}_u"] = ia_f, ja_f, l, u
        out[f"{tag}_density"] = np.array(st[:2])
        out[f"{tag}_solve_l"] = ref.solve_l_block(ia_f, ja_f, l, bs, x)
        out[f"{tag}_solve_u"] = ref.solve_u_block(ia_f, ja_f, u, bs, x)
    u = s.upper()
    out["ua_ia"], out["ua_ja"], out["ua_a"] = u.ia, u.ja, u.a
    for tag, t1, t2 in (("bic_a", 1e-3, 1e-3), ("bic_b", 1e-2, 1e-5)):
        ia_f, ja_f, uf, st = ref.ich2_block(u.ia, u.ja, u.a, bs, tau1=t1, tau2=t2, theta=0.1)
        out[f"{tag}_ia"], out[f"{tag}_ja"], out[f"{tag}_u"] = ia_f, ja_f, uf
        out[f"{tag}_solve_l"] = ref.solve_l_block(ia_f, ja_f, uf, bs, x)
        out[f"{tag}_solve_u"] = ref.solve_u_block(ia_f, ja_f, uf, bs, x)
    path = os.path.join(HERE, "lame_block.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def sha(*arrays):
    """sha256 over the raw bytes of the arrays, in order (a generator pin)."""
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main_cfg():
    """The reference's own solves at benchmark configurations.

    cfg1_heat32.npz: the first benchmark configuration exactly -- 3-D heat,
    7-point stencil, 32^3 (n = 32768), unit conductivity, RHS uniform[-1,1]
    from seed 0; CSVector::SolveSymm(CSMatrixR&) with IC2 tau1 = tau2 = 1e-3,
    theta = 0.1, PCG to relative residual 1e-10 (ittype 0).  Holds the
    solution, the iteration count, the factor density, a hash of the factor
    pattern and the factor's action through SolveL / SolveU on a seeded probe
    vector (4096 sampled entries: the 7.5 MB of factor values stay out).

    cell12_lame_periodic.npz: the homogenisation cell's shape at a size the
    CPU solves in seconds -- periodic Q1 Lame on 12^3 nodes, inclusions of
    radius 1-2 cells at 30% volume fraction, contrast 100, seed 2, node 0
    pinned; its six unit macro-strain load cases each solved by
    CSVector::SolveSymm(CSMatrixRS&) (block IC2 + PCG, tau 1e-3, relative
    residual 1e-8).  Holds the six solutions and each one's distance to a
    sparse direct solve, the accuracy the reference itself reached.
    """
    import scipy.sparse.linalg as spla
    ref = RefLib()
    s = P.config(1)
    u = s.upper()
    b = s.rhs[0]
    x, info = ref.solve_symm(u.ia, u.ja, u.a, b, fcttyp=2, tau1=1e-3, tau2=1e-3, theta=0.1, memory=-1.0, ittype=0,
                             eps=1e-10, niter=3000)
    iu, ju, uu, st = ref.ich2(u.ia, u.ja, u.a, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0)
    rng = np.random.default_rng(101)
    probe = rng.standard_normal(s.n)
    idx = np.sort(rng.choice(s.n, 4096, replace=False)).astype(np.int32)
    out = dict(system_sha=sha(s.ia, s.ja, s.a, b), upper_sha=sha(u.ia, u.ja, u.a), x_ref=x,
               iters=np.array(info["iters"]),
               true_res=np.array(np.linalg.norm(b - s.to_scipy() @ x) / np.linalg.norm(b)),
               density=np.array(st[0]), factor_nnz=np.array(len(ju)), factor_pattern_sha=sha(iu, ju),
               probe_idx=idx, probe_solve_l=ref.solve_l(iu, ju, uu, probe)[idx],
               probe_solve_u=ref.solve_u(iu, ju, uu, probe)[idx])
    path = os.path.join(HERE, "cfg1_heat32.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")

    c = P.lame_periodic(12, 0.3, 1.0, 2.0, 0.3, 100.0, 2)
    cu = c.upper()
    X, infos = ref.solve_symm_block(cu.ia, cu.ja, cu.a, c.bs, c.rhs, tau1=1e-3, tau2=1e-3, theta=0.1, memory=20.0,
                                    ittype=0, eps=1e-8, niter=3000)
    A = c.to_scipy().tocsc()
    lu = spla.splu(A)
    ref_err = []
    for k in range(c.rhs.shape[0]):
        xd = lu.solve(c.rhs[k])
        ref_err.append(np.linalg.norm(X[k] - xd) / np.linalg.norm(xd))
    out = dict(system_sha=sha(c.ia, c.ja, c.a, c.rhs), X_ref=X, iters=np.array([i["iters"] for i in infos]),
               ref_err_vs_direct=np.array(ref_err))
    path = os.path.join(HERE, "cell12_lame_periodic.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes", "ref errors", ref_err)


if __name__ == "__main__":
    if "--cfg" in sys.argv:
        main_cfg()
    else:
        if "--block" not in sys.argv:
            main()
        main_block()
