#!/usr/bin/env python
"""Benchmark of the preconditioned Krylov path on B200.

Metric: wall milliseconds from a device-resident system (A, b) to a solution x
with FP64 true relative residual ||b - Ax|| / ||b|| <= 1e-8, for the learned +
mixed arm: FP32 IC2 factor (= ILU2 of the symmetric matrix) applied by
Jacobi(6) sweeps, followed by the trained U-Net stage, inside FP64
FGMRES(30).  Beside it, the same step with the plain FP64 arm (FP64 factor,
exact triangular solves, PCG), the mixed PCG and the plain mixed FGMRES, and
the HBM bandwidth of the SpMV / sweep kernels and the tensor throughput of
the U-Net convolutions.

Workload: 3-D heat, 7-point stencil, 128^3 cells (n = 2,097,152), conductivity
lognormal(sigma=1.5) per cell from seed 4, RHS uniform[-1,1].  A step is one
complete solve: device matrix set-up, factorisation, the Krylov loop with the
learned stage, the FP64 true residual.  The network (weights/unet_heat64.npz,
trained by learned.py on 2000 pairs from 64^3 instances) is loaded once
before the timed region, like any model.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (torchrun, one rank per GPU) runs N independent replicas ("replicas
only": one system does not shard); the time is the max over ranks.
--impl reference times the reference Bslib CPU solver (oracle/_ref, compiled
from the reference sources) on the same system on rank 0.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "bcm-problems_b200"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "ms to rel. residual 1e-8: learned+mixed FGMRES vs FP64 ILU2-PCG; SpMV HBM GB/s"
WORKLOAD = "heat3d 7-point 128^3, lognormal(sigma=1.5) conductivity, seed 4"
GRID, SIGMA, SEED = 128, 1.5, 4
TOL = 1e-8
TAU = 1e-3


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if s[4 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def make_system(grid=GRID):
    import problems as P
    s = P.heat3d(grid, sigma=SIGMA, seed=SEED)
    return s, s.upper()


def mixed_param(bsg, krylov=0, learned=None):
    """FP32 IC2 factor applied by Jacobi(6) sweeps (a symmetric polynomial
    preconditioner); krylov 0: FP64 PCG, 2: FP64 FGMRES(30) (with the learned
    stage when `learned` is a network); stop confirmed on the FP64 true
    residual."""
    p = bsg.default_param(ordtype=0, fcttyp=2, tau1=TAU, tau2=TAU, theta=0.1, memory=20.0, ittype=0, eps=TOL,
                          niter=3000, precision=1, trisolve=1, nsweeps=6, krylov=krylov, restart=30, sttype=1,
                          true_residual=1)
    if learned is not None:
        p.learned = learned.h.value
    return p


def fp64_param(bsg):
    return bsg.default_param(ordtype=0, fcttyp=2, tau1=TAU, tau2=TAU, theta=0.1, memory=20.0, ittype=0, eps=TOL,
                             niter=3000, precision=0, trisolve=0)


def unet_flops(grid):
    """FLOPs of one U-Net forward on grid^3 (W0 counted with its 16 padded
    input channels, as the tensor cores run it)."""
    import learned
    vox = [grid ** 3 // 8 ** l for l in range(4)]
    level = (0, 1, 2, 3, 2, 1, 0)
    return sum(2 * 27 * ci * co * vox[level[k]] for k, (ci, co) in enumerate(learned.LAYERS))


def run_reference(args, rank):
    """Reference arm: the reference Bslib's own CPU solver on the same system."""
    if rank != 0:
        return 0
    from oracle_ffi import RefLib, REF_SO
    if not os.path.exists(REF_SO):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libbslib_ref.so not built (needs the "
                          "reference sources at build time)"}))
        return 0
    import numpy as np
    s, u = make_system()
    b = s.rhs[0]
    ref = RefLib()
    times = []
    info = None
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        x, info = ref.solve_symm(u.ia, u.ja, u.a, b, fcttyp=2, tau1=TAU, tau2=TAU, theta=0.1, memory=-1.0,
                                 ittype=0, eps=TOL, niter=3000)
        dt = (time.perf_counter() - t0) * 1e3
        if it >= args.warmup:
            times.append(dt)
    r = b - s.to_scipy() @ x
    res = float(np.linalg.norm(r) / np.linalg.norm(b))
    ms = statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "solver": "Bslib SolveSymm: IC2 (tau1=tau2=1e-3) + PCG, natural order",
                       "n": s.n, "nnz": s.nnz},
            "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": 1, "kind": "reference",
                             "sample": "the full system, one solve per step"},
            "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "iterations": info["iters"], "true_residual": res, "tfct_s": info["tfct"], "titr_s": info["titr"],
            "host_cores_available": os.cpu_count()}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bsg", choices=["bsg", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lean", action="store_true",
                    help="timed steps only (no other arms, e2e, kernel timing or CPU baseline): profiling runs")
    ap.add_argument("--grid", type=int, default=GRID, help="cells per side (profiling of smaller cases)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    args.warmup = max(args.warmup, 3)

    import numpy as np
    import torch
    import bsg
    import learned

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    ctx = bsg.Context(local)
    s, u = make_system(args.grid)
    n = s.n
    dev = torch.device("cuda", local)
    d_ia = torch.as_tensor(u.ia, device=dev)
    d_ja = torch.as_tensor(u.ja, device=dev)
    d_a = torch.as_tensor(u.a, device=dev)
    d_b = torch.as_tensor(s.rhs[0], device=dev)
    L = bsg.lib()
    import ctypes as C

    net = bsg.UNet(ctx, args.grid, args.grid, args.grid)
    net.set_weights(learned.load())

    def solve_device(param):
        """One step: device CSR -> device matrix -> factor -> Krylov -> x."""
        mh = C.c_void_p()
        bsg._check(L.bsg_mat_csr_dev(ctx.h, n, C.c_void_p(d_ia.data_ptr()), C.c_void_p(d_ja.data_ptr()),
                                     C.c_void_p(d_a.data_ptr()), 1, C.byref(mh)))
        fh = C.c_void_p()
        bsg._check(L.bsg_fct_ich2(ctx.h, mh, C.byref(param), C.byref(fh)))
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        if param.krylov == 0:
            bsg._check(L.bsg_pcg_dev(ctx.h, mh, fh, C.c_void_p(d_b.data_ptr()), C.c_void_p(x.data_ptr()),
                                     C.byref(param)))
        else:
            bsg._check(L.bsg_gmres_dev(ctx.h, mh, fh, C.c_void_p(d_b.data_ptr()), C.c_void_p(x.data_ptr()),
                                       C.byref(param)))
        L.bsg_fct_free(fh)
        L.bsg_mat_free(mh)
        if param.resfin > TOL:
            raise RuntimeError(f"true residual {param.resfin:.3e} above {TOL}")
        return x

    def barrier():
        if dist is not None:
            dist.barrier()

    def headline():
        return mixed_param(bsg, krylov=2, learned=net)

    for _ in range(args.warmup):
        solve_device(headline())
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = bsg.lib().bsg_launch_count()
    params = []
    with ClockSampler(local) as clk:
        e0.record()
        for _ in range(args.steps):
            p = headline()
            solve_device(p)
            params.append(p)
        e1.record()
        torch.cuda.synchronize()
    launches = bsg.lib().bsg_launch_count() - launches0
    barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if dist is not None:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    p_last = params[-1]
    if args.lean:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
                              "higher_is_better": False, "mode": "lean", "iterations": p_last.nitperf,
                              "true_residual": p_last.resfin, "gpu_launches": int(launches),
                              "config": {"workload": WORKLOAD}}))
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0

    def timed(param):
        e0.record()
        solve_device(param)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), param

    # ---- the other arms on the same system: plain FP64 (FP64 IC2, exact
    #      sync-free solves, PCG), mixed PCG, mixed FGMRES without the network
    ms64, p64 = timed(fp64_param(bsg))
    ms_pcg, p_pcg = timed(mixed_param(bsg, krylov=0))
    ms_fg, p_fg = timed(mixed_param(bsg, krylov=2))

    # ---- end to end through the host-buffer C ABI (pinned host arrays)
    h_ia = torch.from_numpy(u.ia).pin_memory().numpy()
    h_ja = torch.from_numpy(u.ja).pin_memory().numpy()
    h_a = torch.from_numpy(u.a).pin_memory().numpy()
    h_b = torch.from_numpy(np.ascontiguousarray(s.rhs[0])).pin_memory().numpy()
    e2e_ms = []
    for _ in range(max(1, min(args.steps, 3))):
        p = headline()
        t0 = time.perf_counter()
        xh = bsg.solve_symm(ctx, n, h_ia, h_ja, h_a, h_b, p)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        if p.resfin > TOL:
            raise RuntimeError(f"e2e true residual {p.resfin:.3e} above {TOL}")
    h2d = h_ia.nbytes + h_ja.nbytes + h_a.nbytes + h_b.nbytes
    d2h = xh.nbytes

    # ---- roofline of the dominant kernels, CUDA events on the library stream
    mh = C.c_void_p()
    bsg._check(L.bsg_mat_csr_dev(ctx.h, n, C.c_void_p(d_ia.data_ptr()), C.c_void_p(d_ja.data_ptr()),
                                 C.c_void_p(d_a.data_ptr()), 1, C.byref(mh)))
    pr = mixed_param(bsg)
    fh = C.c_void_p()
    bsg._check(L.bsg_fct_ich2(ctx.h, mh, C.byref(pr), C.byref(fh)))
    nn, bs_, nnz = C.c_int(), C.c_int(), C.c_int()
    L.bsg_mat_info(mh, C.byref(nn), C.byref(bs_), C.byref(nnz))
    t_spmv = C.c_double()
    L.bsg_time_kernel.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(C.c_double)]
    bsg._check(L.bsg_time_kernel(ctx.h, 0, mh, None, 0, 0, 50, C.byref(t_spmv)))
    t_sweep = C.c_double()
    bsg._check(L.bsg_time_kernel(ctx.h, 2, None, fh, 1, 1, 50, C.byref(t_sweep)))
    fn, fnnz = C.c_int(), C.c_int()
    L.bsg_fct_info(fh, C.byref(fn), C.byref(fnnz), None, None, None, None)
    nnz_strict = fnnz.value - n
    spmv_bytes = nnz.value * 12 + (n + 1) * 4 + 2 * n * 8
    st = (C.c_longlong * 6)()
    bsg._check(L.bsg_sell_stats(None, fh, st))
    tiled = st[4] > 0  # the backward sweep timed below
    if tiled:  # fp32 value + 16-bit local column; rhs, dinv, y_out; fp32 y_in (staged once per tile)
        sweep_bytes = nnz_strict * 6 + 3 * n * 8 + n * 4
    else:  # fp32 value + int32 column, row pointers; rhs, dinv, y_out; fp32 y_in
        sweep_bytes = nnz_strict * 8 + (n + 1) * 4 + 3 * n * 8 + n * 4
    peak, peak_kind = peaks()
    spmv_gbs = spmv_bytes / (t_spmv.value * 1e-3) / 1e9
    sweep_gbs = sweep_bytes / (t_sweep.value * 1e-3) / 1e9
    # U-Net forward (the learned stage's tensor-core work), same stream
    r_t = torch.randn(n, dtype=torch.float64, device=dev)
    y_t = torch.empty_like(r_t)
    for _ in range(3):
        net.forward(r_t, y_t)
    e0.record()
    for _ in range(20):
        net.forward(r_t, y_t)
    e1.record()
    torch.cuda.synchronize()
    t_unet = e0.elapsed_time(e1) / 20
    conv_tflops = unet_flops(args.grid) / (t_unet * 1e-3) / 1e12
    L.bsg_fct_free(fh)
    L.bsg_mat_free(mh)

    # ---- CPU baseline: the reference Bslib (oracle/_ref) on the same system, rank 0, N = 1
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle_ffi import RefLib, REF_SO
        if os.path.exists(REF_SO):
            t0 = time.perf_counter()
            _, info = RefLib().solve_symm(u.ia, u.ja, u.a, s.rhs[0], fcttyp=2, tau1=TAU, tau2=TAU, theta=0.1,
                                          memory=-1.0, ittype=0, eps=TOL, niter=3000)
            cpu = {"value": round((time.perf_counter() - t0) * 1e3, 1), "unit": "ms", "cores": 1,
                   "kind": "reference",
                   "sample": "one full solve of the benchmark system (IC2 + PCG, natural order)",
                   "iterations": info["iters"], "tfct_s": info["tfct"], "titr_s": info["titr"]}

    if rank == 0:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            bf16_peak = float(json.load(f).get("bf16_tflops", 1590.0))
        line = {
            "metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": n, "nnz": int(nnz.value), "parallelism": f"replicas{world}",
                       "solver": "IC2(tau1=tau2=1e-3) FP32 factor, Jacobi(6) triangular solves, learned U-Net "
                                 "stage (bf16, trained at 64^3), FP64 FGMRES(30)",
                       "l2": "inputs larger than L2 (matrix 175 MB, factor 420 MB)"},
            "iterations": p_last.nitperf, "true_residual": p_last.resfin,
            "fct_ms": round(p_last.timefct * 1e3, 3), "itr_ms": round(p_last.timeitr * 1e3, 3),
            "arms": {
                "fp64_pcg": {"ms": round(ms64, 3), "iterations": p64.nitperf, "itr_ms": round(p64.timeitr * 1e3, 3)},
                "mixed_pcg": {"ms": round(ms_pcg, 3), "iterations": p_pcg.nitperf,
                              "itr_ms": round(p_pcg.timeitr * 1e3, 3)},
                "mixed_fgmres_plain": {"ms": round(ms_fg, 3), "iterations": p_fg.nitperf,
                                       "itr_ms": round(p_fg.timeitr * 1e3, 3)},
            },
            "speedup_vs_fp64_pcg": round(ms64 / ms, 3),
            "e2e": {"value": round(statistics.mean(e2e_ms), 3), "unit": "ms", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "kernel": "k_sell_apply (FP64 SELL-8 SpMV)", "achieved": round(spmv_gbs, 1),
                         "peak": peak, "unit": "GB/s", "frac": round(spmv_gbs / peak, 4), "traffic": None,
                         "algorithmic_bytes": spmv_bytes, "ms_per_launch": t_spmv.value,
                         "peak_source": peak_kind},
            "roofline_trisolve": {"bound": "hbm",
                                  "kernel": ("k_tsell_sweep32 (one FP32 Jacobi sweep, x staged in shared memory)"
                                             if tiled else "k_sell_sweep32 (one FP32 Jacobi sweep)"),
                                  "achieved": round(sweep_gbs, 1), "peak": peak, "unit": "GB/s",
                                  "frac": round(sweep_gbs / peak, 4), "algorithmic_bytes": sweep_bytes,
                                  # dram read + write of one launch, ncu at this workload (128^3)
                                  "traffic": (382960000 if tiled and args.grid == 128 else None),
                                  "traffic_source": "profiles/k_tsell_sweep32_heat128.md",
                                  "ms_per_launch": t_sweep.value},
            "roofline_unet": {"bound": "tensor", "kernel": "U-Net forward (level 0: k_conv3_tc, tcgen05 + TMA; deeper levels: k_conv3t / k_conv3, mma.sync)",
                              "achieved": round(conv_tflops, 1), "peak": bf16_peak, "unit": "TFLOP/s",
                              "frac": round(conv_tflops / bf16_peak, 4), "ms_per_forward": round(t_unet, 4),
                              "flops": unet_flops(args.grid)},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
