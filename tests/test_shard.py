"""Sharding of batched solves (bcm-problems_b200/shard.py) on CPU: the
greedy nnz balance, the local block-diagonal systems, and the world-size-2
gather of per-problem results over gloo.  The per-rank solver is injected (a
sparse direct solve here; the batched GPU PCG in production), so these tests
exercise the host logic of the N > 1 path without a GPU."""
import os
import socket

import numpy as np
import pytest
import scipy.sparse.linalg as spla

import problems as P
import shard


def _cpu_solver(sysm):
    """Direct solve of every segment; 'iterations' = segment size, so the
    gathered values identify the segment they belong to."""
    A = sysm.to_scipy().tocsc()
    b = sysm.rhs[0]
    x = spla.spsolve(A, b)
    parts = sysm.parts
    it = np.diff(parts)
    rs = np.array([np.linalg.norm(b[a:e] - A[a:e, a:e] @ x[a:e]) / np.linalg.norm(b[a:e])
                   for a, e in zip(parts[:-1], parts[1:])])
    return x, it, rs


def test_partition_is_balanced_and_complete():
    w = np.random.default_rng(0).integers(100, 10000, 257)
    for world in (1, 2, 3, 8):
        own = shard.partition_segments(w, world)
        flat = sorted(g for o in own for g in o)
        assert flat == list(range(len(w)))
        loads = [w[o].sum() for o in own]
        assert max(loads) <= np.mean(loads) + w.max()
    for nrhs, world in ((6, 4), (6, 6), (6, 1), (7, 3)):
        rg = shard.partition_rhs(nrhs, world)
        assert rg[0][0] == 0 and rg[-1][1] == nrhs and all(rg[i][1] == rg[i + 1][0] for i in range(world - 1))
        sz = [b - a for a, b in rg]
        assert max(sz) - min(sz) <= 1


def test_local_system_is_the_diagonal_blocks():
    s = P.heat2d_batch(9, 6, 20, sigma=1.0, seed=3)
    segs = [1, 4, 7]
    loc = shard.local_system(s, segs)
    A = s.to_scipy()
    L = loc.to_scipy()
    for q, g in enumerate(segs):
        a, e = s.parts[g], s.parts[g + 1]
        la, le = loc.parts[q], loc.parts[q + 1]
        assert (abs(L[la:le, la:le] - A[a:e, a:e])).max() == 0.0
        assert np.array_equal(loc.rhs[0, la:le], s.rhs[0, a:e])
    assert L.nnz == sum(A[s.parts[g]:s.parts[g + 1], s.parts[g]:s.parts[g + 1]].nnz for g in segs)


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        s = P.heat2d_batch(11, 6, 24, sigma=1.0, seed=3)
        res = shard.solve_segments_sharded(s, _cpu_solver, rank, world)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), segs=np.array(res["segments"]), x=res["x"],
                 it=res["iterations"], rs=res["residuals"])
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_every_problem(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    s = P.heat2d_batch(11, 6, 24, sigma=1.0, seed=3)
    sizes = np.diff(s.parts)
    x_full = spla.spsolve(s.to_scipy().tocsc(), s.rhs[0])
    got = [np.load(tmp_path / f"r{r}.npz") for r in range(2)]
    segs = [set(g["segs"].tolist()) for g in got]
    assert segs[0].isdisjoint(segs[1]) and segs[0] | segs[1] == set(range(11))
    for g in got:
        # both ranks hold every problem's outcome after the gather
        assert np.array_equal(g["it"], sizes)
        assert g["rs"].max() < 1e-12
        # each rank's solution is its problems' part of the global solution
        off = 0
        for q in g["segs"]:
            a, e = s.parts[q], s.parts[q + 1]
            assert np.allclose(g["x"][off:off + e - a], x_full[a:e], rtol=1e-10, atol=1e-12)
            off += e - a


def test_single_rank_needs_no_collective():
    s = P.heat2d_batch(5, 6, 12, sigma=1.0, seed=4)
    res = shard.solve_segments_sharded(s, _cpu_solver, 0, 1)
    assert res["segments"] == list(range(5)) and np.array_equal(res["iterations"], np.diff(s.parts))


@pytest.mark.gpu
@pytest.mark.parametrize("world", [1, 3])
def test_gpu_batch_solver_through_the_shard(ctx, world):
    """The production solver of a rank (shard.gpu_batch_solver: IC2 + batched
    PCG on the GPU) through the sharding code, every rank's share solved in
    turn on the one GPU: every problem reaches 1e-8 and matches a direct
    solve to 1e-6, whichever rank solved it."""
    s = P.heat2d_batch(17, 8, 40, sigma=1.0, seed=3)
    kw = dict(ordtype=0, fcttyp=2, tau1=1e-3, tau2=1e-3, memory=20.0, ittype=0, eps=1e-8, niter=2000,
              precision=1, trisolve=1, nsweeps=6)
    solve = shard.gpu_batch_solver(ctx, kw)
    x_full = spla.spsolve(s.to_scipy().tocsc(), s.rhs[0])
    seen = set()
    for rank in range(world):
        res = shard.solve_segments_sharded(s, solve, rank, world, gather=False)
        off = 0
        for q in res["segments"]:
            a, e = int(s.parts[q]), int(s.parts[q + 1])
            xe = x_full[a:e]
            assert np.linalg.norm(res["x"][off:off + e - a] - xe) <= 1e-6 * np.linalg.norm(xe), q
            off += e - a
            seen.add(q)
    assert seen == set(range(17))
