"""Sharding of batched solves over GPUs, one process per GPU.

One system does not shard (the factorisation and the triangular solves are
sequential across any partition), but batches do:

* independent problems (segments of one block-diagonal system): each rank
  takes a set of whole problems, balanced greedily by nonzeros (longest
  first onto the least-loaded rank), builds the block-diagonal system of its
  problems and solves it with the batched PCG;
* load cases of one matrix: each rank takes a contiguous range of the
  right-hand sides and solves them against its own copy of the matrix.

There is no exchange on the data path.  The only collective is an optional
gather of the per-problem iteration counts and residuals (NCCL between GPUs,
gloo in the CPU tests), after which every rank knows the whole batch's
outcome; solutions stay on the rank that computed them.
"""
import numpy as np

import problems as P


def partition_segments(weights, world):
    """Greedy (longest first) assignment of segments to ranks by weight;
    returns, per rank, its segment indices in ascending order."""
    w = np.asarray(weights, dtype=np.float64)
    load = np.zeros(world)
    own = [[] for _ in range(world)]
    for g in np.argsort(-w, kind="stable"):
        r = int(np.argmin(load))
        own[r].append(int(g))
        load[r] += w[g]
    return [sorted(o) for o in own]


def partition_rhs(nrhs, world):
    """Contiguous right-hand-side ranges, as even as possible."""
    edges = np.linspace(0, nrhs, world + 1).round().astype(int)
    return [(int(edges[r]), int(edges[r + 1])) for r in range(world)]


def segment_weights(system):
    """Nonzeros of each segment of a point system."""
    ia, parts = system.ia, system.parts
    return np.array([ia[parts[g + 1]] - ia[parts[g]] for g in range(len(parts) - 1)], dtype=np.int64)


def local_system(system, segs):
    """The block-diagonal system of the chosen segments (point CSR, rows in
    segment order), with its own segment offsets."""
    ia, ja, a, parts = system.ia, system.ja, system.a, system.parts
    rows, cols, vals, offs, rhs = [], [], [], [0], []
    for g in segs:
        r0, r1 = int(parts[g]), int(parts[g + 1])
        k0, k1 = int(ia[r0]), int(ia[r1])
        shift = offs[-1] - r0
        cols.append(ja[k0:k1] + shift)
        vals.append(a[k0:k1])
        rows.append(np.diff(ia[r0:r1 + 1]))
        rhs.append(system.rhs[:, r0:r1])
        offs.append(offs[-1] + (r1 - r0))
    n = offs[-1]
    lia = np.zeros(n + 1, np.int32)
    np.cumsum(np.concatenate(rows) if rows else np.zeros(0, np.int64), out=lia[1:])
    return P.System(n, 1, lia, np.concatenate(cols).astype(np.int32), np.concatenate(vals),
                    np.concatenate(rhs, axis=1), np.asarray(offs, dtype=np.int64), system.info)


def gpu_batch_solver(ctx, param_kw, upper_input=False):
    """The solver of a rank's share on its GPU: IC2 + batched PCG.  With
    upper_input the share is already stored as its upper triangle (the
    symmetric solve's input format), else it is taken from full storage."""
    def solve(sysm):
        import torch
        import bsg
        p = bsg.default_param(**param_kw)
        if upper_input:
            m = bsg.Matrix(ctx, sysm.n, sysm.ia, sysm.ja, sysm.a, sysm.bs, symm_upper=True)
        else:
            m = bsg.Matrix.from_system(ctx, sysm, symm_upper=True)
        f = bsg.Factor(ctx, m, "ich2", p)
        B = torch.as_tensor(np.ascontiguousarray(sysm.rhs[:1]), device="cuda")
        X = torch.zeros_like(B)
        it, rs, _ = bsg.pcg_batch(ctx, m, f, B, X, p, seg_off=sysm.parts)
        x = X.cpu().numpy()[0]
        f.free()
        m.free()
        return x, it, rs
    return solve


def solve_segments_sharded(system, solve, rank, world, gather=True, group=None):
    """Solve this rank's share of the segments of `system` with `solve`
    (local system -> (x, iterations, residuals)).  Returns the rank's segment
    indices, its local solution and, when `gather`, the iteration counts and
    residuals of all segments in global order (one all-gather of small
    arrays through torch.distributed)."""
    own = partition_segments(segment_weights(system), world)[rank]
    loc = local_system(system, own)
    x, it, rs = solve(loc)
    out = {"segments": own, "x": x, "iterations": None, "residuals": None}
    if gather and world > 1:
        import torch.distributed as dist
        allv = [None] * world
        dist.all_gather_object(allv, (own, np.asarray(it).tolist(), np.asarray(rs).tolist()), group=group)
    else:
        allv = [(own, np.asarray(it).tolist(), np.asarray(rs).tolist())]
    nseg = len(system.parts) - 1
    its = np.zeros(nseg, np.int64)
    res = np.zeros(nseg)
    seen = np.zeros(nseg, bool)
    for segs, i_, r_ in allv:
        for g, a, b in zip(segs, i_, r_):
            its[g], res[g], seen[g] = a, b, True
    if gather and world > 1 or world == 1:
        if not seen.all():
            raise RuntimeError("some segments were solved by no rank")
        out["iterations"], out["residuals"] = its, res
    return out
