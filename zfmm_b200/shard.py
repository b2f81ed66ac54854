"""Multi-GPU sharding of independent units: one process per GPU, no
collective on the data path.

A single FMM runs on one GPU.  What shards are the independent units of the
batched configurations: the right-hand sides of one geometry (the reference
solves each with its own zlfmm3d / zhfmm3d call,
zfmm3d/src/laplace/zlfmm3d.f:14-245) and the instances of a many-instance
solve (each a separate call of zfmm3d/src/helmholtz/zhfmm3d.f:1-249).  Every
rank computes the same partition from the unit sizes alone, solves its share
on its own GPU and keeps its results; `gather_to_root` collects them on rank 0
(torch.distributed object gather) only where a caller wants them in one place,
for example to check them.
"""
import numpy as np

__all__ = ["partition_by_size", "rhs_block", "solve_instances", "gather_to_root",
           "solve_rhs_block"]


def partition_by_size(sizes, world_size):
    """Unit indices per rank: units sorted by decreasing size, dealt in snake
    order (0, 1, ..., N-1, N-1, ..., 0, 0, 1, ...), so that every rank gets a
    similar share of large and small units.  Deterministic: ties keep the
    input order.  Returns a list of world_size lists of indices."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    parts = [[] for _ in range(world_size)]
    for k, i in enumerate(order):
        r, lap = k % world_size, k // world_size
        parts[r if lap % 2 == 0 else world_size - 1 - r].append(i)
    return parts


def rhs_block(nd, rank, world_size):
    """Contiguous block [r0, r1) of nd right-hand sides for `rank`: the first
    nd % world_size ranks take one more."""
    if not 0 <= rank < world_size:
        raise ValueError("rank out of range")
    q, r = divmod(int(nd), world_size)
    r0 = rank * q + min(rank, r)
    return r0, r0 + q + (1 if rank < r else 0)


def solve_instances(solve, instances, rank, world_size, sizes=None):
    """Solves this rank's share of independent instances with
    solve(list_of_instances) -> list_of_results (for example
    zfmm_b200.zhfmm3d_many), and returns {instance index: result}."""
    sizes = [np.asarray(inst["zsrc"]).shape[-1] for inst in instances] if sizes is None else sizes
    mine = partition_by_size(sizes, world_size)[rank]
    res = solve([instances[i] for i in mine]) if mine else []
    return dict(zip(mine, res))


def solve_rhs_block(solve, charge, rank, world_size, dipstr=None):
    """Solves this rank's block of the right-hand sides charge (nd, ns) (and
    dipstr (nd, ns)) with solve(charge_block, dipstr_block) -> (pot, grad) of
    the block, and returns ((r0, r1), result)."""
    nd = np.asarray(charge).shape[0]
    r0, r1 = rhs_block(nd, rank, world_size)
    if r1 <= r0:
        return (r0, r1), None
    ds = None if dipstr is None else dipstr[r0:r1]
    return (r0, r1), solve(charge[r0:r1], ds)


def gather_to_root(local, rank, world_size, group=None):
    """Collects every rank's `local` object on rank 0 (list indexed by rank;
    None on the other ranks).  The only communication of a sharded solve,
    and it is not on the data path of the solve itself."""
    if world_size == 1:
        return [local]
    import torch.distributed as dist
    out = [None] * world_size if rank == 0 else None
    dist.gather_object(local, out, dst=0, group=group)
    return out
