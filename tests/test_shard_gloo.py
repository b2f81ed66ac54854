"""Sharding of independent units across ranks (zfmm_b200.shard), on CPU with
two gloo ranks: the partition is a function of the unit sizes only (every
rank computes the same one), covers every unit exactly once and balances
sizes; each rank solves its share with no communication, and the results
gathered on rank 0 equal the one-rank solve unit for unit.  The per-unit
solve here is the oracle's direct sum (test stand-in for the GPU FMM, which
this machine does not have)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from zfmm_b200 import shard


def test_partition_properties():
    rng = np.random.default_rng(3)
    sizes = np.exp(rng.uniform(np.log(2000), np.log(500000), 200)).astype(int)
    for ws in (1, 2, 3, 4, 8):
        parts = shard.partition_by_size(sizes, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(200))
        load = [sum(sizes[i] for i in p) for p in parts]
        assert max(load) <= 1.15 * (sum(sizes) / ws) + max(sizes) / ws
        assert parts == shard.partition_by_size(list(sizes), ws)  # deterministic
    # right-hand-side blocks tile [0, nd)
    for nd, ws in [(64, 2), (64, 3), (5, 8), (1, 2)]:
        blocks = [shard.rhs_block(nd, r, ws) for r in range(ws)]
        assert blocks[0][0] == 0 and blocks[-1][1] == nd
        assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))


def _instances(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        m = int(rng.integers(40, 300))
        z = rng.uniform(-1, 1, (3, m)) + 0.05j * rng.uniform(-1, 1, (3, m))
        q = rng.standard_normal(m) + 1j * rng.standard_normal(m)
        out.append(dict(zsrc=z, charge=q))
    return out


def _direct_solve(insts):
    import oracle_lib as O
    return [O.zh3ddirect(10 + 0.2j, inst["zsrc"].T, inst["charge"], ifpgh=2)[0] for inst in insts]


def _worker(rank, ws, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        insts = _instances(12, seed=5)
        mine = shard.solve_instances(_direct_solve, insts, rank, ws)
        got = shard.gather_to_root(mine, rank, ws)
        # right-hand-side blocks of one geometry
        rng = np.random.default_rng(9)
        z = rng.uniform(-1, 1, (3, 150)) + 0.05j
        charge = rng.standard_normal((7, 150)) + 1j * rng.standard_normal((7, 150))

        def solve_block(cb, _ds):
            import oracle_lib as O
            return np.stack([O.zh3ddirect(5.0, z.T, c)[0] for c in cb])

        blk = shard.solve_rhs_block(solve_block, charge, rank, ws)
        blks = shard.gather_to_root(blk, rank, ws)
        if rank == 0:
            merged = {}
            for part in got:
                assert not (set(part) & set(merged))  # no unit solved twice
                merged.update(part)
            ref = _direct_solve(insts)
            ok = sorted(merged) == list(range(12)) and all(
                np.array_equal(merged[i], ref[i]) for i in range(12))
            pot = np.concatenate([b[1] for b in blks if b[1] is not None])
            ref_b = solve_block(charge, None)
            ok = ok and np.array_equal(pot, ref_b)
            q.put(ok)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_match_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert q.get(timeout=10) is True
