"""Multi-rank column sharding on CPU (gloo, world_size 2).

Each rank generates only its own shard of the workload (the profile generator
is counter-based, so a column's inputs depend on its global index alone),
runs the oracle on it, and the gathered shards must equal one run over all
columns bit for bit.  This is the partition `bench.py --gpus N` uses, with the
CPU oracle standing in for the GPU kernels.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ccpp_physics_b200 import shard, synthetic

NCOLS, NLAY = 37, 40


def test_column_range_partitions():
    for total in (0, 1, 5, 37, 884736):
        for world in (1, 2, 3, 8):
            rs = [shard.column_range(total, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            sizes = [b - a for a, b in rs]
            assert max(sizes) - min(sizes) <= 1


def test_block_range_keeps_blocks_whole():
    sizes = synthetic.physics_blocks(100_000, seed=3)
    for world in (1, 2, 4, 8):
        rs = [shard.block_range(sizes, r, world) for r in range(world)]
        assert rs[0][0] == 0 and rs[-1][1] == len(sizes)
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
        cols = [sum(sizes[a:b]) for a, b in rs]
        assert max(cols) - min(cols) <= 2 * 256
    with pytest.raises(ValueError):
        shard.column_range(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle
        oracle.rlwinit()
        a, b = shard.column_range(NCOLS, rank, world)
        prof = synthetic.make_profiles(b - a, NLAY, seed=11, col_offset=a)
        rc, msg, out = oracle.rrtmg_lw_run(prof, nthreads=1)
        assert rc == 0, msg
        # gather variable-size shards: pad to the largest
        mx = -(-NCOLS // world)
        top = torch.zeros(mx, 2, dtype=torch.float64)
        top[: b - a] = torch.from_numpy(np.ascontiguousarray(out["topflx"]))
        parts = [torch.zeros_like(top) for _ in range(world)]
        dist.all_gather(parts, top)
        # timing reduction as the bench does it: max over ranks
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            full = np.concatenate([parts[r][: shard.column_range(NCOLS, r, world)[1]
                                             - shard.column_range(NCOLS, r, world)[0]].numpy()
                                   for r in range(world)])
            q.put((full, float(t.item())))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
def test_two_rank_shards_equal_single_run(oracle_lib):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    full, tmax = q.get(timeout=200)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert tmax == float(world)
    prof = synthetic.make_profiles(NCOLS, NLAY, seed=11)
    rc, msg, ref = oracle_lib.rrtmg_lw_run(prof, nthreads=1)
    assert rc == 0, msg
    assert np.array_equal(full, ref["topflx"])


def _sw_rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from ccpp_physics_b200 import rrtmg_sw as sw
        from oracle import oracle_sw
        oracle_sw.rswinit()
        a, b = shard.column_range(NCOLS, rank, world)
        prof = sw.add_sw_inputs(synthetic.make_profiles(b - a, NLAY, seed=21, col_offset=a), seed=21, col_offset=a,
                                night_fraction=0.3)
        out = sw.alloc_outputs(b - a, NLAY)
        rc, msg = oracle_sw.run(prof, out, nthreads=1)
        assert rc == 0, msg
        mx = -(-NCOLS // world)
        top = torch.zeros(mx, 3, dtype=torch.float64)
        top[: b - a] = torch.from_numpy(np.ascontiguousarray(out["topflx"]))
        parts = [torch.zeros_like(top) for _ in range(world)]
        dist.all_gather(parts, top)
        days = torch.zeros(mx, dtype=torch.int64)
        days[: len(prof["idxday"])] = torch.from_numpy(prof["idxday"].astype(np.int64))
        dparts = [torch.zeros_like(days) for _ in range(world)]
        dist.all_gather(dparts, days)
        if rank == 0:
            sizes = [shard.column_range(NCOLS, r, world) for r in range(world)]
            full = np.concatenate([parts[r][: e - s].numpy() for r, (s, e) in enumerate(sizes)])
            q.put((full, [dparts[r].numpy() for r in range(world)]))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
def test_two_rank_sw_shards_equal_single_run():
    """rrtmg_sw_run sharded by columns over two gloo ranks (isubcsw=2 seeds are
    per column, so they follow the columns) equals one run over all columns,
    and each rank's daytime points are the global ones split by
    shard.daytime_points."""
    from ccpp_physics_b200 import rrtmg_sw as sw
    from oracle import oracle_sw
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sw_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    full, dparts = q.get(timeout=200)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    oracle_sw.rswinit()
    prof = sw.add_sw_inputs(synthetic.make_profiles(NCOLS, NLAY, seed=21), seed=21, night_fraction=0.3)
    ref = sw.alloc_outputs(NCOLS, NLAY)
    rc, msg = oracle_sw.run(prof, ref, nthreads=1)
    assert rc == 0, msg
    assert np.array_equal(full, ref["topflx"])
    for r in range(world):
        a, b = shard.column_range(NCOLS, r, world)
        want = shard.daytime_points(prof["idxday"], a, b)
        assert np.array_equal(dparts[r][: len(want)], want)
