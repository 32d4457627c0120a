"""Column sharding across GPUs (one process per GPU).

RRTMG-LW columns are independent (radlw_main.F90:782 loops over columns with
no exchange), and so are RRTMG-SW's daytime points (radsw_main.F90:892), so
a multi-GPU run gives each rank whole physics blocks of consecutive columns
and needs no collective on the data path.  The only
collective a run makes is the reduction of per-rank timings (max over ranks)
outside the timed region.
"""
from __future__ import annotations

import numpy as np


def column_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [start, stop) of `total` columns owned by `rank`; the first
    total % world ranks get one extra column."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def block_range(block_sizes, rank: int, world: int) -> tuple[int, int]:
    """Whole physics blocks [b0, b1) for `rank`, cut where the running column
    count crosses rank/world of the total, so every rank gets about the same
    number of columns and no block is split."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    total = sum(block_sizes)
    cuts, acc, r = [0], 0, 1
    for i, n in enumerate(block_sizes):
        acc += n
        while r < world and acc * world >= r * total:
            cuts.append(i + 1)
            r += 1
    while len(cuts) < world + 1:
        cuts.append(len(block_sizes))
    cuts[world] = len(block_sizes)
    return cuts[rank], cuts[rank + 1]


def daytime_points(idxday, start: int, stop: int) -> np.ndarray:
    """The daytime points of rrtmg_sw_run (idxday: 1-based column indices,
    any order) that fall in the shard of columns [start, stop), renumbered
    within the shard and kept in their order."""
    idx = np.asarray(idxday, dtype=np.int64)
    return (idx[(idx > start) & (idx <= stop)] - start).astype(np.int32)
