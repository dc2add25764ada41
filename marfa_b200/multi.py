"""Several GPUs of one node: one process per GPU, no collective on the data path.

The units of the line-by-line computation -- (profile, level, subinterval) --
are independent and share only the read-only line list, so a computation
spreads over GPUs by giving each rank its own levels (or its own profiles).
Each rank computes and keeps its records; nothing is exchanged but the
timing of the benchmark (a barrier and a max over ranks) and the work counts.
"""
from __future__ import annotations

from typing import List, Sequence


def level_shards(n_levels: int, world: int) -> List[range]:
    """Contiguous level ranges, one per rank, sizes differing by at most one;
    together they cover range(n_levels) exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    base, extra = divmod(n_levels, world)
    out, start = [], 0
    for r in range(world):
        size = base + (1 if r < extra else 0)
        out.append(range(start, start + size))
        start += size
    return out


def shard_profile(pressure: Sequence[float], temperature: Sequence[float], density: Sequence[float],
                  rank: int, world: int):
    """This rank's levels of one profile: (levels, P, T, n)."""
    import numpy as np
    lv = level_shards(len(pressure), world)[rank]
    sl = slice(lv.start, lv.stop)
    return lv, (np.asarray(pressure)[sl], np.asarray(temperature)[sl], np.asarray(density)[sl])


def reduce_step(ms: float, evals: int, dist=None):
    """Benchmark reduction over ranks: the slowest rank's milliseconds per
    step and the evaluations of all ranks (world-wide throughput =
    evals / ms).  Without a process group, the local values."""
    if dist is None or not dist.is_initialized():
        return float(ms), int(evals)
    import torch
    backend = dist.get_backend()
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    e = torch.tensor([int(evals)], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t.item()), int(e.item())
