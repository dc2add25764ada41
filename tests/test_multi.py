"""The multi-GPU host logic with two CPU ranks over gloo: level shards cover
every level exactly once, and the benchmark reduction takes the slowest
rank's time and the sum of the work."""
import os
import socket

import pytest

from marfa_b200.multi import level_shards


def test_level_shards_cover_once():
    for n in (1, 7, 40, 200):
        for world in (1, 2, 3, 8):
            shards = level_shards(n, world)
            assert len(shards) == world
            flat = [i for r in shards for i in r]
            assert flat == list(range(n))
            sizes = [len(r) for r in shards]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist
    from marfa_b200.multi import reduce_step, shard_profile
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = np.linspace(1.0, 40.0, 40)
        lv, (p, t, n) = shard_profile(P, P + 200.0, P * 10.0, rank, world)
        # each rank reports its own time and work
        ms, ev = reduce_step(10.0 + rank, 1000 * len(lv), dist)
        got = [None] * world
        dist.all_gather_object(got, (lv.start, lv.stop, float(p[0])))
        q.put((rank, ms, ev, got))
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo():
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, ev, got in results:
        assert ms == 11.0                 # slowest rank
        assert ev == 1000 * 40            # work of both ranks
        assert [(a, b) for a, b, _ in got] == [(0, 20), (20, 40)]
        assert got[1][2] == 21.0          # rank 1 starts at level 21 of the profile
