"""The N > 1 path on CPU: two gloo ranks agree on the row shards and on graph
placement without exchanging them, shards are disjoint and cover rows
1..kmax, and the max-over-ranks timing reduction returns the maximum."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "d-core-cuda_b200")]
    import torch
    import torch.distributed as dist
    import dcore_dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # weights as every rank derives them from the same graph
        rng = np.random.default_rng(7)
        w = np.sort(rng.integers(1, 10**6, 200))[::-1].astype(np.uint64)
        shards = dcore_dist.row_shards(w, world)
        mine = shards[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        place = dcore_dist.place_graphs(rng.integers(1, 100, 64), world)
        places = [None] * world
        dist.all_gather_object(places, place.tolist())
        t = dcore_dist.max_over_ranks(10.0 + rank, dist)
        q.put((rank, got, shards, places, t))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_ranks_agree(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, shards, places, t in res:
        assert [tuple(x) for x in got] == [tuple(x) for x in shards]  # every rank holds the same plan
        assert places[0] == places[1]
        assert t == 10.0 + world - 1
    shards = res[0][2]
    rows = [k for a, b in shards for k in range(a, b + 1)]
    assert rows == list(range(1, 200))


def test_plan_properties():
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "d-core-cuda_b200"))
    import dcore_dist
    w = np.array([100, 80, 50, 30, 20, 10, 5, 5, 5, 5, 1], np.float64)
    for world in (1, 2, 3, 4, 8, 12):
        sh = dcore_dist.row_shards(w, world)
        assert len(sh) == world
        rows = [k for a, b in sh for k in range(a, b + 1)]
        assert rows == list(range(1, 11))
    assert dcore_dist.row_shards(np.array([5.0]), 3) == [(1, 0)] * 3
    p = dcore_dist.place_graphs([5, 1, 3, 8, 2], 2)
    load = np.bincount(p, weights=[5, 1, 3, 8, 2], minlength=2)
    assert abs(load[0] - load[1]) <= 1
