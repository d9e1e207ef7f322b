"""Sharding of energy points over ranks: the assignment (deterministic longest-first) and the
gather, run as two gloo ranks on the CPU with a stand-in for the per-rank GPU evaluation."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from dwba_b200.distributed import partition_points, point_cost, radial_ME_all_L_sweep_distributed


class _Grid:
    def __init__(self, n):
        self.r = np.linspace(0.01, 10.0, n)


def _points():
    rng = np.random.default_rng(3)
    pts = []
    for e in range(13):
        n = int(200 + 2000 * rng.random())
        pts.append(dict(grid=_Grid(n), bound_i=object(), pairs=[(e, q) for q in range(1 + e % 4)]))
    return pts


def _fake_compute(points, L_max):
    # stands in for the GPU sweep: a value that identifies the point and the pair
    return [[(len(pt["grid"].r), p, L_max) for p in pt["pairs"]] for pt in points]


def test_partition_is_a_balanced_cover():
    costs = [point_cost(p) for p in _points()]
    for world in (1, 2, 3, 8):
        parts = partition_points(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: max load <= mean + largest job
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
    assert partition_points(costs, 2) == partition_points(costs, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = radial_ME_all_L_sweep_distributed(_points(), 4, compute=_fake_compute)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_gather_every_point_in_order():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    want = _fake_compute(_points(), 4)
    assert results[0] == want and results[1] == want
