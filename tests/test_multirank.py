"""The multi-GPU plumbing of bench.py on CPU: two gloo ranks (127.0.0.1).

Checks the reductions the bench takes over ranks (max of device times, sum of
cell-steps) and the film partition of the batched legs: every film is advanced by
exactly one rank, the same on every rank, with balanced transform cost."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "llg-sim_b200"))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    import workloads as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank
        mx = bench.reduce_over_ranks(dist, local_ms, "max", "cpu")
        sm = bench.reduce_over_ranks(dist, 100.0 * (rank + 1), "sum", "cpu")
        films, _ = W.mixed_film_batch(256)
        mine = W.partition_films(films, world, rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out.put((rank, mx, sm, gathered))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_partition():
    import multiprocessing as mp

    import workloads as W

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    films, _ = W.mixed_film_batch(256)
    for rank, mx, sm, gathered in res:
        assert mx == 15.0            # slowest rank's time
        assert sm == 300.0           # all ranks' work
        flat = sorted(i for part in gathered for i in part)
        assert flat == list(range(len(films)))       # each film exactly once
        assert gathered[rank] == W.partition_films(films, world, rank)
        loads = [sum(W.film_cost(films[i]) for i in part) for part in gathered]
        assert max(loads) / min(loads) < 1.05


@pytest.mark.parametrize("world", [1, 3, 8])
def test_partition_covers_and_balances(world):
    import workloads as W

    films, _ = W.mixed_film_batch(256)
    parts = [W.partition_films(films, world, r) for r in range(world)]
    assert sorted(i for p in parts for i in p) == list(range(256))
    loads = [sum(W.film_cost(films[i]) for i in p) for p in parts]
    assert max(loads) / (sum(loads) / world) < 1.05
