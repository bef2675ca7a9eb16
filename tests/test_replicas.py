"""Multi-process host logic of the N-GPU path, run as two gloo ranks on the CPU."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from foilbench_b200.replicas import job_throughput, max_over_ranks, partition


def test_partition_is_balanced_and_complete():
    w = [5, 1, 4, 2, 3, 3, 8, 1]
    parts = partition(w, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(w)))
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)
    assert partition(w, 3) == parts
    assert partition([], 2) == [[], []]
    with pytest.raises(ValueError):
        partition(w, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r processed (r + 1) * 100 units in (r + 1) * 2 s
        t = max_over_ranks((rank + 1) * 2.0)
        rate = job_throughput((rank + 1) * 100.0, (rank + 1) * 2.0)
        mine = partition([3, 1, 2, 2], world)[rank]
        out.put((rank, t, rate, mine))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_time_and_throughput():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate, _ in res:
        assert t == 4.0  # slowest rank
        assert rate == pytest.approx(300.0 / 4.0)
    assert sorted(res[0][3] + res[1][3]) == [0, 1, 2, 3]
