"""Multi-rank host logic of the replica mode, run as world_size-2 gloo process groups on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from pfsoftlib_b200 import replicas


def test_shard_covers_every_transform_once():
    bw = [32, 48, 64, 96, 128] * 20 + [16, 256]
    for world in (1, 2, 3, 8):
        plan = replicas.shard(bw, world)
        got = sorted(i for lst in plan for i in lst)
        assert got == list(range(len(bw)))
    assert replicas.imbalance(bw, replicas.shard(bw, 4)) < 1.1


def test_shard_is_deterministic():
    bw = [64, 32, 128, 96] * 5
    assert replicas.shard(bw, 3) == replicas.shard(list(bw), 3)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    bw = [32, 48, 64, 96, 128] * 4
    plan = replicas.shard(bw, world)          # every rank computes the same plan
    mine = plan[rank]
    elapsed = 1.0 + rank                       # a stand-in per-rank device time
    worst = replicas.max_over_ranks(elapsed)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mine, worst))


def test_two_rank_gloo_plan_and_max_timing():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert out[0][2] == out[1][2] == 2.0      # max over ranks
    assert sorted(out[0][1] + out[1][1]) == list(range(20))
    assert set(out[0][1]).isdisjoint(out[1][1])
