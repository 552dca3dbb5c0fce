"""Replicas-only multi-GPU host logic, on CPU: two gloo ranks run the timing
collectives the bench uses (barrier, max over ranks), take distinct seeds and
disjoint right-hand-side shards.  No GPU and no data-path collective."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from multigrid_meshless_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = replicas.Timing(dist)
        t.barrier()
        mx = t.max_over_ranks(10.0 + rank)      # per-rank "device time"
        start, stop = replicas.shard(64, world, rank)
        q.put((rank, mx, replicas.replica_seed(1, rank), start, stop))
        t.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_and_shard():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [11.0, 11.0]          # max over ranks on every rank
    assert out[0][2] != out[1][2]                         # one cloud seed per replica
    assert out[0][3:] == (0, 32) and out[1][3:] == (32, 64)


@pytest.mark.parametrize("count,world", [(64, 1), (64, 3), (7, 4), (0, 2), (3, 8)])
def test_shards_cover_once(count, world):
    seen = []
    sizes = []
    for r in range(world):
        a, b = replicas.shard(count, world, r)
        seen.extend(range(a, b))
        sizes.append(b - a)
    assert seen == list(range(count))
    assert max(sizes) - min(sizes) <= 1


def test_no_group_is_identity():
    t = replicas.Timing(None)
    t.barrier()
    assert t.max_over_ranks(3.5) == 3.5
    assert replicas.replica_seed(1, 0) == 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)
