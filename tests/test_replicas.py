"""Multi-process (world size 2, gloo, CPU) check of the replica reduction
that bench.py applies across ranks, and of the unit sharding."""
import os
import socket

import pytest

from yafray_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t, u = replicas.combine(1.5 + rank, 1000.0 * (rank + 1))
    dist.destroy_process_group()
    q.put((rank, t, u))


def test_combine_two_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, u in out:
        assert t == pytest.approx(2.5)   # slowest rank
        assert u == pytest.approx(3000.0)  # all ranks' rays


def test_combine_without_group_is_identity():
    assert replicas.combine(2.0, 7.0) == (2.0, 7.0)


@pytest.mark.parametrize("n,world", [(0, 2), (1, 2), (7, 3), (256, 8), (5, 8)])
def test_shard_covers_once(n, world):
    seen = []
    sizes = []
    for r in range(world):
        rg = replicas.shard(n, r, world)
        seen += list(rg)
        sizes.append(len(rg))
    assert seen == list(range(n))
    assert max(sizes) - min(sizes) <= 1
