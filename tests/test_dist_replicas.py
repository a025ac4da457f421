"""Replica sharding over 2 ranks with the gloo backend on CPU (no GPU needed).

The multi-GPU path of this project is "replicas only": each rank runs its own lattices and
only the measurements are combined.  This test runs the host logic of that path in two real
processes: every replica is owned by exactly one rank, results are gathered in replica order
and the timing reduction is the max over ranks.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from cudakpz_b200 import replicas
    mine = replicas.shard(n, world, rank)
    vals = [100.0 + i for i in mine]  # stand-in per-replica W^2
    allv = replicas.gather_results(n, mine, vals)
    tmax = replicas.max_over_ranks(1.5 + rank)
    q.put((rank, mine, allv, tmax))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_replica_sharding():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    n, world, port = 11, 2, _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=90) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    owned = sorted(i for _, mine, _, _ in res for i in mine)
    assert owned == list(range(n))
    for _, _, allv, tmax in res:
        assert allv == [100.0 + i for i in range(n)]
        assert tmax == 2.5


def test_shard_and_stream_ids():
    from cudakpz_b200 import replicas
    assert replicas.shard(5, 2, 0) == [0, 2, 4]
    assert replicas.shard(5, 2, 1) == [1, 3]
    assert replicas.stream_id(7) == 7
    with pytest.raises(ValueError):
        replicas.shard(5, 2, 2)
