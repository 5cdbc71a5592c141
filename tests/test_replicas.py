"""Multi-process (world size 2, gloo on CPU) check of bench.py's replica
aggregation: every rank runs an independent replica, the job time is the
maximum over ranks and the value counts all ranks' cell updates."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    barrier, reduce_max = bench.make_reducers(dist, "cpu")
    barrier()
    local_ms = 100.0 + 50.0 * rank           # rank 1 is the slow one
    ms = reduce_max(local_ms)
    q.put((rank, ms, bench.replica_glups(world, 1000, 10, ms)))
    barrier()
    dist.destroy_process_group()


def test_replica_aggregation_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [150.0, 150.0]                    # max over ranks, on every rank
    assert res[0][2] == pytest.approx(2 * 1000 * 10 / 0.150 / 1e9)  # all ranks' cell updates


def test_single_rank_reducers_are_identity():
    barrier, reduce_max = bench.make_reducers(None, "cpu")
    barrier()
    assert reduce_max(3.5) == 3.5
