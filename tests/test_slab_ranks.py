"""Host logic of the rank-per-GPU z-slab split (nlos_lbm/ranks.py), on CPU
with gloo at world sizes 2 and 3: the layer split, the neighbour pairing and
the point-to-point transport.  Each rank stands for its slab with a small
array of planes and sends its boundary planes as the messages; after one
exchange every halo plane must hold the neighbour's boundary plane."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from nlos_lbm import ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, nz, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    b = ranks.slab_bounds(nz, world)
    k0, k1 = b[rank], b[rank + 1]
    # global planes 0..nz+1 (halo included); plane k holds values 1000 k + column
    glob = 1000.0 * np.arange(nz + 2)[:, None] + np.arange(6)[None, :]
    mine = np.zeros((k1 - k0 + 2, 6))
    mine[1:-1] = glob[k0 + 1:k1 + 1]
    peers = ranks.neighbours(rank, world)
    send = {0: torch.from_numpy(mine[1].copy()), 1: torch.from_numpy(mine[-2].copy())}
    recv = {s: torch.zeros(6, dtype=torch.float64) for s in peers}
    send = {s: send[s] for s in peers}
    ranks.exchange_messages(dist, send, recv, peers)
    for s, t in recv.items():
        mine[0 if s == 0 else -1] = t.numpy()
    ok = True
    if 0 in peers:
        ok &= np.array_equal(mine[0], glob[k0])          # the plane just below this slab
    if 1 in peers:
        ok &= np.array_equal(mine[-1], glob[k1 + 1])     # the plane just above it
    q.put((rank, bool(ok), sorted(peers.items())))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,nz", [(2, 9), (3, 10)])
def test_cut_messages_reach_the_neighbours_halo(world, nz):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, nz, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert all(r[1] for r in res)
    assert res[0][2] == [(1, 1)] and res[-1][2] == [(0, world - 2)]


def test_slab_bounds_cover_the_grid():
    for nz, world in ((256, 8), (10, 3), (7, 7)):
        b = ranks.slab_bounds(nz, world)
        assert b[0] == 0 and b[-1] == nz and len(b) == world + 1
        sizes = np.diff(b)
        assert sizes.min() >= 1 and sizes.max() - sizes.min() <= 1
    with pytest.raises(ValueError):
        ranks.slab_bounds(3, 4)


def test_single_process_stand_in():
    one = ranks._OneRank()
    assert one.get_rank() == 0 and one.get_world_size() == 1
    parts = [None]
    one.all_gather_object(parts, "mine")
    assert parts == ["mine"]
    assert ranks.neighbours(0, 1) == {}
