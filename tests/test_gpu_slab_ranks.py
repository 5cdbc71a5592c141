"""The rank-per-GPU z-slab path (nlos_lbm/ranks.py: lbm_slab_pack /
lbm_slab_unpack and point-to-point messages) with two processes, gloo, the
messages staged through host memory, both slabs on the one GPU this suite
has: the split run reproduces the undivided run bit for bit.  No kernel of
one process waits for the other's (the exchange is on the host), so the two
processes may share the GPU.  The NCCL transport between GPUs (device
messages) is the same code with staging="device"; it needs two GPUs."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, name, storage, steps, q):
    import datetime

    sys.path[:0] = [REPO, os.path.join(REPO, "city-scale-nlos-acoustic-engine-code_b200"), os.path.join(REPO, "tests")]
    import torch
    import torch.distributed as dist

    import scenarios
    from nlos_lbm import abi, ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    kw = dict(storage=abi.LBM_STORE_F16, f16_scale=1e3) if storage == "fp16" else {}
    sc = scenarios.scenario(name, **kw)
    r = ranks.SlabRank(sc["cfg"], dist, sc["sources"], sc["probes"], triangles=sc["triangles"], device=0,
                       staging="host")
    r.step(steps)
    p = r.get_probes()
    rho = r.solver.get_rho()
    q.put((rank, p, rho, r.bounds))
    dist.barrier()
    r.close()
    del r
    dist.destroy_process_group()
    torch.cuda.synchronize()


@pytest.mark.parametrize("name,storage,world", [("city_small", "fp32", 2), ("scatter_small", "fp16", 2),
                                                ("scatter_small", "fp32", 3)])
def test_rank_split_is_bit_identical(name, storage, world, gpu):
    import scenarios
    from nlos_lbm import Solver, abi

    steps = 40
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, name, storage, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=600) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    kw = dict(storage=abi.LBM_STORE_F16, f16_scale=1e3) if storage == "fp16" else {}
    sc = scenarios.scenario(name, **kw)
    g = Solver(sc["cfg"], sc["sources"], sc["probes"], triangles=sc["triangles"])
    g.step(steps)
    assert np.max(np.abs(g.get_probes())) > 0
    for _, p, _, _ in res:
        assert np.array_equal(p, g.get_probes(), equal_nan=True)
    assert np.array_equal(np.concatenate([r[2] for r in res], axis=0), g.get_rho())
