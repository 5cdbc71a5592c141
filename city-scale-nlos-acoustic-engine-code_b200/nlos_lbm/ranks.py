"""One z-slab of a grid per process (a rank per GPU).

The reference decomposes its domain over MPI ranks and exchanges whole faces
every step (06_transient_localization_dx1.cpp:336-364, 837-903).  Here each
rank holds one z-slab handle (lbm_config.slab_k0 / slab_nz) and, once per
step between the halo fill and the collision, sends its neighbours only what
their next step pulls across the cut: the message lbm_slab_pack writes (the 5
populations with ez toward the neighbour of its boundary plane, and 2 x-face
ghost rows), received into the neighbour's halo plane by lbm_slab_unpack.

Transport: torch.distributed point-to-point.  With NCCL the messages stay in
device memory (NVLink between GPUs of one node); with gloo they are staged
through pinned host memory.  No collective is involved: each cut is one
message each way between two neighbours.
"""
import numpy as np

from . import abi
from .solver import Solver


def slab_bounds(nz, world):
    """Layer boundaries of `world` near-equal z-slabs of nz layers."""
    if world < 1 or world > nz:
        raise ValueError("need 1 <= world <= nz")
    return [round(i * nz / world) for i in range(world + 1)]


def neighbours(rank, world):
    """{side: peer rank}: side 0 is the slab below, side 1 the slab above."""
    out = {}
    if rank > 0:
        out[0] = rank - 1
    if rank < world - 1:
        out[1] = rank + 1
    return out


def exchange_messages(dist, send, recv, peers, group=None):
    """Send send[side] to peers[side] and receive recv[side] from it, for
    every side at once (non-blocking point-to-point, so the ranks cannot
    deadlock on the order); returns when all have completed."""
    ops = []
    for side, peer in peers.items():
        ops.append(dist.P2POp(dist.isend, send[side], peer, group))
        ops.append(dist.P2POp(dist.irecv, recv[side], peer, group))
    if not ops:
        return
    for r in dist.batch_isend_irecv(ops):
        r.wait()


class _OneRank:
    """The torch.distributed calls SlabRank makes, for a process that runs alone
    (no process group): rank 0 of 1, and a gather that returns its own part."""

    @staticmethod
    def get_rank(group=None):
        return 0

    @staticmethod
    def get_world_size(group=None):
        return 1

    @staticmethod
    def all_gather_object(parts, obj, group=None):
        parts[0] = obj


class SlabRank:
    """This rank's z-slab of the grid `cfg`, stepped with the reference's
    loop body (source, halo fill, cut messages, collision, probes).

    dist: torch.distributed, initialised, or None for one process holding the
    whole grid (no cut, no messages); rank/world from it.  staging:
    "device" (NCCL: messages sent from device memory) or "host" (any
    backend: messages copied through pinned host memory)."""

    def __init__(self, cfg, dist, sources=(), probes=None, triangles=None, device=0, staging="device", group=None):
        import torch

        self.torch = torch
        self.dist = dist if dist is not None else _OneRank()
        self.group = group
        self.rank = self.dist.get_rank(group)
        self.world = self.dist.get_world_size(group)
        nz = int((cfg.z_max - cfg.z_min) / cfg.dx + 0.5)
        self.bounds = slab_bounds(nz, self.world)
        c = abi.LbmConfig.from_buffer_copy(cfg)
        c.slab_k0 = self.bounds[self.rank]
        c.slab_nz = self.bounds[self.rank + 1] - self.bounds[self.rank]
        c.device = device
        self.solver = Solver(c, sources, probes, triangles=triangles)
        self.lib, self.h = self.solver.lib, self.solver.h
        self.peers = neighbours(self.rank, self.world)
        nbytes = self.lib.lbm_slab_message_bytes(self.h) if self.world > 1 else 0
        dev = torch.device("cuda", device)
        self.staging = staging
        self.send = {s: torch.empty(nbytes, dtype=torch.uint8, device=dev) for s in self.peers}
        self.recv = {s: torch.empty(nbytes, dtype=torch.uint8, device=dev) for s in self.peers}
        if staging == "host":
            self.send_h = {s: torch.empty(nbytes, dtype=torch.uint8).pin_memory() for s in self.peers}
            self.recv_h = {s: torch.empty(nbytes, dtype=torch.uint8).pin_memory() for s in self.peers}
        self.stream = torch.cuda.ExternalStream(self.solver.stream, device=dev)
        self.steps = 0

    def _check(self, st, what):
        return self.solver._check(st, what)

    def _transfer(self):
        torch = self.torch
        if self.staging == "host":
            with torch.cuda.stream(self.stream):
                for s in self.peers:
                    self.send_h[s].copy_(self.send[s], non_blocking=True)
            self.stream.synchronize()
            exchange_messages(self.dist, self.send_h, self.recv_h, self.peers, self.group)
            with torch.cuda.stream(self.stream):
                for s in self.peers:
                    self.recv[s].copy_(self.recv_h[s], non_blocking=True)
            return
        # device messages: the transfer's stream waits for the packs, the
        # library's stream for the transfer
        cur = torch.cuda.current_stream(self.stream.device)
        cur.wait_stream(self.stream)
        exchange_messages(self.dist, self.send, self.recv, self.peers, self.group)
        self.stream.wait_stream(cur)

    def step(self, n=1):
        s = self.solver
        for _ in range(int(n)):
            s.apply_source(self.steps * s.dt)
            s.exchange_halos()
            for side in self.peers:
                self._check(self.lib.lbm_slab_pack(self.h, side, self.send[side].data_ptr()), "lbm_slab_pack")
            self._transfer()
            for side in self.peers:
                self._check(self.lib.lbm_slab_unpack(self.h, side, self.recv[side].data_ptr()), "lbm_slab_unpack")
            s.step_collision_bgk()
            s.record_probes()
            self.steps += 1

    def get_probes(self):
        """[step][probe] of the whole grid, on every rank: each probe from the
        rank whose slab holds its cell (NaN outside the grid)."""
        mine = self.solver.get_probes()
        parts = [None] * self.world
        self.dist.all_gather_object(parts, mine, group=self.group)
        out = parts[0].copy()
        for p in parts[1:]:
            out = np.where(np.isnan(out), p, out)
        return out

    def close(self):
        """Frees the message buffers (after the library's stream has finished
        with them) and then the slab handle.  Pinned host buffers record an
        event on the streams that used them when they are freed, so they must
        go while the CUDA context is alive: call close() before the process
        ends rather than leaving them to interpreter shutdown."""
        if getattr(self, "solver", None) is None:
            return
        self.stream.synchronize()
        self.send, self.recv = {}, {}
        self.send_h, self.recv_h = {}, {}
        self.torch.cuda.synchronize(self.stream.device)
        self.solver.close()
        self.solver = None
