"""One block (or one s-slab of a block) per process.

The reference runs a two-block problem with one MPI rank per block and
exchanges the interface face every RK stage (exchange_fields_interface and
exchange_materials_interface, src/domain.f90:696-754).  Here each process
(one per GPU, torch.distributed) holds one block as a :class:`Domain` with
``remote_block`` set; every stage it packs its face trace into the library's
send buffer, swaps it with the peer, and runs the stage, whose interface
kernel reads the peer's trace and computes this side only.  Each process
keeps its own fault slip state and adds to it once per stage, like each
rank of the reference.

Backends: ``nccl`` exchanges the device buffers directly on the domain's
stream; ``gloo`` goes through host copies (CPU-only plumbing and single-GPU
runs of both ranks).
"""
from __future__ import annotations

from typing import Optional

import numpy as np


class _DeviceArray:
    """Zero-copy view of a library device buffer for torch (__cuda_array_interface__)."""

    def __init__(self, ptr: int, n: int, elem_bytes: int):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8" if elem_bytes == 8 else "<f4",
                                         "data": (int(ptr), False), "version": 3, "strides": None,
                                         "stream": None}


def exchange_tensors(send, recv, peer: int):
    """Swap ``send`` with the peer's and receive its into ``recv`` (same shape)."""
    import torch.distributed as dist
    ops = [dist.P2POp(dist.isend, send, peer), dist.P2POp(dist.irecv, recv, peer)]
    for w in dist.batch_isend_irecv(ops):
        w.wait()


def exchange_array(a: np.ndarray, peer: int, device=None) -> np.ndarray:
    """The peer's copy of a same-shaped host array (set-up data such as the
    face material)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
    if device is not None:
        t = t.to(device)
    r = torch.empty_like(t)
    exchange_tensors(t, r, peer)
    return r.cpu().numpy()


class FaceExchange:
    """The per-stage face swap of one process."""

    def __init__(self, domain, peer: int, backend: str):
        import torch
        self.domain = domain
        self.peer = peer
        self.backend = backend
        snd, rcv, count, eb = domain.interface_buffers()
        self.count = count
        dtype = torch.float64 if eb == 8 else torch.float32
        self.send = torch.as_tensor(_DeviceArray(snd, count, eb), device="cuda")
        self.recv = torch.as_tensor(_DeviceArray(rcv, count, eb), device="cuda")
        self.stream = torch.cuda.ExternalStream(domain.stream_handle())
        if backend == "gloo":
            self.hsend = torch.empty(count, dtype=dtype, pin_memory=True)
            self.hrecv = torch.empty(count, dtype=dtype, pin_memory=True)

    def exchange(self):
        import torch
        if self.backend == "nccl":
            with torch.cuda.stream(self.stream):
                exchange_tensors(self.send, self.recv, self.peer)
        else:
            with torch.cuda.stream(self.stream):
                self.hsend.copy_(self.send, non_blocking=True)
            self.stream.synchronize()
            exchange_tensors(self.hsend, self.hrecv, self.peer)
            with torch.cuda.stream(self.stream):
                self.recv.copy_(self.hrecv, non_blocking=True)


def remote_step(domain, xch, n: int, dt: float):
    """Time step n of a remote-interface domain: the stage-1 receiver sample,
    then per RK stage: pack the face trace, swap it with the peer, run the
    stage (time_step.f90:109-147 with exchange_fields_interface between)."""
    domain.begin_step(n)
    for s in range(1, 6):
        domain.pack_interface()
        xch.exchange()
        domain.stage(s, dt)


class BlockRank:
    """Block ``rank`` (0 or 1) of a two-block problem on this process; its peer
    holds the other block (process 1 - rank, or ``peer`` when several pairs
    share the process group)."""

    def __init__(self, problem, rank: int, backend: str = "nccl", precision: str = "fp64",
                 nsteps_hint: Optional[int] = None, exchange=None, peer: Optional[int] = None):
        from .domain import Domain
        self.rank = rank
        self.peer = 1 - rank if peer is None else peer
        self.domain = Domain(problem, precision=precision, nsteps_hint=nsteps_hint, remote_block=rank)
        dev = "cuda" if backend == "nccl" else None
        Mpeer = exchange_array(self.domain.interface_material(), self.peer, device=dev)
        self.domain.set_interface_remote_material(Mpeer)
        self.xch = exchange if exchange is not None else FaceExchange(self.domain, self.peer, backend)
        self.n = 1

    def step(self, dt: Optional[float] = None):
        """One time step: sample, then per stage pack / swap / stage."""
        d = self.domain
        remote_step(d, self.xch, self.n, d.dt if dt is None else dt)
        self.n += 1

    def run(self, nsteps: int, dt: Optional[float] = None):
        for _ in range(nsteps):
            self.step(dt)

    def close(self):
        """Release the exchange buffers while the domain's stream exists (torch
        records an event on it when a pinned buffer used there is freed), then
        the domain."""
        import gc

        import torch
        self.domain.synchronize()
        self.xch = None
        gc.collect()
        torch.cuda.synchronize()
        self.domain.close()


def swap_faces(send, recv, count: int, rank: int, nranks: int):
    """Ghost-plane swap of s-slab ``rank``: the lower face of ``send`` goes to
    rank - 1, whose upper face arrives in the lower face of ``recv``, and the
    upper face to rank + 1 (buffers [lower face | upper face] of ``count``
    elements each)."""
    import torch.distributed as dist
    c = count
    ops = []
    if rank > 0:
        ops += [dist.P2POp(dist.isend, send[0:c], rank - 1), dist.P2POp(dist.irecv, recv[0:c], rank - 1)]
    if rank < nranks - 1:
        ops += [dist.P2POp(dist.isend, send[c:2 * c], rank + 1), dist.P2POp(dist.irecv, recv[c:2 * c], rank + 1)]
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


class HaloExchange:
    """The per-stage ghost-plane swap of one s-slab process with its lower
    (rank - 1) and upper (rank + 1) neighbours; buffers are [lower face |
    upper face] (wql3d_halo_buffers)."""

    def __init__(self, domain, rank: int, nranks: int, backend: str, kind: int):
        import torch
        self.domain, self.rank, self.nranks, self.backend, self.kind = domain, rank, nranks, backend, kind
        snd, rcv, count, eb = domain.halo_buffers(kind)
        self.count = count
        dtype = torch.float64 if eb == 8 else torch.float32
        self.send = torch.as_tensor(_DeviceArray(snd, 2 * count, eb), device="cuda")
        self.recv = torch.as_tensor(_DeviceArray(rcv, 2 * count, eb), device="cuda")
        self.stream = torch.cuda.ExternalStream(domain.stream_handle())
        if backend == "gloo":
            self.hsend = torch.empty(2 * count, dtype=dtype, pin_memory=True)
            self.hrecv = torch.empty(2 * count, dtype=dtype, pin_memory=True)

    def _swap(self, send, recv):
        swap_faces(send, recv, self.count, self.rank, self.nranks)

    def exchange(self):
        import torch
        d = self.domain
        d.pack_halo(self.kind)
        if self.backend == "nccl":
            with torch.cuda.stream(self.stream):
                self._swap(self.send, self.recv)
        else:
            with torch.cuda.stream(self.stream):
                self.hsend.copy_(self.send, non_blocking=True)
            self.stream.synchronize()
            self._swap(self.hsend, self.hrecv)
            with torch.cuda.stream(self.stream):
                self.recv.copy_(self.hrecv, non_blocking=True)
        d.unpack_halo(self.kind)


def slab_step(domain, xch, n: int, dt: float):
    """Time step n of an s-slab domain: the stage-1 receiver sample, then per
    RK stage the ghost-plane exchange and the stage."""
    domain.begin_step(n)
    for s in range(1, 6):
        xch.exchange()
        domain.stage(s, dt)


class SlabRank:
    """s-slab ``rank`` of ``nranks`` of a one-block problem on this process
    (one slab per GPU, torch.distributed for the ghost planes)."""

    def __init__(self, problem, rank: int, nranks: int, backend: str = "nccl", precision: str = "fp64",
                 nsteps_hint: Optional[int] = None, cuts=None):
        from .domain import Domain
        from .slabs import HALO_FIELDS, HALO_METRIC, split_s
        self.rank, self.nranks = rank, nranks
        self.part = split_s(problem, nranks, cuts)[rank]
        self.domain = Domain(self.part.problem, precision=precision, nsteps_hint=nsteps_hint, slab=self.part)
        HaloExchange(self.domain, rank, nranks, backend, HALO_METRIC).exchange()
        self.xch = HaloExchange(self.domain, rank, nranks, backend, HALO_FIELDS)
        self.n = 1

    def step(self):
        slab_step(self.domain, self.xch, self.n, self.domain.dt)
        self.n += 1

    def run(self, nsteps: int):
        for _ in range(nsteps):
            self.step()

    def close(self):
        import gc

        import torch
        self.domain.synchronize()
        self.xch = None
        gc.collect()
        torch.cuda.synchronize()
        self.domain.close()
