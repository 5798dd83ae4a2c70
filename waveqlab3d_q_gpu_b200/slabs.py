"""One block split into s-slabs, one slab per domain.

The reference decomposes a block over MPI ranks and fills the 3 ghost
layers of every field from the neighbours before each stage
(src/mpi3dcomm.f90:459-528, called from src/fields.f90:306-321).  Here a
one-block problem is cut along s into slabs: slab r holds the global planes
``z0 + 1 .. z0 + ns`` as a domain with ``slab`` set; its faces inside the
block are open (no boundary condition or PML, central SBP rows up to the
face, 3 ghost planes).  Before every stage each slab packs the 3 planes next
to its open faces, the planes go to the neighbours, and each slab unpacks
them into its ghost planes; the metric (and J) ghost planes are exchanged once
after set-up.

:func:`split_s` builds the slab problems.  Sources and receivers go to the
slab that holds their nearest node (a source's delta support must lie inside
that slab).  :class:`SlabSet` runs all slabs of a problem in one process on
one device (the exchange is a device copy between the domains' buffers);
:class:`waveqlab3d_q_gpu_b200.distributed.SlabRank` runs one slab per process.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

HALO_FIELDS = 0
HALO_METRIC = 1


@dataclass
class SlabPart:
    """Slab r of a split block: its problem, global plane offset, the block's
    plane count, the ghost-plane coordinates (curvilinear) and the time step
    of the whole problem."""
    problem: object
    rank: int
    z0: int
    ns_global: int
    ghost_coords: Optional[np.ndarray]
    dt: float
    rec_index: np.ndarray          # indices of the whole problem's receivers held here

    @property
    def open_lo(self) -> bool:
        return self.z0 > 0

    @property
    def open_hi(self) -> bool:
        return self.z0 + self.problem.blocks[0].nqrs[2] < self.ns_global


def block_coords(problem, b) -> np.ndarray:
    """(3, ns, nr, nq) node coordinates of block b (Cartesian grids from aqrs/bqrs)."""
    nq, nr, ns = b.nqrs
    if problem.type_of_mesh == "curvilinear":
        return np.asarray(b.coords, dtype=np.float64)
    ax = [b.aqrs[c] + np.arange(n) * ((b.bqrs[c] - b.aqrs[c]) / (n - 1)) for c, n in enumerate((nq, nr, ns))]
    X = np.empty((3, ns, nr, nq))
    X[0] = ax[0][None, None, :]
    X[1] = ax[1][None, :, None]
    X[2] = ax[2][:, None, None]
    return X


def nearest_plane(X: np.ndarray, xyz: Sequence[float]) -> int:
    """0-based s index of the node nearest to xyz (the last of equal
    distances in s, r, q order, as the library's search takes)."""
    d = (X[0] - xyz[0]) ** 2 + (X[1] - xyz[1]) ** 2 + (X[2] - xyz[2]) ** 2
    flat = d.ravel()
    i = flat.size - 1 - int(np.argmin(flat[::-1]))
    return i // (X.shape[2] * X.shape[3])


def split_s(problem, nslabs: int, cuts: Optional[Sequence[int]] = None) -> List[SlabPart]:
    """Cut the one block of ``problem`` into ``nslabs`` s-slabs (``cuts``: the
    global plane counts of the slabs, default as even as possible)."""
    if len(problem.blocks) != 1:
        raise ValueError("split_s takes a one-block problem")
    if problem.mms is not None:
        raise ValueError("manufactured-solution runs are not split")
    b = problem.blocks[0]
    nq, nr, ns = b.nqrs
    if cuts is None:
        base, extra = divmod(ns, nslabs)
        cuts = [base + (1 if r < extra else 0) for r in range(nslabs)]
    if sum(cuts) != ns or len(cuts) != nslabs:
        raise ValueError("slab plane counts must add up to the block's")
    if min(cuts) < 13:
        raise ValueError("each slab needs at least 13 planes")
    X = block_coords(problem, b)
    half = 4 if problem.source_order == 4 else 2
    z0s = np.concatenate([[0], np.cumsum(cuts)[:-1]]).astype(int)
    src_rank = []
    for s in b.sources:
        zs = nearest_plane(X, (s.x, s.y, s.z))
        r = int(np.searchsorted(z0s, zs, side="right") - 1)
        if zs - half < z0s[r] or zs + half >= z0s[r] + cuts[r]:
            raise ValueError(f"source at plane {zs + 1} has delta support across a slab boundary")
        src_rank.append(r)
    rec = np.zeros((0, 3)) if b.receivers is None else np.asarray(b.receivers, dtype=np.float64)
    rec_rank = np.array([int(np.searchsorted(z0s, nearest_plane(X, p), side="right") - 1) for p in rec], dtype=int)
    dt = problem.dt()
    parts = []
    for r in range(nslabs):
        z0, n = int(z0s[r]), int(cuts[r])
        sl = slice(z0, z0 + n)
        nb = copy.copy(b)
        nb.nqrs = (nq, nr, n)
        if b.coords is not None:
            nb.coords = np.ascontiguousarray(np.asarray(b.coords)[:, sl])
        if b.material is not None:
            nb.material = np.ascontiguousarray(np.asarray(b.material)[:, sl])
        if b.qs_inv is not None:
            nb.qs_inv = np.ascontiguousarray(np.asarray(b.qs_inv)[sl])
        if b.qp_inv is not None:
            nb.qp_inv = np.ascontiguousarray(np.asarray(b.qp_inv)[sl])
        nb.sources = [s for s, sr in zip(b.sources, src_rank) if sr == r]
        idx = np.nonzero(rec_rank == r)[0]
        nb.receivers = rec[idx] if len(idx) else None
        gc = None
        if problem.type_of_mesh == "curvilinear":
            gc = np.zeros((3, 6, nr, nq))
            for k in range(6):
                zg = z0 - 3 + k if k < 3 else z0 + n + (k - 3)
                if 0 <= zg < ns:
                    gc[:, k] = X[:, zg]
        p = copy.copy(problem)
        p.blocks = [nb]
        parts.append(SlabPart(problem=p, rank=r, z0=z0, ns_global=ns, ghost_coords=gc, dt=dt, rec_index=idx))
    return parts


class SlabSet:
    """All slabs of a split block on one device in one process: the ghost
    planes move between the domains' buffers by device copies between
    stages (no kernel waits on another)."""

    def __init__(self, problem, nslabs: int, precision: str = "fp64", nsteps_hint: Optional[int] = None,
                 cuts: Optional[Sequence[int]] = None):
        import torch

        from .distributed import _DeviceArray
        from .domain import Domain
        self.parts = split_s(problem, nslabs, cuts)
        self.domains = [Domain(p.problem, precision=precision, nsteps_hint=nsteps_hint, slab=p) for p in self.parts]
        self.dt = self.parts[0].dt
        self.n = 1
        self._views = {}
        for kind in (HALO_FIELDS, HALO_METRIC):
            v = []
            for d in self.domains:
                snd, rcv, cnt, eb = d.halo_buffers(kind)
                v.append((torch.as_tensor(_DeviceArray(snd, 2 * cnt, eb), device="cuda"),
                          torch.as_tensor(_DeviceArray(rcv, 2 * cnt, eb), device="cuda"), cnt))
            self._views[kind] = v
        self.exchange(HALO_METRIC)

    def exchange(self, kind: int = HALO_FIELDS):
        """Pack every slab's planes, move them to the neighbours, unpack."""
        import torch
        for d in self.domains:
            d.pack_halo(kind)
        for d in self.domains:
            d.synchronize()
        v = self._views[kind]
        for r in range(len(self.domains) - 1):
            send_b, recv_b, c = v[r]          # slab r (below); buffers are [lower face | upper face]
            send_a, recv_a, _ = v[r + 1]      # slab r + 1 (above)
            recv_b[c:2 * c].copy_(send_a[0:c])    # r's upper ghost planes <- r+1's lowest planes
            recv_a[0:c].copy_(send_b[c:2 * c])    # r+1's lower ghost planes <- r's highest planes
        torch.cuda.synchronize()
        for d in self.domains:
            d.unpack_halo(kind)

    def step(self):
        for d in self.domains:
            d.begin_step(self.n)
        for s in range(1, 6):
            self.exchange(HALO_FIELDS)
            for d in self.domains:
                d.stage(s, self.dt)
        self.n += 1

    def run(self, nsteps: int):
        for _ in range(nsteps):
            self.step()
        for d in self.domains:
            d.synchronize()

    def fields(self) -> np.ndarray:
        """(9, ns, nr, nq) fields of the whole block."""
        return np.concatenate([d.fields(0) for d in self.domains], axis=1)

    def seismograms(self) -> List[np.ndarray]:
        return [d.seismograms(0) for d in self.domains]

    def close(self):
        for d in self.domains:
            d.synchronize()
        self._views = {}
        import gc
        gc.collect()
        for d in self.domains:
            d.close()
