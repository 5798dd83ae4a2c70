"""s-slab decomposition of one block, host side (no GPU).

Checks the split (plane counts, ghost-plane coordinates, sources and
receivers to the slab holding their node, refusals) and, on three gloo ranks,
the ghost-plane swap: each rank's lower ghost face receives the lower
neighbour's upper planes and its upper ghost face the upper neighbour's lower
planes, every stage, in stage order.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cases import small_case
from waveqlab3d_q_gpu_b200.slabs import block_coords, nearest_plane, split_s

CUTS = (13, 14, 13)


def _case(mesh="curvilinear"):
    return small_case(mesh=mesh, response="anelastic-Q8", pml=True, n=(21, 23, 40))


@pytest.mark.parametrize("mesh", ["cartesian", "curvilinear"])
def test_split_planes_sources_receivers(mesh):
    p = _case(mesh)
    parts = split_s(p, 3, CUTS)
    X = block_coords(p, p.blocks[0])
    assert [q.problem.blocks[0].nqrs[2] for q in parts] == list(CUTS)
    assert [q.z0 for q in parts] == [0, 13, 27]
    assert [q.open_lo for q in parts] == [False, True, True]
    assert [q.open_hi for q in parts] == [True, True, False]
    # every source and receiver lands in exactly one slab, the one holding its node
    assert sum(len(q.problem.blocks[0].sources) for q in parts) == len(p.blocks[0].sources)
    assert sorted(np.concatenate([q.rec_index for q in parts]).tolist()) == list(range(len(p.blocks[0].receivers)))
    for q in parts:
        for s in q.problem.blocks[0].sources:
            assert q.z0 <= nearest_plane(X, (s.x, s.y, s.z)) < q.z0 + q.problem.blocks[0].nqrs[2]
        if mesh == "curvilinear":
            b = q.problem.blocks[0]
            assert np.array_equal(b.coords, X[:, q.z0:q.z0 + b.nqrs[2]])
            if q.open_lo:
                assert np.array_equal(q.ghost_coords[:, :3], X[:, q.z0 - 3:q.z0])
            if q.open_hi:
                n = b.nqrs[2]
                assert np.array_equal(q.ghost_coords[:, 3:], X[:, q.z0 + n:q.z0 + n + 3])
        else:
            assert q.ghost_coords is None
        assert q.dt == p.dt()


def test_split_refusals():
    p = _case()
    with pytest.raises(ValueError):
        split_s(p, 4)                      # 10-plane slabs
    with pytest.raises(ValueError):
        split_s(p, 2, (20, 20))            # a source's delta support crosses plane 20
    with pytest.raises(ValueError):
        split_s(p, 2, (13, 13))            # counts do not add up


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class _FakeSlab:
    """Stand-in for an s-slab domain: pack writes rank-, step-, stage- and
    face-dependent planes; stage records the ghost faces that arrived."""

    def __init__(self, rank, count=6):
        self.rank, self.count = rank, count
        self.send = torch.zeros(2 * count, dtype=torch.float64)
        self.recv = torch.full((2 * count,), -1.0, dtype=torch.float64)
        self.step_no = self.stage_no = 0
        self.seen = []

    def begin_step(self, n):
        self.step_no = n

    def pack(self):
        tag = 1000.0 * self.rank + 10.0 * self.step_no + (self.stage_no % 5)
        self.send[:self.count] = tag + 0.1     # lowest planes
        self.send[self.count:] = tag + 0.2     # highest planes

    def stage(self, s, dt):
        self.seen.append((float(self.recv[0]), float(self.recv[self.count])))
        self.stage_no += 1


class _Xch:
    def __init__(self, dom, nranks):
        self.dom, self.nranks = dom, nranks

    def exchange(self):
        from waveqlab3d_q_gpu_b200.distributed import swap_faces
        self.dom.pack()
        swap_faces(self.dom.send, self.dom.recv, self.dom.count, self.dom.rank, self.nranks)


def _worker(rank, port, out, nranks):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks)
    try:
        from waveqlab3d_q_gpu_b200.distributed import slab_step
        dom = _FakeSlab(rank)
        xch = _Xch(dom, nranks)
        for n in (1, 2):
            slab_step(dom, xch, n, 0.1)
        np.save(os.path.join(out, f"r{rank}.npy"), np.array(dom.seen))
    finally:
        dist.destroy_process_group()


def test_ghost_plane_swap_three_ranks(tmp_path):
    nranks = 3
    port = _free_port()
    mp.start_processes(_worker, args=(port, str(tmp_path), nranks), nprocs=nranks, join=True, start_method="spawn")
    for r in range(nranks):
        seen = np.load(tmp_path / f"r{r}.npy")
        for i, (lo, hi) in enumerate(seen):
            n, k = 1 + i // 5, i % 5
            exp_lo = 1000.0 * (r - 1) + 10.0 * n + k + 0.2 if r > 0 else -1.0
            exp_hi = 1000.0 * (r + 1) + 10.0 * n + k + 0.1 if r < nranks - 1 else -1.0
            assert lo == pytest.approx(exp_lo) and hi == pytest.approx(exp_hi)
