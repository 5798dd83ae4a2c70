"""Host-side plumbing of the one-block-per-process run on two gloo ranks (CPU).

Checks the face swap (each rank receives the other's trace every stage, in
stage order) and the one-off material exchange, with a stand-in for the
library domain: its "stage" records what arrived, its "pack" writes a
rank- and stage-dependent trace.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class _FakeDomain:
    def __init__(self, rank, n=12):
        self.rank = rank
        self.send = torch.zeros(n, dtype=torch.float64)
        self.recv = torch.zeros(n, dtype=torch.float64)
        self.stage_no = 0
        self.step_no = 0
        self.seen = []

    def begin_step(self, n):
        self.step_no = n

    def pack_interface(self):
        self.send.fill_(100.0 * self.rank + 10.0 * self.step_no + (self.stage_no % 5) + 1)

    def stage(self, s, dt):
        self.seen.append(float(self.recv[0]))
        self.stage_no += 1


class _HostExchange:
    def __init__(self, dom, peer):
        self.dom, self.peer = dom, peer

    def exchange(self):
        from waveqlab3d_q_gpu_b200.distributed import exchange_tensors
        exchange_tensors(self.dom.send, self.dom.recv, self.peer)


def _worker(rank, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        from waveqlab3d_q_gpu_b200.distributed import exchange_array, remote_step
        peer = 1 - rank
        M = np.full((3, 4, 5), float(rank + 1))
        Mp = exchange_array(M, peer)
        dom = _FakeDomain(rank)
        xch = _HostExchange(dom, peer)
        for n in (1, 2):
            remote_step(dom, xch, n, 0.1)
        np.save(os.path.join(out, f"r{rank}.npy"), np.array([Mp.mean()] + dom.seen))
    finally:
        dist.destroy_process_group()


def test_face_swap_and_material_exchange(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0 = np.load(tmp_path / "r0.npy")
    r1 = np.load(tmp_path / "r1.npy")
    assert r0[0] == 2.0 and r1[0] == 1.0
    # each stage sees the peer's trace of that step and stage
    exp0 = [100.0 * 1 + 10.0 * n + k + 1 for n in (1, 2) for k in range(5)]
    exp1 = [100.0 * 0 + 10.0 * n + k + 1 for n in (1, 2) for k in range(5)]
    assert list(r0[1:]) == exp0
    assert list(r1[1:]) == exp1
