"""The gradient configuration's reduction over shots on two gloo ranks (CPU):
shots dealt round-robin, one all-reduce of the misfit, the material gradient
and the stacked per-shot moment-tensor gradients.  A stand-in replaces the
per-shot forward + adjoint solve (which needs the GPU): it returns values
that depend on the shot, so the test sees which rank solved which shot and
that every rank ends with the full sums."""
import os
import socket
from types import SimpleNamespace

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

SHAPE = (3, 4, 5, 6)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _shots():
    shots = []
    for i in range(5):
        blk = SimpleNamespace(sources=[None] * (1 + i % 2))
        shots.append((SimpleNamespace(blocks=[blk], tag=i), np.full((4, 2, 3), float(i))))
    return shots


def _solve(solved):
    def solve(problem, observed, material):
        i = problem.tag
        solved.append(i)
        gm = np.full(material.shape, float(i + 1))
        gM = np.arange(6 * len(problem.blocks[0].sources), dtype=np.float64).reshape(-1, 6) + 100 * i
        return float(10 * (i + 1)), gm, gM
    return solve


def _expected():
    material = np.zeros(SHAPE)
    chi = sum(10.0 * (i + 1) for i in range(5))
    g = np.full(SHAPE, float(sum(i + 1 for i in range(5))))
    gms = [np.arange(6 * (1 + i % 2), dtype=np.float64).reshape(-1, 6) + 100 * i for i in range(5)]
    return material, chi, g, gms


def _worker(rank, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        from waveqlab3d_q_gpu_b200.adjoint import gradient_over_shots
        solved = []
        material, _, _, _ = _expected()
        chi, g, gms = gradient_over_shots(_shots(), material, solve=_solve(solved))
        np.savez(os.path.join(out, f"r{rank}.npz"), chi=chi, g=g, solved=np.array(solved),
                 **{f"m{i}": m for i, m in enumerate(gms)})
    finally:
        dist.destroy_process_group()


def test_shots_dealt_round_robin_and_reduced(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    _, chi, g, gms = _expected()
    for rank in (0, 1):
        r = np.load(tmp_path / f"r{rank}.npz")
        assert list(r["solved"]) == list(range(rank, 5, 2))
        assert float(r["chi"]) == chi
        assert np.array_equal(r["g"], g)
        for i in range(5):
            assert np.array_equal(r[f"m{i}"], gms[i])


def test_single_process_sums_locally():
    from waveqlab3d_q_gpu_b200.adjoint import gradient_over_shots
    solved = []
    material, chi, g, gms = _expected()
    c, gg, m = gradient_over_shots(_shots(), material, solve=_solve(solved))
    assert solved == list(range(5)) and c == chi and np.array_equal(gg, g)
    assert all(np.array_equal(a, b) for a, b in zip(m, gms))
