"""One block split into s-slabs on the CUDA path equals the whole block.

Three slabs of a 21 x 23 x 40 block (13, 14, 13 planes) run in one process
on the test GPU (:class:`SlabSet`: ghost planes copied between the slab
domains' buffers before every stage, the metric ghost planes once) from a
random initial state with sources and receivers.  The slabs' fields and
seismograms equal the whole-block run: each point takes the same stencil
rows and the same arithmetic, so the FP64 results agree to rounding of the
order of 1e-15 (tolerance 1e-12), the FP32 ones to 1e-6.  Cases: Cartesian
elastic, Cartesian Q4 with PML on both s faces, curvilinear Q8 with PML.
"""
import numpy as np
import pytest

from cases import random_state, rel_l2, small_case
from waveqlab3d_q_gpu_b200.domain import Domain
from waveqlab3d_q_gpu_b200.slabs import SlabSet

pytestmark = pytest.mark.gpu

CUTS = (13, 14, 13)
NSTEPS = 8


def _runs(mesh, response, pml, precision):
    p = small_case(mesh=mesh, response=response, pml=pml, n=(21, 23, 40))
    (F0, _), = random_state(p, seed=5, scale=1e-3)
    g = Domain(p, precision=precision, nsteps_hint=NSTEPS + 2)
    g.set_fields(F0)
    g.run(NSTEPS)
    g.synchronize()
    F, seis = g.fields(0), g.seismograms(0)
    g.close()
    ss = SlabSet(p, 3, precision=precision, nsteps_hint=NSTEPS + 2, cuts=CUTS)
    for part, d in zip(ss.parts, ss.domains):
        d.set_fields(F0[:, part.z0:part.z0 + part.problem.blocks[0].nqrs[2]])
    ss.run(NSTEPS)
    Fs = ss.fields()
    seis_s = np.zeros_like(seis)
    for part, sg in zip(ss.parts, ss.seismograms()):
        if len(part.rec_index):
            seis_s[:, part.rec_index] = sg
    ss.close()
    return F, Fs, seis, seis_s


@pytest.mark.parametrize("mesh,response,pml", [("cartesian", "elastic", False),
                                               ("cartesian", "anelastic-Q4", True),
                                               ("curvilinear", "anelastic-Q8", True)])
def test_slabs_equal_whole_block_fp64(mesh, response, pml):
    F, Fs, seis, seis_s = _runs(mesh, response, pml, "fp64")
    assert np.abs(F).max() > 0
    assert rel_l2(Fs, F) < 1e-12
    assert rel_l2(seis_s, seis) < 1e-12


def test_slabs_equal_whole_block_fp32():
    F, Fs, seis, seis_s = _runs("curvilinear", "anelastic-Q8", True, "fp32")
    assert rel_l2(Fs, F) < 1e-6
    assert rel_l2(seis_s, seis) < 1e-6


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _slab_worker(rank, port, out, nranks):
    import os
    import sys

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=nranks)
    try:
        sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
        from waveqlab3d_q_gpu_b200.distributed import SlabRank
        p = small_case(mesh="curvilinear", response="anelastic-Q8", pml=True, n=(21, 23, 40))
        (F0, _), = random_state(p, seed=5, scale=1e-3)
        sr = SlabRank(p, rank, nranks, backend="gloo", nsteps_hint=NSTEPS + 2, cuts=CUTS)
        z0, n = sr.part.z0, sr.part.problem.blocks[0].nqrs[2]
        sr.domain.set_fields(F0[:, z0:z0 + n])
        sr.run(NSTEPS)
        sr.domain.synchronize()
        np.save(os.path.join(out, f"F{rank}.npy"), sr.domain.fields(0))
        sr.close()
    finally:
        dist.destroy_process_group()


def test_slab_per_rank_equals_whole_block(wql3d_lib, tmp_path):
    """Three processes (gloo, ghost planes through host memory), one slab
    each, on the one test GPU; nothing on the device waits for another
    process."""
    import torch.multiprocessing as mp
    nranks = 3
    mp.start_processes(_slab_worker, args=(_free_port(), str(tmp_path), nranks), nprocs=nranks, join=True,
                       start_method="spawn")
    p = small_case(mesh="curvilinear", response="anelastic-Q8", pml=True, n=(21, 23, 40))
    (F0, _), = random_state(p, seed=5, scale=1e-3)
    g = Domain(p, nsteps_hint=NSTEPS + 2)
    g.set_fields(F0)
    g.run(NSTEPS)
    F = g.fields(0)
    g.close()
    Fs = np.concatenate([np.load(tmp_path / f"F{r}.npy") for r in range(nranks)], axis=1)
    assert rel_l2(Fs, F) < 1e-12
