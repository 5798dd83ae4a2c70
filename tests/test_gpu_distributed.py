"""One block per process on the CUDA path: the TPV5 two-block problem run as
two ranks (each holding one block, the interface face swapped every stage)
equals the single-process two-block run with one slip accumulation per stage.
A curvilinear Q8 + PML two-block problem with a locked interface does too
(with friction, the two sides of a curvilinear fault would keep slightly
different slip -- each side's normals come from its own block's metric --
as the reference's two ranks do).

Both ranks run on the one GPU of the test box with the gloo backend (face
traces go through host memory); nothing on the device waits for the other
process.
"""
import os
import socket

import numpy as np
import pytest

from cases import rel_l2, tpv5_case, two_block_case

pytestmark = pytest.mark.gpu

NSTEPS = 12


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, port, out, which):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        import sys
        sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
        from waveqlab3d_q_gpu_b200.distributed import BlockRank
        p = tpv5_case() if which == "tpv5" else two_block_case(mesh="curvilinear", coupling="locked",
                                                                response="anelastic-Q8", pml=True)
        br = BlockRank(p, rank, backend="gloo", nsteps_hint=NSTEPS)
        br.run(NSTEPS)
        d = br.domain
        d.synchronize()
        np.save(os.path.join(out, f"F{rank}.npy"), d.fields(0))
        np.save(os.path.join(out, f"S{rank}.npy"), d.fault("S"))
        np.save(os.path.join(out, f"seis{rank}.npy"), d.seismograms(0))
        br.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("which", ["tpv5", "curvilinear_q8_pml"])
def test_block_per_rank_equals_two_block_run(wql3d_lib, tmp_path, which):
    import torch.multiprocessing as mp
    from waveqlab3d_q_gpu_b200.domain import Domain
    port = _free_port()
    mp.start_processes(_worker, args=(port, str(tmp_path), which), nprocs=2, join=True, start_method="spawn")
    p = tpv5_case() if which == "tpv5" else two_block_case(mesh="curvilinear", coupling="locked",
                                                            response="anelastic-Q8", pml=True)
    g = Domain(p, nsteps_hint=NSTEPS)
    for n in range(1, NSTEPS + 1):
        g.time_step_RK(n)
    for b in (0, 1):
        Fb = np.load(tmp_path / f"F{b}.npy")
        assert rel_l2(Fb, g.fields(b)) < 1e-12, (b, rel_l2(Fb, g.fields(b)))
        sb = np.load(tmp_path / f"seis{b}.npy")
        sg = g.seismograms(b)
        assert sb.shape == sg.shape
        assert rel_l2(sb[:, :, 1:], sg[:, :, 1:]) < 1e-12
    # side 1 keeps the slip state the one-process run keeps
    S0 = np.load(tmp_path / "S0.npy")
    Sg = g.fault("S")
    if np.abs(Sg).max() > 1e-15:
        assert rel_l2(S0, Sg) < 1e-12
    g.close()
