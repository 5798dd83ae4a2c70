"""The fault output files of a GPU TPV5 run, read back in the layout of the
reference's python/read_binary.py, against the archived truth
(test_problems/truth/1 as tests/golden/tpv5_cartesian_truth.npz) on the part
of the fault the fault edges cannot have reached (the same cores and
tolerances as the in-memory check in test_gpu_interface.py), and equal to the
in-memory outputs rounded to float32."""
import os

import numpy as np
import pytest

from cases import tpv5_case

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tpv5_cartesian_truth.npz")


def test_tpv5_fault_files_match_truth(wql3d_lib, tmp_path):
    from waveqlab3d_q_gpu_b200.domain import Domain
    from waveqlab3d_q_gpu_b200.fault_output import FILES, read_fault_output, run_with_fault_output
    truth = dict(np.load(GOLDEN))
    g = Domain(tpv5_case(), nsteps_hint=4)
    prefix = str(tmp_path / "test_rup_cart_fric")
    assert run_with_fault_output(g, 3, prefix) == 3
    got = {name: read_fault_output(prefix, name, 21, 21) for name, _ in FILES}
    for name, nc in FILES:
        assert os.path.getsize(f"{prefix}_interface.{name}") == 3 * nc * 21 * 21 * 4
    # the last records equal the domain's outputs rounded to float32
    for name in ("Uhat", "Vhat", "Svel", "trup"):
        assert np.array_equal(got[name][-1], g.fault(name).astype(np.float32)), name
    core = ((0, 0, 3e-7), (1, 6, 3e-6), (2, 8, 1e-6))
    for n, m, tol in core:
        for name in ("S", "Svel", "Uface", "Vface", "Uhat", "Vhat"):
            if name == "S" and n == 0:
                continue
            a = got[name][n].astype(np.float64)
            b = truth[name][n].astype(np.float64)
            err = np.abs(a[:, m:21 - m, m:21 - m] - b[:, m:21 - m, m:21 - m]).max() / max(np.abs(b).max(), 1e-30)
            assert err <= tol, (n, name, err)
    g.close()
