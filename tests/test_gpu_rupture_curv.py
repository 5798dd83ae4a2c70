"""Curvilinear two-block rupture (TPV28 on the 'analytical_test_problem'
fault) on the CUDA path: the device-built mesh (wql3d_tfi_grid), the
face-basis prestress and the curved-fault interface law against the oracle
step by step, and the fault core against the reference's archived output
(test_problems/truth/2) with the settings that archive was written with."""
import numpy as np
import pytest

from cases import rel_l2, tpv28_case
from test_gpu_interface import FAULT, _compare_fault
from test_oracle_rupture_curv import ARCHIVED_STATION1, ARCHIVED_STRESS, CORE, GOLDEN

pytestmark = pytest.mark.gpu


def _case(stress, serial=False):
    from waveqlab3d_q_gpu_b200.mesh import tfi_grid
    p = tpv28_case(tfi_grid, serial_shared=serial)
    p.interface.stress = stress
    p.blocks[0].receivers = np.array([ARCHIVED_STATION1])
    return p


@pytest.mark.parametrize("stress,serial", [(ARCHIVED_STRESS, False), (None, False), (None, True)])
def test_tpv28_steps_match_oracle(wql3d_lib, oracle_lib, stress, serial):
    """12 steps one at a time: fault outputs every step, both blocks' fields
    and the stations at the end."""
    from waveqlab3d_q_gpu_b200.domain import Domain
    p = _case(stress, serial)
    o = oracle_lib.OracleDomain(p)
    g = Domain(p, nsteps_hint=12)
    seis_o = [[], []]
    for n in range(1, 13):
        s = o.run(1)
        for b in (0, 1):
            seis_o[b].append(s[b][0])
        g.time_step_RK(n)
        _compare_fault(g, o, 1e-11)
    for b in (0, 1):
        assert rel_l2(g.fields(b), o.fields(b)) < 1e-11
        assert rel_l2(g.seismograms(b)[:, :, 1:], np.array(seis_o[b])[:, :, 1:]) < 1e-11
    g.close()


def test_tpv28_graph_run_equals_steps(wql3d_lib):
    from waveqlab3d_q_gpu_b200.domain import Domain
    p = _case(ARCHIVED_STRESS)
    a = Domain(p, nsteps_hint=20)
    a.run(20)
    b = Domain(p, nsteps_hint=20)
    for n in range(1, 21):
        b.time_step_RK(n)
    for k in (0, 1):
        assert np.array_equal(a.fields(k), b.fields(k))
    for name in FAULT:
        assert np.array_equal(a.fault(name), b.fault(name))


def test_tpv28_fault_core_matches_archived_truth(wql3d_lib):
    from waveqlab3d_q_gpu_b200.domain import Domain
    truth = dict(np.load(GOLDEN))
    g = Domain(_case(ARCHIVED_STRESS), nsteps_hint=4)
    for n, m, tol in CORE:
        mine = {"S": g.fault("S"), "Uface": g.fields(0)[:, :, :, -1], "Vface": g.fields(1)[:, :, :, 0]}
        g.time_step_RK(n + 1)
        for k in ("Svel", "Uhat", "Vhat"):
            mine[k] = g.fault(k)
        for name, a in mine.items():
            if name == "S" and n == 0:
                continue
            b = truth[name][n].astype(np.float64)
            err = np.abs(a[:, m:21 - m, m:21 - m] - b[:, m:21 - m, m:21 - m]).max() / max(np.abs(b).max(), 1e-30)
            assert err <= tol, (n, name, err)
    for bi, key in ((0, "seis_block1"), (1, "seis_block2")):
        assert np.abs(g.seismograms(bi)[:4, 0] - truth[key][:4]).max() <= 6e-7
    g.close()
