"""Oracle pin for the block interface: the reference's archived TPV5 rupture output.

test_problems/truth/1 holds the fault output of test_rup_cart_fric.in (two
21^3 Cartesian blocks, slip-weakening TPV5 fault, 46 samples), written by a
historical build in a four-rank layout.  The reference's own notes record
that the current code is not qualified against it
(PHASE2_SCRATCH_MEMORY_AUDIT.md:143-146 of the reference).  The current
interface law, SAT coupling and slip integration reproduce it to the float32
rounding of the files on the part of the fault that the fault edges have not
yet influenced: after step k only points at least m_k nodes from every edge
are compared.  The fault-edge treatment differs from the historical build
(errors of ~1e-2 after one step, right at the four fault edges) and is not
pinned by these files.

The same files decide how often the slip rate DS is accumulated per stage:
once (as each rank of a one-rank-per-block run does), not twice (as a
one-process two-block run of the current reference does, because both
blocks' Interface_RHS calls add to the shared iface).
"""
import os

import numpy as np
import pytest

from cases import tpv5_case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tpv5_cartesian_truth.npz")

# (sample, interior margin m, relative tolerance): points with m <= y, z <= 20 - m (0-based)
CORE = ((0, 0, 3e-7), (1, 6, 3e-6), (2, 8, 1e-6))


def _record(D, nsamp):
    out = {k: [] for k in ("S", "Svel", "Uface", "Vface", "Uhat", "Vhat", "trup")}
    seis = [[], []]
    for n in range(nsamp):
        out["S"].append(D.fault("S"))
        out["Uface"].append(D.fields(0)[:, :, :, -1])
        out["Vface"].append(D.fields(1)[:, :, :, 0])
        s = D.run(1)
        seis[0].append(s[0][0, 0])
        seis[1].append(s[1][0, 0])
        for k in ("Svel", "Uhat", "Vhat", "trup"):
            out[k].append(D.fault(k))
    return {k: np.array(v) for k, v in out.items()}, [np.array(a) for a in seis]


def _core_errors(mine, truth):
    errs = []
    for n, m, tol in CORE:
        for name in ("S", "Svel", "Uface", "Vface", "Uhat", "Vhat"):
            if name == "S" and n == 0:
                continue
            a = mine[name][n][:, m:21 - m, m:21 - m]
            b = truth[name][n][:, m:21 - m, m:21 - m].astype(np.float64)
            scale = max(float(np.abs(truth[name][n]).max()), 1e-30)
            errs.append((n, name, float(np.abs(a - b).max()) / scale, tol))
    return errs


@pytest.fixture(scope="module")
def truth():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="module")
def tpv5_single(oracle_lib):
    D = oracle_lib.OracleDomain(tpv5_case(serial_shared=False))
    return _record(D, 4)


def test_fault_core_matches_archived_truth(truth, tpv5_single):
    mine, _ = tpv5_single
    for n, name, err, tol in _core_errors(mine, truth):
        assert err <= tol, (n, name, err)


def test_fault_centre_stations_match_archived_seismograms(truth, tpv5_single):
    # the two stations sit at the fault centre (10 nodes from every edge);
    # the files carry 6 decimals
    _, seis = tpv5_single
    for bi, key in ((0, "seis_block1"), (1, "seis_block2")):
        assert np.abs(seis[bi][:4] - truth[key][:4]).max() <= 6e-7


def test_prestress_and_edge_locking_at_sample0(truth, tpv5_single):
    # Uhat / Vhat components 4:6 are the hat tractions plus prestress: 75.8 on
    # the boxcar edges (y = 6, 9 or z = +-1.5), 81.24 = 0.677 * 120 where the
    # fault starts above strength and slips
    mine, _ = tpv5_single
    for name in ("Uhat", "Vhat"):
        np.testing.assert_allclose(mine[name][0][3:], truth[name][0][3:].astype(np.float64), rtol=0, atol=2e-5)
    assert np.all(mine["trup"][0][0, 1:-1, 1:-1] == 0.0)      # slipping at t = 0
    assert np.all(mine["trup"][0][0, 0, :] == 1.0e9)          # z = -1.5 edge still locked


def test_double_accumulation_departs_from_truth(oracle_lib, truth):
    D = oracle_lib.OracleDomain(tpv5_case(serial_shared=True))
    mine, _ = _record(D, 2)
    m = 6
    # slip along l and cumulative slip integrate about twice as fast (not
    # exactly: the larger slip weakens the fault within the step)
    a = mine["S"][1][2:, m:21 - m, m:21 - m]
    b = truth["S"][1][2:, m:21 - m, m:21 - m].astype(np.float64)
    ratio = a / b
    assert ratio.min() > 1.9 and ratio.max() < 2.3
