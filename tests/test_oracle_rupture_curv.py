"""Oracle pin for the curvilinear block interface: the reference's archived
TPV28 rupture output.

test_problems/truth/2 holds the fault output of test_rup_curv_fric.in (two
21^3 curvilinear blocks meeting on the 'analytical_test_problem' fault
surface, slip-weakening TPV28 fault, 46 samples), written by a historical
build.  The surface, the unit normals and the strike / dip vectors written
beside it (the *_fault_topography_AX.dat and *_unit_*_vector_fractal_fault.dat
files) are the oracle's to rounding.  Two settings of that build differ from
the current sources, and the files fix both:

* the background stress: the sample-0 normal traction equals n.sigma.n at
  every fault point to float32 rounding with sigma_zz = -60, while
  src/initial_stress_condition.f90:78-84 now sets sigma_zz = +60 (the two
  agree only where n_z = 0: the grid lines y = 6, 7.5, 9 and z = -0.75, 0.75
  outside the Gaussian bump at the fault centre);
* block 1's station: the file is named for node (21, 11, 11), the fault node
  at (0.1, 7.5, 0); the current Find_Coordinates (src/seismogram.f90:772-872)
  picks node (20, 11, 11) for the listed station (-0, 7.5, 0), 0.055 away
  against 0.1.

With those two settings the curved-fault interface law, the curvilinear SAT
coupling and the slip integration reproduce the files to their float32
rounding on the part of the fault the fault edges have not yet influenced,
as for the Cartesian TPV5 pin; the fault-edge treatment of the historical
build differs (errors of ~1e-1 right at the edges after one step).
"""
import os

import numpy as np
import pytest

from cases import tpv28_case
from test_oracle_rupture import _record

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tpv28_curvilinear_truth.npz")

# background stress of the archived run (sxx, syy, szz, sxy, sxz, syz)
ARCHIVED_STRESS = (-60.0, 0.0, -60.0, 0.0, 29.38, 0.0)
# block 1's archived station node, the fault node (21, 11, 11)
ARCHIVED_STATION1 = (0.1, 7.5, 0.0)

# (sample, interior margin m, relative tolerance): points with m <= y, z <= 20 - m (0-based)
CORE = ((0, 0, 1e-7), (1, 8, 1e-6), (2, 9, 1e-6), (3, 10, 3e-7))


def archived_case(oracle_lib, **kw):
    from waveqlab3d_q_gpu_b200.mesh import pack_surfaces
    p = tpv28_case(lambda s, n: oracle_lib.tfi_grid(pack_surfaces(s), n), **kw)
    p.interface.stress = ARCHIVED_STRESS
    p.blocks[0].receivers = np.array([ARCHIVED_STATION1])
    return p


def core_errors(mine, truth):
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
def tpv28_single(oracle_lib):
    return _record(oracle_lib.OracleDomain(archived_case(oracle_lib)), 4)


def test_fault_core_matches_archived_truth(truth, tpv28_single):
    mine, _ = tpv28_single
    for n, name, err, tol in core_errors(mine, truth):
        assert err <= tol, (n, name, err)


def test_stations_match_archived_seismograms(truth, tpv28_single):
    # both stations sit on the fault centre; the files carry 6 decimals
    _, seis = tpv28_single
    for bi, key in ((0, "seis_block1"), (1, "seis_block2")):
        assert np.abs(seis[bi][:4] - truth[key][:4]).max() <= 6e-7


def test_sample0_prestress_is_the_projected_tensor(truth, tpv28_single):
    # Uhat / Vhat 4:6 at sample 0: T0 + hat traction; where the fault starts
    # locked the hat traction is zero and n.sigma.n is the normal component
    mine, _ = tpv28_single
    for name in ("Uhat", "Vhat"):
        np.testing.assert_allclose(mine[name][0][3:], truth[name][0][3:].astype(np.float64), rtol=0, atol=3e-5)


def test_current_source_stress_departs_from_the_archive(oracle_lib, truth):
    # sigma_zz = +60 (the current source) shifts the sample-0 normal traction
    # by 120 n_z^2 off the n_z = 0 lines
    p = archived_case(oracle_lib)
    p.interface.stress = None
    mine, _ = _record(oracle_lib.OracleDomain(p), 1)
    d = np.abs(mine["Uhat"][0][3] - truth["Uhat"][0][3].astype(np.float64))
    assert d.max() > 4.0
    lines = np.zeros((21, 21), bool)
    lines[:, (0, 10, 20)] = True       # y = 6, 7.5, 9
    lines[(5, 15), :] = True           # z = -0.75, 0.75
    lines[7:14, 7:14] = False          # the Gaussian bump tilts n off these lines
    assert d[lines].max() < 1e-3       # the tail of the bump
