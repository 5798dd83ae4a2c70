"""The planar-fault fQ8 configuration (two Cartesian blocks with a
slip-weakening interface, von Karman medium, overstressed nucleation
patch) at reduced size on the CUDA path against the CPU oracle: both blocks'
fields, the memory variables and the fault outputs after 8 steps of
rupture (1e-11), and the FP32 path within 1e-6 of FP64 (measured 4.8e-8
on the fields, 3.7e-8 on the slip)."""
import numpy as np
import pytest

from cases import rel_l2

pytestmark = pytest.mark.gpu


def _case():
    from waveqlab3d_q_gpu_b200.configs import planar_fault_fq8
    return planar_fault_fq8(nq=30, nr=25, ns=23, h=0.5, steps=10)


def test_planar_fault_matches_oracle(wql3d_lib, oracle_lib):
    from waveqlab3d_q_gpu_b200.domain import Domain
    p = _case()
    o = oracle_lib.OracleDomain(p)
    so = o.run(8)
    g = Domain(p, nsteps_hint=8)
    g.run(8)
    assert np.abs(o.fault("Svel")).max() > 0.1          # the patch ruptures
    for b in (0, 1):
        assert rel_l2(g.fields(b), o.fields(b)) < 1e-11
        assert rel_l2(g.eta(b), o.eta(b)) < 1e-11
        assert rel_l2(g.seismograms(b)[:, :, 1:], so[b][:, :, 1:]) < 1e-11
    for name in ("S", "Svel", "Uhat", "Vhat"):
        assert rel_l2(g.fault(name), o.fault(name)) < 1e-11, name
    assert np.array_equal(g.fault("trup"), o.fault("trup"))


def test_planar_fault_fp32(wql3d_lib):
    from waveqlab3d_q_gpu_b200.domain import Domain
    p = _case()
    a = Domain(p, nsteps_hint=8)
    b = Domain(p, precision="fp32", nsteps_hint=8)
    a.run(8)
    b.run(8)
    for k in (0, 1):
        assert rel_l2(b.fields(k), a.fields(k)) < 1e-6
    assert rel_l2(b.fault("S"), a.fault("S")) < 1e-6
