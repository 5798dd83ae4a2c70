"""The CPU oracle against the reference's own known answers (no GPU)."""
import numpy as np
import pytest

from cases import PIN_MAX_FIELD, pin_case


def test_elastic_traditional_o6_final_state(oracle_lib):
    """inputfile/test_elastic_traditional_o6.in -> 1.6623128367649574E+02 (16 digits published)."""
    for f32 in (True, False):
        p = pin_case(closure_f32_literal=f32)
        assert p.nt() == 6
        d = oracle_lib.OracleDomain(p)
        d.run(p.nt())
        mf, me, _ = d.final_state()
        assert abs(mf - PIN_MAX_FIELD) / PIN_MAX_FIELD < 1e-13, "%.16E" % mf
        assert me == 0.0


def test_dt_and_nt_follow_block_time_step():
    """dt = CFL*h/sqrt(cs^2+cp^2) with scalar rho_s_p (src/block.f90:495-510), nt = floor(t_final/dt)."""
    p = pin_case()
    assert abs(p.dt() - 0.2 * 0.1 / np.sqrt(3.464 ** 2 + 36.0)) < 1e-18
    assert p.nt() == 6


def test_oracle_metrics_cartesian(oracle_lib):
    """Metrics of a Cartesian block: diagonal 1/(b-a) up to the SBP row residuals.

    With double-precision closure literals the off-diagonal metric entries are
    roundoff (< 1e-14).  With the single-precision row-4 literal (reference
    built without -r8) they reach ~1e-10, which is why the near-boundary
    operator keeps the full metric even on Cartesian grids.
    """
    off = {}
    for f32 in (False, True):
        d = oracle_lib.OracleDomain(pin_case(closure_f32_literal=f32))
        m = d.metrics()
        assert np.allclose(m[0], 0.25, rtol=1e-8)
        assert np.allclose(m[9], 64.0, rtol=1e-8)
        off[f32] = np.abs(m[[1, 2, 3, 5, 6, 7]]).max()
    assert off[False] < 1e-14
    assert 1e-11 < off[True] < 1e-8
