"""The CPU oracle against the reference's own known answers (no GPU)."""
import numpy as np
import pytest

from cases import (LOCKED_PIN_BLOCK_MAX, PIN_MAX_FIELD, UPWIND4_PIN, locked_pin_case, pin_case, round_sig,
                   upwind4_pin_case)


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


def test_elastic_locked_interface_o6_block_maxima(oracle_lib):
    """inputfile/test_elastic_locked_interface_o6.in -> block1 max = 2.0699E+03,
    block2 max = 1.6389E+03 (the 5 printed digits).  103 steps: the wave crosses
    the locked interface and reaches the absorbing outer faces, so this pins the
    interface SAT and the physical-boundary SATs that the 6-step pin above never
    reaches.  Locked coupling does not feed the slip back, so the one-process
    double slip accumulation does not change the fields."""
    p = locked_pin_case()
    assert p.nt() == 103
    d = oracle_lib.OracleDomain(p)
    d.run(p.nt())
    mf, me, bm = d.final_state()
    assert me == 0.0
    assert [round_sig(v) for v in bm[:2]] == list(LOCKED_PIN_BLOCK_MAX), bm
    assert mf == max(bm[:2])


@pytest.mark.parametrize("response", ["anelastic-Q8", "anelastic-Q4"])
def test_anelastic_upwind4_dynamic_final_state(oracle_lib, response):
    """inputfile/test_anelastic_Q8_dynamic.in -> 1.8221E+02 / 1.4544E+01 and
    test_anelastic_Q4_dynamic.in -> 1.8221E+02 / 1.1049E+01 (max|field|,
    max|memory variable|, 5 printed digits).  Upwind order 4 with SAT penalty
    144/49; the published memory-variable maxima pin the Q4 / Q8 updates."""
    for f32 in (False, True):
        p = upwind4_pin_case(response, closure_f32_literal=f32)
        assert p.nt() == 5 and p.fd_operator() == 1
        assert abs(p.sat_penalty() - 144.0 / 49.0) < 1e-15
        d = oracle_lib.OracleDomain(p)
        d.run(p.nt())
        mf, me, _ = d.final_state()
        assert (round_sig(mf), round_sig(me)) == UPWIND4_PIN[response], (mf, me)


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
