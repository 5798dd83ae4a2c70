"""The CPU oracle against the reference's own known answers (no GPU)."""
import numpy as np
import pytest

from cases import (LOCKED_PIN_BLOCK_MAX, ORDER6_PIN, PIN_MAX_FIELD, UPWIND4_PIN, locked_pin_case, pin_case,
                   round_sig, upwind4_pin_case)


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


@pytest.mark.parametrize("fd_type,order", sorted(ORDER6_PIN))
def test_elastic_order6_upwind_final_state(oracle_lib, fd_type, order):
    """inputfile/test_elastic_upwind_o6.in -> 1.6563E+02 and
    test_elastic_upwind_drp_o6.in -> 1.6567E+02 (5 printed digits): the
    upwind-6 and upwind-DRP-6 interiors (6 steps do not reach the closures;
    test_upwind_pairs_are_sbp pins those)."""
    p = pin_case(fd_type=fd_type, order=order)
    assert p.nt() == 6
    d = oracle_lib.OracleDomain(p)
    d.run(p.nt())
    mf, me, _ = d.final_state()
    assert round_sig(mf) == ORDER6_PIN[(fd_type, order)], mf
    assert me == 0.0


@pytest.mark.parametrize("fd,degree", [(1, 2), (2, 3), (3, 3)])
def test_upwind_pairs_are_sbp(oracle_lib, fd, degree):
    """The transcribed closure tables of upwind-4 / upwind-6 / upwind-DRP-6:
    a diagonal norm H > 0 with H D+ + (H D-)^T = diag(-1, 0, .., 0, 1) exists
    (the upwind summation-by-parts property) and H (D+ - D-) is symmetric
    negative semidefinite (the upwind dissipation); every closure row
    differentiates polynomials of the closure degree exactly.  A wrong digit,
    sign or mirror in a table breaks all three."""
    n = 41
    Dp, Dm = np.zeros((n, n)), np.zeros((n, n))
    for i in range(1, n + 1):
        for plus, D in ((True, Dp), (False, Dm)):
            idx, c = oracle_lib.upwind_row(fd, plus, i, n)
            for j, v in zip(idx, c):
                D[i - 1, j - 1] += v
            x = idx.astype(np.float64) - i
            for k in range(degree + 1):
                exact = 1.0 if k == 1 else 0.0
                assert abs(np.sum(c * x ** k) - exact) < 1e-12 * max(1.0, np.abs(x).max() ** k), (i, plus, k)
    B = np.zeros((n, n))
    B[0, 0], B[-1, -1] = -1.0, 1.0
    A = np.zeros((n * n, n))
    for i in range(n):
        for j in range(n):
            A[i * n + j, i] += Dp[i, j]
            A[i * n + j, j] += Dm[j, i]
    h = np.linalg.lstsq(A, B.ravel(), rcond=None)[0]
    H = np.diag(h)
    assert h.min() > 0.2
    assert np.abs(H @ Dp + (H @ Dm).T - B).max() < 1e-13
    S = H @ (Dp - Dm)
    assert np.abs(S - S.T).max() < 1e-13
    assert np.linalg.eigvalsh(0.5 * (S + S.T)).max() < 1e-13


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
