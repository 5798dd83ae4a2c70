"""Setup-time anelastic coefficients (host code, no GPU).

Known answers from the reference's tests/fq8_effective_response_test.f90 and
the fixed Q4 / Q8 coefficient builders (checked against the oracle).
"""
import numpy as np
import pytest

from waveqlab3d_q_gpu_b200 import fq8
from waveqlab3d_q_gpu_b200.anelastic import coefficients, corrected_material
from waveqlab3d_q_gpu_b200.problem import AnelasticParams


def _withers(policy="table-exact"):
    return AnelasticParams(Qs0=50.0, Qp0=50.0, gamma=0.6, f_transition=1.0, fref=1.0, coarse_grain=2,
                           coefficient_method="withers-2015", weight_policy=policy)


def test_fq8_withers_known_answers():
    tau, ss, sp = fq8.build_fq8_coefficients(_withers())
    q = fq8.effective_q(1.0, tau, ss)
    scale = fq8.common_modulus_scale(1.0, tau, ss)
    ratio = fq8.phase_velocity_ratio(1.0, 1.0, tau, ss)
    assert abs(q - 54.8324966843126) <= 1e-11
    assert abs(scale - 1.01727165422423) <= 1e-11
    assert abs(ratio - 1.0) <= 1e-13
    assert np.abs(ss - sp).max() <= 1e-15
    assert abs(ss[0] - (-0.000688)) <= 1e-14
    # coarse cell: one common modulus, velocities reproduced at fref
    rho, vs, vp = 2.7, 3.464, 6.0
    mu = rho * vs ** 2 * scale
    lam = rho * vp ** 2 * scale - 2 * mu
    assert abs(np.sqrt(mu / (rho * scale)) * ratio - vs) <= 1e-13
    assert abs(np.sqrt((lam + 2 * mu) / (rho * scale)) * ratio - vp) <= 1e-13


def test_fq8_nonnegative_refit():
    tau, ss, _ = fq8.build_fq8_coefficients(_withers())
    tau_r, ss_r, sp_r = fq8.build_fq8_coefficients(_withers("nonnegative-refit"))
    assert np.all(ss_r >= 0) and np.all(sp_r >= 0)
    assert abs(fq8.effective_q(1.0, tau_r, ss_r) - fq8.effective_q(1.0, tau, ss)) <= 1e-11
    assert np.abs(ss_r - sp_r).max() <= 1e-15
    f = 0.05 * (20.0 / 0.05) ** (np.arange(512) / 511.0)
    dq = max(abs(fq8.effective_q(x, tau_r, ss_r) / fq8.effective_q(x, tau, ss) - 1) for x in f)
    dv = max(abs(fq8.phase_velocity_ratio(x, 1.0, tau_r, ss_r) / fq8.phase_velocity_ratio(x, 1.0, tau, ss) - 1)
             for x in f)
    assert dq <= 0.0128 and dv <= 1.3e-5


def test_fq8_rejects_raw_withers_without_coarse_grain():
    p = _withers()
    p.coarse_grain = 0
    with pytest.raises(ValueError):
        fq8.build_fq8_coefficients(p)


def test_fq8_conventional_fit_quality():
    p = AnelasticParams(Qs0=100.0, Qp0=200.0, gamma=0.6, f_transition=1.0, fref=1.0, coarse_grain=0)
    tau, ss, sp = fq8.build_fq8_coefficients(p)
    assert np.all(ss >= 0) and ss.sum() < 1
    f = 0.1 * 100.0 ** (np.arange(64) / 63.0)
    target = np.where(f < 1.0, 100.0, 100.0 * f ** 0.6)
    err = max(abs(fq8.realized_q(x, tau, ss) / t - 1) for x, t in zip(f, target))
    assert err < 0.1


@pytest.mark.parametrize("resp", ["anelastic-Q4", "anelastic-Q8"])
def test_q4_q8_coefficients_match_oracle(oracle_lib, resp):
    import ctypes as C
    p = AnelasticParams(fmin=0.05, fmax=20.0)
    tau, w, _ = coefficients(resp, p)
    n = len(tau)
    t2 = np.zeros(8)
    w2 = np.zeros(8)
    f = oracle_lib.lib().orc_q4_coefficients if n == 4 else oracle_lib.lib().orc_q8_coefficients
    f(0.05, 20.0, t2.ctypes.data_as(C.POINTER(C.c_double)), w2.ctypes.data_as(C.POINTER(C.c_double)))
    assert np.array_equal(tau, t2[:n]) and np.array_equal(w, w2[:n])


def test_modulus_correction_matches_oracle(oracle_lib):
    import ctypes as C
    from cases import small_case
    pr = small_case(response="anelastic-Q8")
    blk = pr.blocks[0]
    m = corrected_material(pr, blk)
    tau, w, _ = coefficients(pr.response, pr.anelastic)
    base = np.array(blk.material, copy=True)
    lam, mu, rho = base[0].copy(), base[1].copy(), base[2].copy()
    qs = np.full_like(mu, 1 / pr.anelastic.Qs0)
    qp = np.full_like(mu, 1 / pr.anelastic.Qp0)
    dp = C.POINTER(C.c_double)
    t8 = np.zeros(8); t8[:len(tau)] = tau
    w8 = np.zeros(8); w8[:len(w)] = w
    oracle_lib.lib().orc_modulus_correction(len(tau), t8.ctypes.data_as(dp), w8.ctypes.data_as(dp), 1.0, lam.size,
                                            lam.ctypes.data_as(dp), mu.ctypes.data_as(dp), rho.ctypes.data_as(dp),
                                            qs.ctypes.data_as(dp), qp.ctypes.data_as(dp))
    assert np.allclose(m[0], lam, rtol=1e-15, atol=0) and np.allclose(m[1], mu, rtol=1e-15, atol=0)
