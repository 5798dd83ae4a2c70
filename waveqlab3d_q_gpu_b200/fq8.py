"""Frequency-dependent Q (fQ8) coefficients: relaxation times and strengths.

Restates the reference's fQ8 model (src/anelastic_fq8_model.f90:112-316,
src/withers_tables.f90:151-294), which follows Withers, Olsen & Day (2015),
"Memory-efficient simulation of frequency-dependent Q", BSSA 105(6),
3129-3142:

* relaxation times log-spaced between tau_min(gamma) and tau_max(gamma)
  (eq. 15), divided by the transition frequency;
* ``conventional-nnls``: co-located strengths from a non-negative least-squares
  fit of Im(M) - Re(M)/Q(f) = 0 over 0.1 .. 10 f_transition (256 log-spaced
  frequencies, cyclic coordinate descent);
* ``withers-2015``: the published weights w_k = a_k/Q^2 + b_k/Q (Q <= 200,
  Table 2) or w_k = W_k/Q (Q > 200, Table 1), linearly interpolated in gamma,
  for the 2x2x2 coarse-grained layout, optionally rescaled to non-negative
  values that keep the effective Q at fref.

The tabulated numbers are the published coefficients of the paper.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np

PI = 3.141592653589793
N_MECH = 8
MINIMUM_Q = 15.0

TAU_MIN = [0.0032] * 7 + [0.0066, 0.0066, 0.0085]
TAU_MAX = [15.9155] * 7 + [3.9789, 3.9789, 3.9789]

# Table 1 (Q > 200): unscaled weights W_k per gamma row
W_HIGH_Q = [
    [0.8867, 0.8323, 0.5615, 0.8110, 0.4641, 1.0440, 0.0423, 1.7275],
    [0.3273, 0.8478, 0.3690, 0.9393, 0.4474, 1.0434, 0.0440, 1.7268],
    [0.0010, 0.8040, 0.2005, 1.0407, 0.4452, 1.0349, 0.0497, 1.7245],
    [0.0010, 0.6143, 0.0918, 1.1003, 0.4659, 1.0135, 0.0621, 1.7198],
    [0.0010, 0.4639, 0.0010, 1.1275, 0.5090, 0.9782, 0.0820, 1.7122],
    [0.2073, 0.1872, 0.0010, 1.0810, 0.6016, 0.9120, 0.1186, 1.6984],
    [0.3112, 0.0010, 0.0010, 1.0117, 0.7123, 0.8339, 0.1616, 1.6821],
    [0.1219, 0.0010, 0.0010, 0.2999, 1.3635, 0.0010, 0.5084, 1.2197],
    [0.0462, 0.0010, 0.0010, 0.1585, 1.4986, 0.0010, 0.4157, 1.3005],
    [0.0010, 0.0010, 0.0010, 0.1935, 1.5297, 0.0010, 0.1342, 1.5755],
]
# Table 2 (15 <= Q <= 200): w_k = a_k/Q^2 + b_k/Q
A_COEF = [
    [-27.50, -34.10, -1.62, -27.70, 14.60, -52.20, 72.00, -82.80],
    [7.37, -37.60, 13.10, -36.10, 12.30, -51.40, 69.00, -83.10],
    [31.80, -42.00, 25.70, -40.80, 7.02, -49.20, 65.40, -83.20],
    [43.70, -43.40, 34.30, -41.40, -2.87, -45.30, 60.90, -83.10],
    [41.60, -41.10, 38.00, -43.20, 5.63, -73.00, 103.00, -164.00],
    [20.00, -23.07, 31.40, -25.10, -45.20, -27.80, 45.90, -81.60],
    [8.08, -13.00, 25.40, -10.40, -75.90, -13.20, 35.70, -79.90],
    [1.99, -2.70, 0.00, 41.30, -88.80, 0.00, 40.70, -76.60],
    [5.16, -8.20, 0.00, 58.90, -108.60, 15.02, -5.88, -46.50],
    [-0.811, 0.00, 0.00, 56.03, -116.90, 22.00, 0.03, -61.90],
]
B_COEF = [
    [7.410, 6.020, 4.680, 6.280, 3.880, 8.170, 0.529, 13.190],
    [4.165, 5.520, 3.470, 7.210, 3.610, 8.193, 0.498, 13.130],
    [1.612, 5.080, 2.280, 7.931, 3.460, 8.150, 0.511, 13.070],
    [-0.109, 4.580, 1.190, 8.390, 3.530, 8.020, 0.592, 13.000],
    [-0.734, 3.820, 0.393, 8.670, 3.320, 8.580, -0.419, 14.900],
    [-0.435, 2.670, -0.043, 8.245, 4.847, 7.190, 1.150, 12.800],
    [-0.196, 1.810, -0.394, 7.657, 6.170, 6.360, 1.680, 12.700],
    [0.418, 0.590, 0.000, 2.180, 11.000, 0.000, 1.950, 11.300],
    [0.212, 0.345, 0.000, 0.813, 12.400, -0.283, 1.420, 11.700],
    [0.162, 0.000, 0.000, 0.797, 13.020, -0.402, -0.001, 12.500],
]
# exact decimal gamma grid 0.0, 0.1, ..., 0.9 as the reference writes it
GAMMA_VALUES = [0.0, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9]


def _gamma_bracket(gamma: float) -> Tuple[int, int, float]:
    """Bracketing table rows and linear weight (src/withers_tables.f90:207-244)."""
    g = max(0.0, min(0.9, gamma))
    lo, hi = 0, 0
    for i in range(9):
        if GAMMA_VALUES[i] <= g <= GAMMA_VALUES[i + 1]:
            lo, hi = i, i + 1
            break
    if g <= GAMMA_VALUES[0]:
        return 0, 0, 0.0
    if g >= GAMMA_VALUES[-1]:
        return 9, 9, 0.0
    return lo, hi, (g - GAMMA_VALUES[lo]) / (GAMMA_VALUES[hi] - GAMMA_VALUES[lo])


def relaxation_times(gamma: float) -> np.ndarray:
    """Withers eq. (15) relaxation times before the f_transition scaling."""
    lo, hi, a = _gamma_bracket(gamma)
    tmin = (1.0 - a) * TAU_MIN[lo] + a * TAU_MIN[hi]
    tmax = (1.0 - a) * TAU_MAX[lo] + a * TAU_MAX[hi]
    return np.array([math.exp(math.log(tmin) + float(2 * k - 1) / 16.0 * (math.log(tmax) - math.log(tmin)))
                     for k in range(1, N_MECH + 1)])


def withers_weights(gamma: float, Q: float) -> np.ndarray:
    """Published weights for (gamma, Q) (src/withers_tables.f90:178-294)."""
    lo, hi, a = _gamma_bracket(gamma)
    w = np.zeros(N_MECH)
    if Q > 200.0:
        for k in range(N_MECH):
            w[k] = ((1.0 - a) * W_HIGH_Q[lo][k] + a * W_HIGH_Q[hi][k]) / Q
    else:
        q = max(Q, 15.0)
        for k in range(N_MECH):
            ak = (1.0 - a) * A_COEF[lo][k] + a * A_COEF[hi][k]
            bk = (1.0 - a) * B_COEF[lo][k] + a * B_COEF[hi][k]
            w[k] = ak / (q ** 2) + bk / q
    return w


def fit_conventional_strengths(q0: float, gamma: float, f_transition: float, tau: np.ndarray) -> np.ndarray:
    """Non-negative least squares by cyclic coordinate descent (anelastic_fq8_model.f90:195-227)."""
    nfreq = 256
    A = np.zeros((nfreq, N_MECH))
    for i in range(nfreq):
        f = 0.1 * f_transition * 100.0 ** (float(i) / float(nfreq - 1))
        target = q0 if f < f_transition else q0 * (f / f_transition) ** gamma
        for j in range(N_MECH):
            x = 2.0 * PI * f * tau[j]
            A[i, j] = (target * x + 1.0) / (1.0 + x * x)
    s = np.zeros(N_MECH)
    r = np.ones(nfreq)
    norms = np.maximum(np.einsum("ij,ij->j", A, A), np.finfo(float).tiny)
    for _ in range(20000):
        maxd = 0.0
        for j in range(N_MECH):
            old = s[j]
            new = max(0.0, old + float(np.dot(A[:, j], r)) / norms[j])
            d = new - old
            if d != 0.0:
                r -= d * A[:, j]
            s[j] = new
            maxd = max(maxd, abs(d))
        if maxd < 1.0e-13:
            break
    return s


def harmonic_response(frequency: float, tau, strength) -> complex:
    """Coarse-cell harmonic-mean modulus response (anelastic_fq8_model.f90:248-262)."""
    inv = 0j
    for t, s in zip(tau, strength):
        local = 1.0 - s / complex(1.0, 2.0 * PI * frequency * t)
        inv += 1.0 / local
    return float(len(tau)) / inv


def effective_q(frequency: float, tau, strength) -> float:
    r = harmonic_response(frequency, tau, strength)
    if r.imag <= np.finfo(float).tiny:
        return float(np.finfo(float).max)
    return r.real / r.imag


def realized_q(frequency: float, tau, strength) -> float:
    """Co-located realized Q (anelastic_fq8_model.f90:229-246)."""
    re, im = 1.0, 0.0
    for t, s in zip(tau, strength):
        x = 2.0 * PI * frequency * t
        re -= s / (1.0 + x * x)
        im += s * x / (1.0 + x * x)
    if im <= np.finfo(float).tiny:
        return float(np.finfo(float).max)
    return abs(re / im)


def common_modulus_scale(fref: float, tau, strength) -> float:
    r = harmonic_response(fref, tau, strength)
    return (1.0 / np.sqrt(r)).real ** 2


def phase_velocity_ratio(frequency: float, fref: float, tau, strength) -> float:
    scale = common_modulus_scale(fref, tau, strength)
    r = scale * harmonic_response(frequency, tau, strength)
    return 1.0 / (1.0 / np.sqrt(r)).real


def refit_nonnegative(fref: float, tau, strength) -> np.ndarray:
    """Clip negative Withers strengths and rescale to keep Qeff(fref) (bisection, 100 iterations)."""
    s = np.asarray(strength, float).copy()
    if np.all(s >= 0.0):
        return s
    target = effective_q(fref, tau, s)
    s = np.maximum(s, 0.0)
    if s.sum() <= np.finfo(float).tiny:
        raise ValueError("nonnegative-refit has no positive strengths to rescale")
    maxf = (1.0 - 100.0 * np.finfo(float).eps) / s.sum()
    lo, hi = 0.0, min(2.0, maxf)
    if effective_q(fref, tau, hi * s) > target:
        raise ValueError("nonnegative-refit cannot bracket reference effective Q")
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if effective_q(fref, tau, mid * s) > target:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi) * s


def build_fq8_coefficients(params) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(tau, S strengths, P strengths) for an :class:`AnelasticParams` (anelastic_fq8_model.f90:112-152)."""
    method = getattr(params, "coefficient_method", None) or ("withers-2015" if params.coarse_grain == 2
                                                              else "conventional-nnls")
    policy = getattr(params, "weight_policy", None) or "table-exact"
    if params.coarse_grain == 0 and method == "withers-2015":
        raise ValueError("anelastic-fQ8 coarse_grain=0 requires coefficient_method=conventional-nnls")
    if params.Qs0 < MINIMUM_Q or params.Qp0 < MINIMUM_Q:
        raise ValueError("anelastic-fQ8 requires Qs0 and Qp0 >= 15")
    if not (0.0 <= params.gamma <= 0.9):
        raise ValueError("anelastic-fQ8 gamma must be in [0, 0.9]")
    tau = relaxation_times(params.gamma) / params.f_transition
    if method == "conventional-nnls":
        ss = fit_conventional_strengths(params.Qs0, params.gamma, params.f_transition, tau)
        sp = fit_conventional_strengths(params.Qp0, params.gamma, params.f_transition, tau)
    else:
        ss = withers_weights(params.gamma, params.Qs0)
        sp = withers_weights(params.gamma, params.Qp0)
        if policy == "nonnegative-refit":
            ss = refit_nonnegative(params.fref, tau, ss)
            sp = refit_nonnegative(params.fref, tau, sp)
    if ss.sum() >= 1.0 or sp.sum() >= 1.0:
        raise ValueError("anelastic-fQ8 coefficients leave a non-positive relaxed modulus")
    return tau, ss, sp


def relaxation_dt_limit(params) -> float:
    tau, _, _ = build_fq8_coefficients(params)
    return 2.0 * float(tau.min())
