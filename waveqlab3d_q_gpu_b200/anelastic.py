"""Setup-time anelastic coefficients and modulus correction (host side).

These run once before time stepping, like the reference's material setup:

* Q4 / Q8 relaxation times log-spaced over [1/(2 pi fmax), 1/(2 pi fmin)] with
  fixed weights (src/anelastic_q4_model.f90:97-111,
  src/anelastic_q8_model.f90:100-116);
* fQ8 relaxation times and strengths (src/anelastic_fq8_model.f90:112-152,
  src/withers_tables.f90), see :mod:`waveqlab3d_q_gpu_b200.fq8`;
* unrelaxed-modulus correction at ``fref`` (src/material.f90:156-298 Q4,
  :330-485 Q8, :1823-1985 fQ8).

The reference fills Qs^-1 / Qp^-1 from the scalars Qs0 / Qp0
(src/material.f90:232-233); this library also accepts per-point arrays
(``Block.qs_inv`` / ``Block.qp_inv``) for spatially varying Q.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np

PI = 3.141592653589793

Q4_WEIGHTS = (1.549360, 0.804277, 0.887718, 1.464160)
Q8_WEIGHTS = (1.50589707, 0.0, 0.52793567, 0.53065494, 0.32862132, 0.64375916, 0.0, 1.32751442)


def _log_spaced_tau(fmin: float, fmax: float, n: int) -> np.ndarray:
    taumin = 1.0 / (2.0 * PI * fmax)
    taumax = 1.0 / (2.0 * PI * fmin)
    return np.array([math.exp(math.log(taumin) + (2.0 * k - 1.0) / (2.0 * n) * math.log(taumax / taumin))
                     for k in range(1, n + 1)])


def coefficients(response: str, params) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(tau, weight-or-S-strength, P-strength) for the response."""
    if response == "anelastic-Q4":
        tau = np.asarray(params.tau, float) if params.tau is not None else _log_spaced_tau(params.fmin, params.fmax, 4)
        w = np.asarray(params.weight, float) if params.weight is not None else np.array(Q4_WEIGHTS)
        return tau, w, w
    if response == "anelastic-Q8":
        tau = np.asarray(params.tau, float) if params.tau is not None else _log_spaced_tau(params.fmin, params.fmax, 8)
        w = np.asarray(params.weight, float) if params.weight is not None else np.array(Q8_WEIGHTS)
        return tau, w, w
    if response == "anelastic-fQ8":
        if params.tau is not None:
            return (np.asarray(params.tau, float), np.asarray(params.strength_s, float),
                    np.asarray(params.strength_p, float))
        from .fq8 import build_fq8_coefficients
        return build_fq8_coefficients(params)
    raise ValueError(f"no anelastic coefficients for response {response!r}")


def q_inverse(problem, block) -> Tuple[np.ndarray, np.ndarray]:
    """Per-point Qs^-1, Qp^-1 arrays (ns, nr, nq)."""
    nq, nr, ns = block.nqrs
    p = problem.anelastic
    qs = block.qs_inv if block.qs_inv is not None else np.full((ns, nr, nq), 1.0 / p.Qs0)
    qp = block.qp_inv if block.qp_inv is not None else np.full((ns, nr, nq), 1.0 / p.Qp0)
    return np.ascontiguousarray(qs, float), np.ascontiguousarray(qp, float)


def base_material(block) -> np.ndarray:
    """lambda, mu, rho (3, ns, nr, nq) before any anelastic correction (src/material.f90:696-701)."""
    nq, nr, ns = block.nqrs
    if block.material is not None:
        return np.array(block.material, dtype=np.float64, copy=True)
    rho, cs, cp = block.rho_s_p
    m = np.empty((3, ns, nr, nq))
    m[0] = rho * (cp ** 2 - 2.0 * cs ** 2)
    m[1] = rho * cs ** 2
    m[2] = rho
    return m


def corrected_material(problem, block) -> np.ndarray:
    """Material with the unrelaxed-modulus correction of the response applied."""
    m = base_material(block)
    if problem.response == "elastic":
        return m
    tau, c1, c2 = coefficients(problem.response, problem.anelastic)
    lam, mu, rho = m[0], m[1], m[2]
    wref = 2.0 * PI * problem.anelastic.fref
    if problem.response in ("anelastic-Q4", "anelastic-Q8"):
        qs, qp = q_inverse(problem, block)
        val_s = np.zeros_like(mu)
        val_p = np.zeros_like(mu)
        for l in range(len(tau)):
            den_s = ((wref * wref) * (tau[l] * tau[l]) + 1.0) * (1.0 / qs)
            den_p = ((wref * wref) * (tau[l] * tau[l]) + 1.0) * (1.0 / qp)
            val_s = val_s + c1[l] / den_s
            val_p = val_p + c1[l] / den_p
        if np.any(val_s >= 1.0) or np.any(val_p >= 1.0):
            raise ValueError("invalid anelastic modulus correction: weight/Q sum >= 1")
        vs = np.sqrt(mu / rho)
        vp = np.sqrt((lam + 2.0 * mu) / rho)
        mu_s = rho * (vs * vs) / (1.0 - val_s)
        mu_p = rho * (vp * vp) / (1.0 - val_p)
    else:  # fQ8, src/material.f90:1880-1925
        from .fq8 import common_modulus_scale
        vs = np.sqrt(mu / rho)
        vp = np.sqrt((lam + 2.0 * mu) / rho)
        if problem.anelastic.coarse_grain == 2:
            mu_s = rho * (vs * vs) * common_modulus_scale(problem.anelastic.fref, tau, c1)
            mu_p = rho * (vp * vp) * common_modulus_scale(problem.anelastic.fref, tau, c2)
        else:
            val_s = 0.0
            val_p = 0.0
            for l in range(len(tau)):
                den = (wref * wref) * (tau[l] * tau[l]) + 1.0
                val_s = val_s + c1[l] / den
                val_p = val_p + c2[l] / den
            mu_s = rho * (vs * vs) / (1.0 - val_s)
            mu_p = rho * (vp * vp) / (1.0 - val_p)
    vs = np.sqrt(mu_s / rho)
    vp = np.sqrt(mu_p / rho)
    out = np.empty_like(m)
    out[1] = (vs * vs) * rho
    out[0] = (vp * vp) * rho - 2.0 * out[1]
    out[2] = rho
    return out
