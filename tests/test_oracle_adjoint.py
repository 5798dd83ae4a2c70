"""The oracle's discrete adjoint (test infrastructure for the CUDA adjoint):
the transpose identity <L u, v> = <u, L^T v> of the elastic right-hand side,
and the waveform-misfit gradient against central finite differences.

The reference has no adjoint; what pins it is its own forward operator: L is
the oracle's set_rates + face SATs (src/RHS_Interior.f90:136-281, :1584-1768,
src/JU_xJU_yJU_z6.f90:12-809, :16088-16640), which the published final
states pin."""
import numpy as np
import pytest

from cases import small_case
from waveqlab3d_q_gpu_b200.problem import Source


def _rhs(oracle_lib, p, u):
    o = oracle_lib.OracleDomain(p)
    o.set_fields(u)
    o.set_rates(np.zeros_like(u))
    o.stage(1, p.dt())  # A(1) = 0: the rates are L u
    return o.rates()


@pytest.mark.parametrize("mesh", ["cartesian", "curvilinear"])
@pytest.mark.parametrize("fd", ["traditional", "upwind"])
def test_transpose_identity_and_material_derivative(oracle_lib, mesh, fd):
    p = small_case(mesh=mesh, sources=False, receivers=False, n=(15, 16, 17))
    if fd == "upwind":
        p.fd_type, p.order = "upwind", 4
    rng = np.random.default_rng(0)
    shape = (9,) + tuple(reversed(p.blocks[0].nqrs))
    u, v = rng.standard_normal(shape), rng.standard_normal(shape)
    Lu = _rhs(oracle_lib, p, u)
    o = oracle_lib.OracleDomain(p)
    o.set_fields(u)
    Ltv, g = o.adjoint_rhs(v)
    assert abs(np.vdot(Lu, v) - np.vdot(u, Ltv)) <= 1e-13 * abs(np.vdot(Lu, v))
    # d <v, L(m) u> / dm in a random direction (SAT material terms included)
    M = p.blocks[0].material.copy()
    dM = rng.standard_normal(M.shape) * M * 1e-3
    vals = []
    for s in (1.0, -1.0):
        p.blocks[0].material = M + s * dM
        vals.append(np.vdot(_rhs(oracle_lib, p, u), v))
    p.blocks[0].material = M
    fdv = (vals[0] - vals[1]) / 2.0
    assert abs(fdv - np.vdot(g, dM)) <= 1e-6 * abs(fdv)


@pytest.mark.parametrize("mesh", ["cartesian", "curvilinear"])
def test_misfit_gradient_against_finite_differences(oracle_lib, mesh):
    """25 steps, one Ricker moment source, 4 stations: d chi / d(lambda, mu, rho)
    and d chi / dM against central differences."""
    p = small_case(mesh=mesh, n=(15, 16, 17))
    p.blocks[0].sources = [Source("ricker", 8.0, 0.1, 1.0, 0.8, 1.2, 0.3, -0.2, 0.1, 0.9, 1.1, 1.05)]
    N = 25
    rng = np.random.default_rng(1)
    seis0 = oracle_lib.OracleDomain(p).run(N)[0][:, :, 1:4]
    observed = 0.9 * seis0 + 1e-3 * np.abs(seis0).max() * rng.standard_normal(seis0.shape)
    chi, seis, gmat, gM = oracle_lib.OracleDomain(p).misfit_gradient(observed, N)
    assert np.array_equal(seis, seis0)

    def chi_of():
        s = oracle_lib.OracleDomain(p).run(N)[0][:, :, 1:4]
        return 0.5 * np.sum((s - observed) ** 2)

    M = p.blocks[0].material.copy()
    dM = rng.standard_normal(M.shape) * M * 1e-2
    eps = 1e-3
    vals = []
    for s in (eps, -eps):
        p.blocks[0].material = M + s * dM
        vals.append(chi_of())
    p.blocks[0].material = M
    fdv = (vals[0] - vals[1]) / (2 * eps)
    assert abs(fdv - np.vdot(gmat, dM)) <= 1e-6 * abs(fdv)
    s0 = p.blocks[0].sources[0]
    m0 = np.array([s0.mxx, s0.myy, s0.mzz, s0.mxy, s0.mxz, s0.myz])
    dm = rng.standard_normal(6)
    vals = []
    for s in (eps, -eps):
        p.blocks[0].sources = [Source("ricker", 8.0, 0.1, *(m0 + s * dm), 0.9, 1.1, 1.05)]
        vals.append(chi_of())
    fdv = (vals[0] - vals[1]) / (2 * eps)
    assert abs(fdv - np.dot(gM[0], dm)) <= 1e-9 * abs(fdv)
