"""Discrete adjoint on the CUDA path (libwql3d.so through the C ABI) against
the oracle's discrete adjoint, the transpose identity of the GPU's own
forward stage, central finite differences of the GPU forward, and the
torch.autograd.Function with sqrt(N) checkpointing."""
import numpy as np
import pytest

from cases import rel_l2, small_case
from waveqlab3d_q_gpu_b200.problem import Source

pytestmark = pytest.mark.gpu


def _problem(mesh):
    p = small_case(mesh=mesh, n=(15, 16, 17))
    p.blocks[0].sources = [Source("ricker", 8.0, 0.1, 1.0, 0.8, 1.2, 0.3, -0.2, 0.1, 0.9, 1.1, 1.05)]
    return p


def _gpu_rhs(p, u):
    """L u from the GPU's split stage operations (scale by 0, RHS, SATs); no sources."""
    from waveqlab3d_q_gpu_b200.domain import Domain
    g = Domain(p)
    g.set_fields(u)
    g.scale_rates(0.0)
    g.set_rates()
    g.enforce_bound_iface_conditions(1)
    r = g.rates()
    g.close()
    return r


@pytest.mark.parametrize("mesh", ["curvilinear", "cartesian"])
def test_adjoint_rhs_transpose_and_oracle(wql3d_lib, oracle_lib, mesh):
    """<L u, v> = <u, L^T v> with the GPU forward (1e-12); L^T v and the material
    term against the oracle's transpose (1e-12)."""
    import ctypes as C
    from waveqlab3d_q_gpu_b200 import _lib
    from waveqlab3d_q_gpu_b200.domain import Domain, _ptr
    p = small_case(mesh=mesh, sources=False, receivers=False, n=(15, 16, 17))
    rng = np.random.default_rng(0)
    shape = (9,) + tuple(reversed(p.blocks[0].nqrs))
    u, v = rng.standard_normal(shape), rng.standard_normal(shape)
    Lu = _gpu_rhs(p, u)
    g = Domain(p)
    L = wql3d_lib
    _lib.check(L.wql3d_adjoint_enable(g.handle), "enable")
    g.set_fields(u)
    Fb = np.zeros(shape)
    gm = np.zeros((3,) + shape[1:])
    vv = np.ascontiguousarray(v)
    _lib.check(L.wql3d_adjoint_rhs(g.handle, 0, _ptr(vv), _ptr(Fb), _ptr(gm)), "adjoint_rhs")
    lhs, rhs = np.vdot(Lu, v), np.vdot(u, Fb)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    o = oracle_lib.OracleDomain(p)
    o.set_fields(u)
    Fo, go = o.adjoint_rhs(v)
    assert rel_l2(Fb, Fo) < 1e-12
    assert rel_l2(gm, go) < 1e-12
    g.close()


@pytest.mark.parametrize("mesh", ["curvilinear", "cartesian"])
def test_misfit_gradient_matches_oracle_and_fd(wql3d_lib, oracle_lib, mesh):
    """25 steps: GPU gradients (material, moment) equal the oracle's discrete
    adjoint to 1e-10 and central differences of the GPU forward to 1e-6."""
    from waveqlab3d_q_gpu_b200.adjoint import AdjointSolver
    p = _problem(mesh)
    N = 25
    rng = np.random.default_rng(1)
    sol = AdjointSolver(p, N)
    seis0 = sol.forward()
    observed = 0.9 * seis0 + 1e-3 * np.abs(seis0).max() * rng.standard_normal(seis0.shape)
    seis = sol.forward()
    assert np.array_equal(seis, seis0)
    gmat, gM = sol.backward(seis - observed)
    chi_o, seis_o, gmat_o, gM_o = oracle_lib.OracleDomain(p).misfit_gradient(observed, N)
    assert rel_l2(seis, seis_o) < 1e-11
    assert rel_l2(gmat, gmat_o) < 1e-10
    assert rel_l2(gM, gM_o) < 1e-10
    M = p.blocks[0].material.copy()
    dM = rng.standard_normal(M.shape) * M * 1e-2
    eps = 1e-3
    vals = []
    for s in (eps, -eps):
        sol.set_parameters(material=M + s * dM)
        vals.append(0.5 * np.sum((sol.forward() - observed) ** 2))
    sol.set_parameters(material=M)
    fdv = (vals[0] - vals[1]) / (2 * eps)
    assert abs(fdv - np.vdot(gmat, dM)) <= 1e-6 * abs(fdv)
    s0 = p.blocks[0].sources[0]
    m0 = np.array([[s0.mxx, s0.myy, s0.mzz, s0.mxy, s0.mxz, s0.myz]])
    dm = rng.standard_normal((1, 6))
    vals = []
    for s in (eps, -eps):
        sol.set_parameters(moment=m0 + s * dm)
        vals.append(0.5 * np.sum((sol.forward() - observed) ** 2))
    fdv = (vals[0] - vals[1]) / (2 * eps)
    assert abs(fdv - np.vdot(gM, dm)) <= 1e-9 * abs(fdv)
    sol.close()


def test_autograd_function_and_checkpoint_interval(wql3d_lib):
    """torch.autograd through WaveformMisfit: the gradient is independent of the
    checkpoint interval (K = 1, sqrt(N), N) and of recording the stage inputs
    versus recomputing them, and equals the solver's backward."""
    import torch
    from waveqlab3d_q_gpu_b200.adjoint import AdjointSolver, waveform_misfit
    p = _problem("curvilinear")
    N = 30
    ref = AdjointSolver(p, N)
    seis0 = ref.forward()
    rng = np.random.default_rng(2)
    observed = 0.8 * seis0 + 1e-3 * np.abs(seis0).max() * rng.standard_normal(seis0.shape)
    grads = []
    for K, rec in ((1, True), (None, True), (N, True), (None, False)):
        sol = AdjointSolver(p, N, checkpoint_every=K, record_stages=rec)
        mat = torch.tensor(p.blocks[0].material, dtype=torch.float64, device="cuda", requires_grad=True)
        s0 = p.blocks[0].sources[0]
        mom = torch.tensor([[s0.mxx, s0.myy, s0.mzz, s0.mxy, s0.mxz, s0.myz]], dtype=torch.float64, device="cuda",
                           requires_grad=True)
        chi = waveform_misfit(mat, mom, sol, observed)
        chi.backward()
        grads.append((mat.grad.cpu().numpy(), mom.grad.cpu().numpy(), float(chi.detach())))
        sol.close()
    for gm, gmom, chi in grads[1:]:
        assert chi == grads[0][2]
        assert rel_l2(gm, grads[0][0]) < 1e-13
        assert rel_l2(gmom, grads[0][1]) < 1e-13
    gmat, gM = ref.backward(ref.forward() - observed)
    assert rel_l2(grads[0][0], gmat) < 1e-13
    ref.close()


def test_gradient_over_shots_sums_the_shots(wql3d_lib):
    """gradient_over_shots in one process: the misfit and material gradient
    are the sums of the shots' own adjoint solves, the moment gradients each
    shot's own (the reduction path of the multi-GPU gradient configuration,
    whose all-reduce the gloo test covers)."""
    import copy
    from waveqlab3d_q_gpu_b200.adjoint import AdjointSolver, gradient_over_shots
    from waveqlab3d_q_gpu_b200.problem import Source
    N = 16
    shots = []
    for i, (x, y) in enumerate(((0.9, 1.1), (1.2, 0.8))):
        p = _problem("curvilinear")
        p.blocks[0].sources = [Source("ricker", 8.0, 0.1, 1.0, 0.8, 1.2, 0.3, -0.2, 0.1, x, y, 1.05)]
        sol = AdjointSolver(p, N)
        obs = 0.9 * sol.forward()
        sol.close()
        shots.append((p, obs))
    mat = copy.deepcopy(shots[0][0].blocks[0].material) * 1.01
    chi, g, gms = gradient_over_shots(shots, mat)
    chi_sum, g_sum = 0.0, np.zeros_like(mat)
    for (p, obs), gM_got in zip(shots, gms):
        sol = AdjointSolver(p, N)
        sol.set_parameters(material=mat)
        res = sol.forward() - obs
        gm, gM = sol.backward(res)
        sol.close()
        chi_sum += 0.5 * float(np.sum(res * res))
        g_sum += gm
        assert np.array_equal(gM_got, gM)
    assert chi == chi_sum
    assert np.array_equal(g, g_sum)
