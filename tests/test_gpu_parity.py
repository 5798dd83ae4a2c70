"""CUDA path (libwql3d.so through the C ABI) against the CPU oracle."""
import numpy as np
import pytest

from cases import PIN_MAX_FIELD, pin_case, random_state, rel_l2, small_case

pytestmark = pytest.mark.gpu


def _domain(problem, **kw):
    from waveqlab3d_q_gpu_b200.domain import Domain
    return Domain(problem, **kw)


def test_pin_case_final_state(wql3d_lib, oracle_lib):
    """test_elastic_traditional_o6: GPU final state equals the published 16-digit value to 1e-13."""
    for f32 in (True, False):
        p = pin_case(closure_f32_literal=f32)
        g = _domain(p)
        for n in range(1, p.nt() + 1):
            g.time_step_RK(n)
        mf, _, _ = g.close_domain(verbose=False)
        assert abs(mf - PIN_MAX_FIELD) / PIN_MAX_FIELD < 1e-13, "%.16E" % mf
        o = oracle_lib.OracleDomain(p)
        o.run(p.nt())
        assert rel_l2(g.fields(), o.fields()) < 1e-12


@pytest.mark.parametrize("mesh", ["cartesian", "curvilinear"])
@pytest.mark.parametrize("response", ["elastic", "anelastic-Q4", "anelastic-Q8", "anelastic-fQ8"])
@pytest.mark.parametrize("pml", [False, True])
@pytest.mark.parametrize("f32lit", [False, True])
def test_single_stage_random_state(wql3d_lib, oracle_lib, mesh, response, pml, f32lit):
    """One full RK stage from a random state: rates and fields to 1e-12 relative."""
    p = small_case(mesh=mesh, response=response, pml=pml)
    p.closure_f32_literal = f32lit
    (F, DF), = random_state(p)
    dt = p.dt()
    o = oracle_lib.OracleDomain(p)
    g = _domain(p)
    for dom in (o, g):
        dom.set_fields(F)
    o.set_rates(DF)
    g.set_rates_array(DF)
    for st in (1, 2):
        o.stage(st, dt)
        g.stage(st, dt)
    assert rel_l2(g.rates(), o.rates()) < 1e-12
    assert rel_l2(g.fields(), o.fields()) < 1e-12


@pytest.mark.parametrize("mesh", ["cartesian", "curvilinear"])
@pytest.mark.parametrize("response,pml,f32lit", [("elastic", False, False), ("elastic", True, False),
                                                 ("elastic", True, True), ("anelastic-Q8", True, True),
                                                 ("anelastic-Q4", False, False), ("anelastic-fQ8", True, False)])
def test_multi_step_run(wql3d_lib, oracle_lib, mesh, response, pml, f32lit):
    """40 steps from rest with sources, SATs, receivers: fields, memory variables, seismograms.

    f32lit selects the single-precision row-4 literal, whose off-diagonal
    metric terms (~1e-10) send Cartesian blocks through the full-metric
    near-boundary path instead of the separable one.
    """
    p = small_case(mesh=mesh, response=response, pml=pml)
    p.closure_f32_literal = f32lit
    nsteps = 40
    o = oracle_lib.OracleDomain(p)
    so = o.run(nsteps)[0]
    g = _domain(p, nsteps_hint=nsteps)
    g.run(nsteps)
    sg = g.seismograms()
    assert rel_l2(g.fields(), o.fields()) < 1e-11
    assert np.array_equal(g.receiver_index(), o.receiver_index())
    assert sg.shape == so.shape
    assert np.allclose(sg[:, :, 0], so[:, :, 0], rtol=0, atol=1e-15)
    assert rel_l2(sg[:, :, 1:], so[:, :, 1:]) < 1e-11
    if response != "elastic":
        assert rel_l2(g.eta(), o.eta()) < 1e-11
    mg, eg, _ = g.final_state()
    mo, eo, _ = o.final_state()
    assert abs(mg - mo) <= 1e-11 * mo


def test_run_equals_time_steps_and_split_ops(wql3d_lib):
    """Graph-captured run == eager time steps == the split scale/set/enforce/update
    sequence, with the stage-1 station sample taken by begin_step in the split
    sequence (time_step.f90:137).  The split set_rates evaluates the sources at
    the domain time, so the driver sets t0 + C_s dt before each stage's update
    the way time_step_RK advances D%t."""
    from waveqlab3d_q_gpu_b200.problem import RK_A, RK_B, RK_C
    p = small_case(mesh="curvilinear", response="anelastic-Q4", pml=True)
    dt = p.dt()
    a = _domain(p, nsteps_hint=6)
    a.run(6)
    b = _domain(p, nsteps_hint=6)
    for n in range(1, 7):
        b.time_step_RK(n)
    assert np.array_equal(a.fields(), b.fields())
    assert np.array_equal(a.seismograms(), b.seismograms())
    c = _domain(p, nsteps_hint=6)
    for n in range(1, 7):
        c.begin_step(n)
        t0 = c.t
        for st in range(1, 6):
            c.scale_rates(RK_A[st - 1])
            c.set_rates()
            c.enforce_bound_iface_conditions(st)
            c.t = t0 + RK_C[st] * dt
            c.update_fields(RK_B[st - 1] * dt)
    assert rel_l2(c.fields(), b.fields()) < 1e-13
    sb, sc = b.seismograms(), c.seismograms()
    assert sb.shape == sc.shape and sb.shape[0] == 6
    assert np.allclose(sc[:, :, 0], sb[:, :, 0], rtol=0, atol=1e-15)
    assert rel_l2(sc[:, :, 1:], sb[:, :, 1:]) < 1e-13


def test_rk_vector_kernels_exact(wql3d_lib):
    """tests/rk_vector_kernel_test.f90: rate*=-0.375; state+=0.125*rate on a 7x5x3x4 array, exact."""
    import ctypes as C
    import torch
    rng = np.random.default_rng(0)
    state = rng.standard_normal((4, 3, 5, 7))
    rate = rng.standard_normal((4, 3, 5, 7))
    ts = torch.tensor(state, device="cuda")
    tr = torch.tensor(rate, device="cuda")
    L = wql3d_lib
    assert L.wql3d_scale_rate_array(C.c_void_p(tr.data_ptr()), tr.numel(), -0.375, None) == 0
    assert L.wql3d_update_state_array(C.c_void_p(ts.data_ptr()), C.c_void_p(tr.data_ptr()), ts.numel(), 0.125, None) == 0
    torch.cuda.synchronize()
    exp_rate = -0.375 * rate
    exp_state = state + 0.125 * exp_rate
    assert np.array_equal(tr.cpu().numpy(), exp_rate)
    assert np.abs(ts.cpu().numpy() - exp_state).max() <= 32 * np.finfo(float).eps * np.abs(exp_state).max()


def test_metrics_match_oracle(wql3d_lib, oracle_lib):
    """Device metric kernel (D6 of the coordinates) against the oracle's derivatives()."""
    p = small_case(mesh="curvilinear")
    g = _domain(p)
    o = oracle_lib.OracleDomain(p)
    assert rel_l2(g.metrics(), o.metrics()) < 1e-15


def test_nonfinite_station_sample_is_reported(wql3d_lib):
    """A NaN planted in the initial state at a station's node reaches that
    station's stage-1 sample; wql3d_check_status reports WQL3D_ENONFINITE with
    the first such step (the reference's RUN-STATION-001 check,
    src/seismogram.f90:516-524), while a clean run reports 0."""
    from waveqlab3d_q_gpu_b200._lib import Wql3dError
    p = small_case(mesh="curvilinear", response="elastic")
    g = _domain(p, nsteps_hint=8)
    g.run(3)
    assert g.check_status() == 0
    idx = g.receiver_index()[0]
    F = g.fields()
    F[0, idx[2] - 1, idx[1] - 1, idx[0] - 1] = float("nan")
    g.set_fields(F)
    g.run(2)
    with pytest.raises(Wql3dError, match="ENONFINITE"):
        g.check_status()
    g.close()
