"""Two-block runs on the CUDA path (libwql3d.so through the C ABI): the block
interface (locked, linear friction, slip-weakening with TPV5 or map
prestress) against the CPU oracle, and the TPV5 fault core against the
reference's archived rupture output."""
import os

import numpy as np
import pytest

from cases import random_state, rel_l2, tpv5_case, two_block_case

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tpv5_cartesian_truth.npz")
FAULT = ("S", "Svel", "Uhat", "Vhat", "trup")


def _domain(problem, **kw):
    from waveqlab3d_q_gpu_b200.domain import Domain
    return Domain(problem, **kw)


def _compare_fault(g, o, tol):
    for name in FAULT:
        a, b = g.fault(name), o.fault(name)
        if name == "trup":
            assert np.array_equal(a, b), name
        elif np.abs(b).max() < 1e-15:
            # a locked (or alpha = 1e14 linear) fault: slip is roundoff on both sides
            assert np.abs(a).max() < 1e-15, name
        else:
            assert rel_l2(a, b) < tol, (name, rel_l2(a, b))


@pytest.mark.parametrize("serial", [False, True])
def test_tpv5_steps_match_oracle(wql3d_lib, oracle_lib, serial):
    """TPV5 2 x 21^3, 12 steps one at a time: both blocks' fields, the stage-1
    fault outputs of every step, the stations."""
    p = tpv5_case(serial_shared=serial)
    o = oracle_lib.OracleDomain(p)
    g = _domain(p, nsteps_hint=12)
    seis_o = [[], []]
    for n in range(1, 13):
        s = o.run(1)
        for b in (0, 1):
            seis_o[b].append(s[b][0])
        g.time_step_RK(n)
        _compare_fault(g, o, 1e-12)
    for b in (0, 1):
        assert rel_l2(g.fields(b), o.fields(b)) < 1e-12
        so = np.array(seis_o[b])
        sg = g.seismograms(b)
        assert sg.shape == so.shape
        assert np.allclose(sg[:, :, 0], so[:, :, 0], rtol=0, atol=1e-15)
        assert rel_l2(sg[:, :, 1:], so[:, :, 1:]) < 1e-12


def test_tpv5_graph_run_equals_steps(wql3d_lib):
    p = tpv5_case()
    a = _domain(p, nsteps_hint=20)
    a.run(20)
    b = _domain(p, nsteps_hint=20)
    for n in range(1, 21):
        b.time_step_RK(n)
    for k in (0, 1):
        assert np.array_equal(a.fields(k), b.fields(k))
    for name in FAULT:
        assert np.array_equal(a.fault(name), b.fault(name))


def test_tpv5_fault_core_matches_archived_truth(wql3d_lib):
    """The GPU path itself against test_problems/truth/1 on the fault core
    (points the fault edges cannot have influenced yet)."""
    truth = dict(np.load(GOLDEN))
    g = _domain(tpv5_case(), nsteps_hint=4)
    core = ((0, 0, 3e-7), (1, 6, 3e-6), (2, 8, 1e-6))
    for n, m, tol in core:
        mine = {"S": g.fault("S"), "Uface": g.fields(0)[:, :, :, -1], "Vface": g.fields(1)[:, :, :, 0]}
        g.time_step_RK(n + 1)
        for k in ("Svel", "Uhat", "Vhat"):
            mine[k] = g.fault(k)
        for name, a in mine.items():
            if name == "S" and n == 0:
                continue
            b = truth[name][n].astype(np.float64)
            err = np.abs(a[:, m:21 - m, m:21 - m] - b[:, m:21 - m, m:21 - m]).max() / max(np.abs(b).max(), 1e-30)
            assert err <= tol, (n, name, err)


@pytest.mark.parametrize("mesh", ["cartesian", "curvilinear"])
@pytest.mark.parametrize("coupling", ["locked", "slip-weakening_friction", "linear_friction"])
def test_two_block_run_matches_oracle(wql3d_lib, oracle_lib, mesh, coupling):
    """Heterogeneous two-block problem with sources, stations, free surface,
    clamped and absorbing faces: 16 graph-captured steps."""
    p = two_block_case(mesh=mesh, coupling=coupling)
    o = oracle_lib.OracleDomain(p)
    so = o.run(16)
    g = _domain(p, nsteps_hint=16)
    g.run(16)
    for b in (0, 1):
        assert rel_l2(g.fields(b), o.fields(b)) < 1e-11
        sg = g.seismograms(b)
        assert rel_l2(sg[:, :, 1:], so[b][:, :, 1:]) < 1e-11
    _compare_fault(g, o, 1e-11)


@pytest.mark.parametrize("response,pml", [("anelastic-Q8", False), ("elastic", True), ("anelastic-Q4", True)])
def test_two_block_anelastic_pml(wql3d_lib, oracle_lib, response, pml):
    p = two_block_case(mesh="curvilinear", coupling="slip-weakening_friction", response=response, pml=pml)
    o = oracle_lib.OracleDomain(p)
    o.run(10)
    g = _domain(p, nsteps_hint=10)
    g.run(10)
    for b in (0, 1):
        assert rel_l2(g.fields(b), o.fields(b)) < 1e-11
    if response != "elastic":
        assert rel_l2(g.eta(1), o.eta(1)) < 1e-11
    _compare_fault(g, o, 1e-11)


def test_two_block_random_state_stages(wql3d_lib, oracle_lib):
    """Two stages from random fields and rates on both blocks (the interface
    starts far from equilibrium, so the fault slips everywhere)."""
    p = two_block_case(mesh="curvilinear", coupling="slip-weakening_friction")
    dt = p.dt()
    o = oracle_lib.OracleDomain(p)
    g = _domain(p)
    for b, (F, DF) in enumerate(random_state(p, seed=11, scale=10.0)):
        o.set_fields(F, b)
        g.set_fields(F, b)
        o.set_rates(DF, b)
        g.set_rates_array(DF, b)
    for st in (1, 2):
        o.stage(st, dt)
        g.stage(st, dt)
    for b in (0, 1):
        assert rel_l2(g.rates(b), o.rates(b)) < 1e-12
        assert rel_l2(g.fields(b), o.fields(b)) < 1e-12
    _compare_fault(g, o, 1e-12)


def test_two_block_split_ops_equal_steps(wql3d_lib):
    from waveqlab3d_q_gpu_b200.problem import RK_A, RK_B, RK_C
    p = two_block_case(mesh="cartesian", coupling="slip-weakening_friction")
    dt = p.dt()
    a = _domain(p, nsteps_hint=5)
    for n in range(1, 6):
        a.time_step_RK(n)
    c = _domain(p, nsteps_hint=5)
    for n in range(1, 6):
        t0 = c.t
        for st in range(1, 6):
            c.scale_rates(RK_A[st - 1])
            c.set_rates()
            c.enforce_bound_iface_conditions(st)
            c.t = t0 + RK_C[st] * dt
            c.update_fields(RK_B[st - 1] * dt)
    for b in (0, 1):
        assert rel_l2(c.fields(b), a.fields(b)) < 1e-13
    assert rel_l2(c.fault("S"), a.fault("S")) < 1e-13


def test_fp32_two_block_tracks_fp64(wql3d_lib):
    """FP32 fields with compensated accumulation: a TPV5 run stays within
    single-precision distance of the FP64 run."""
    p = tpv5_case()
    a = _domain(p, nsteps_hint=20)
    a.run(20)
    b = _domain(p, precision="fp32", nsteps_hint=20)
    b.run(20)
    for k in (0, 1):
        assert rel_l2(b.fields(k), a.fields(k)) < 2e-5
    assert rel_l2(b.fault("S"), a.fault("S")) < 2e-5
