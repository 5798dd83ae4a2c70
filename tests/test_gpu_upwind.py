"""Upwind operators on the CUDA path (libwql3d.so through the C ABI) against
the CPU oracle and the reference's published final states.

Velocities by the forward operator D+, stresses by the backward operator D-:
fd_type = 'upwind', order = 4 (src/JU_xJU_yJU_z6.f90:1439-2033 near the
boundaries, :17865-18400 in the interior, SAT penalty 144/49), order = 6
(:2665-3688, :18958-19510, 42300/13613) and fd_type = 'upwind_drp', order = 6
(:10556-12058 and its interior routine, 3.39644507697204); penalties of
src/block.f90:242-300.
"""
import numpy as np
import pytest

from cases import ORDER6_PIN, UPWIND4_PIN, pin_case, random_state, rel_l2, round_sig, small_case, upwind4_pin_case

pytestmark = pytest.mark.gpu


def _domain(problem, **kw):
    from waveqlab3d_q_gpu_b200.domain import Domain
    return Domain(problem, **kw)


OPERATORS = [("upwind", 4), ("upwind", 6), ("upwind_drp", 6)]


def _upwind(p, op=("upwind", 4)):
    p.fd_type, p.order = op
    return p


@pytest.mark.parametrize("op", sorted(ORDER6_PIN))
def test_elastic_order6_upwind_pin(wql3d_lib, oracle_lib, op):
    """test_elastic_upwind_o6 / test_elastic_upwind_drp_o6: the GPU final
    max|field| equals the published 5 digits and the oracle's fields to 1e-12."""
    p = pin_case(fd_type=op[0], order=op[1])
    g = _domain(p, nsteps_hint=p.nt())
    for n in range(1, p.nt() + 1):
        g.time_step_RK(n)
    mg, _, _ = g.final_state()
    assert round_sig(mg) == ORDER6_PIN[op], mg
    o = oracle_lib.OracleDomain(p)
    o.run(p.nt())
    assert rel_l2(g.fields(), o.fields()) < 1e-12


@pytest.mark.parametrize("response", ["anelastic-Q8", "anelastic-Q4"])
def test_anelastic_upwind4_dynamic_pin(wql3d_lib, oracle_lib, response):
    """test_anelastic_Q8_dynamic / test_anelastic_Q4_dynamic: GPU final
    max|field| and max|memory variable| equal the published 5 digits and the
    oracle's to 1e-11; fields and memory variables to 1e-11."""
    p = upwind4_pin_case(response)
    g = _domain(p, nsteps_hint=p.nt())
    for n in range(1, p.nt() + 1):
        g.time_step_RK(n)
    mg, eg, _ = g.final_state()
    assert (round_sig(mg), round_sig(eg)) == UPWIND4_PIN[response], (mg, eg)
    o = oracle_lib.OracleDomain(p)
    o.run(p.nt())
    mo, eo, _ = o.final_state()
    assert abs(mg - mo) <= 1e-11 * mo and abs(eg - eo) <= 1e-11 * eo
    assert rel_l2(g.fields(), o.fields()) < 1e-11
    assert rel_l2(g.eta(), o.eta()) < 1e-11


@pytest.mark.parametrize("op", OPERATORS)
@pytest.mark.parametrize("mesh", ["cartesian", "curvilinear"])
@pytest.mark.parametrize("response", ["elastic", "anelastic-Q8", "anelastic-fQ8"])
@pytest.mark.parametrize("pml", [False, True])
def test_upwind_single_stage_random_state(wql3d_lib, oracle_lib, op, mesh, response, pml):
    """Two RK stages from a random state (every closure row and the interior
    see nonzero data): rates and fields to 1e-12 relative."""
    p = _upwind(small_case(mesh=mesh, response=response, pml=pml), op)
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


@pytest.mark.parametrize("op", OPERATORS)
@pytest.mark.parametrize("mesh", ["cartesian", "curvilinear"])
def test_upwind_multi_step_run(wql3d_lib, oracle_lib, op, mesh):
    """40 graph-captured steps from rest, Q4 + PML with sources, SATs and
    stations: fields, memory variables and seismograms to 1e-11."""
    p = _upwind(small_case(mesh=mesh, response="anelastic-Q4", pml=True), op)
    nsteps = 40
    o = oracle_lib.OracleDomain(p)
    so = o.run(nsteps)[0]
    g = _domain(p, nsteps_hint=nsteps)
    g.run(nsteps)
    sg = g.seismograms()
    assert rel_l2(g.fields(), o.fields()) < 1e-11
    assert rel_l2(g.eta(), o.eta()) < 1e-11
    assert sg.shape == so.shape
    assert rel_l2(sg[:, :, 1:], so[:, :, 1:]) < 1e-11
    assert np.abs(so[:, :, 1:]).max() > 0.0


@pytest.mark.parametrize("op", OPERATORS)
def test_upwind_two_block_locked(wql3d_lib, oracle_lib, op):
    """Two curvilinear blocks with a locked interface under the upwind
    operators (interface SAT with the operator's tau0), 20 steps: both blocks
    to 1e-11."""
    from cases import two_block_case
    p = _upwind(two_block_case(mesh="curvilinear", coupling="locked", response="anelastic-Q8", pml=True), op)
    nsteps = 20
    o = oracle_lib.OracleDomain(p)
    o.run(nsteps)
    g = _domain(p, nsteps_hint=nsteps)
    g.run(nsteps)
    for b in (0, 1):
        assert rel_l2(g.fields(b), o.fields(b)) < 1e-11
        assert rel_l2(g.eta(b), o.eta(b)) < 1e-11
