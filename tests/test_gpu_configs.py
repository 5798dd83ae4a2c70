"""The CUDA path on the reference's locked-interface regression input and on
the benchmark configuration builders at reduced size, against the CPU oracle.

* inputfile/test_elastic_locked_interface_o6.in (two 41^3 Cartesian blocks,
  locked interface, 103 steps): the published per-block maxima of the final
  state (5 digits) and the oracle's fields.
* configs.hill_two_block_q8 (curvilinear two-block Q8 + PML hill, the
  default bench workload) and configs.cartesian_101 (plain Cartesian block
  with a free surface and an explosive Ricker source) built at n = 41: the
  same builders, meshes, media, sources and stations as the full-size runs.
"""
import numpy as np
import pytest

from cases import LOCKED_PIN_BLOCK_MAX, locked_pin_case, rel_l2, round_sig

pytestmark = pytest.mark.gpu


def _domain(problem, **kw):
    from waveqlab3d_q_gpu_b200.domain import Domain
    return Domain(problem, **kw)


def _compare_run(g, o, nblocks, so, tol=1e-11, eta=False):
    for b in range(nblocks):
        assert rel_l2(g.fields(b), o.fields(b)) < tol, b
        if eta:
            assert rel_l2(g.eta(b), o.eta(b)) < tol, b
        if so[b] is not None and so[b].size:
            sg = g.seismograms(b)
            assert sg.shape == so[b].shape
            assert np.allclose(sg[:, :, 0], so[b][:, :, 0], rtol=0, atol=1e-15)
            assert rel_l2(sg[:, :, 1:], so[b][:, :, 1:]) < tol


def test_locked_interface_o6_block_maxima(wql3d_lib, oracle_lib):
    """test_elastic_locked_interface_o6: GPU block maxima equal the published
    2.0699E+03 / 1.6389E+03 to the printed digits and the oracle's to 1e-11;
    fields of both blocks equal the oracle's to 1e-11."""
    p = locked_pin_case()
    nt = p.nt()
    g = _domain(p, nsteps_hint=nt)
    g.run(nt)
    mg, eg, bg = g.final_state()
    assert [round_sig(v) for v in bg[:2]] == list(LOCKED_PIN_BLOCK_MAX), bg
    o = oracle_lib.OracleDomain(p)
    o.run(nt)
    mo, _, bo = o.final_state()
    for b in range(2):
        assert abs(bg[b] - bo[b]) <= 1e-11 * bo[b]
        assert rel_l2(g.fields(b), o.fields(b)) < 1e-11


def test_hill_two_block_q8_reduced(wql3d_lib, oracle_lib):
    """configs.hill_two_block_q8 at n = 41 (two 21 x 41 x 41 curvilinear blocks,
    Gaussian hill + seeded bumps, layered Vs, per-point Q8, 6-point PML on the
    sides and bottom, locked interface, Ricker double couple, 5 x 5 surface
    stations), 30 steps: fields, memory variables and stations to 1e-11."""
    from waveqlab3d_q_gpu_b200 import configs
    p = configs.hill_two_block_q8(n=41, h=0.25, npml=6, steps=30, nrec=5)
    nsteps = 30
    o = oracle_lib.OracleDomain(p)
    so = o.run(nsteps)
    g = _domain(p, nsteps_hint=nsteps)
    g.run(nsteps)
    _compare_run(g, o, 2, so, eta=True)
    assert np.abs(so[0][:, :, 1:]).max() > 0.0
    mg, eg, _ = g.final_state()
    mo, eo, _ = o.final_state()
    assert abs(mg - mo) <= 1e-11 * mo and abs(eg - eo) <= 1e-11 * eo


def test_cartesian_101_reduced(wql3d_lib, oracle_lib):
    """configs.cartesian_101 at n = 41 (free surface on the q-min face,
    absorbing elsewhere, explosive Ricker source at the centre, 10 x 10
    surface stations), 60 steps: fields and stations to 1e-11."""
    from waveqlab3d_q_gpu_b200 import configs
    p = configs.cartesian_101(n=41, steps=60)
    nsteps = p.nt()
    assert nsteps == 60
    o = oracle_lib.OracleDomain(p)
    so = o.run(nsteps)
    g = _domain(p, nsteps_hint=nsteps)
    g.run(nsteps)
    _compare_run(g, o, 1, so)
    assert np.abs(so[0][:, :, 1:]).max() > 0.0
