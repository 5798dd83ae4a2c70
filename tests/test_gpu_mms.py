"""Manufactured solution on the CUDA path: parity with the oracle and the
convergence order (src/mms.f90:136-235)."""
import numpy as np
import pytest

from cases import mms_case, mms_error, rel_l2

pytestmark = pytest.mark.gpu


def _domain(problem, **kw):
    from waveqlab3d_q_gpu_b200.domain import Domain
    return Domain(problem, **kw)


@pytest.mark.parametrize("mesh", ["cartesian", "curvilinear"])
def test_mms_matches_oracle(wql3d_lib, oracle_lib, mesh):
    """Forcing and exact boundary data on the GPU equal the oracle's to 1e-11
    after 10 steps from the exact state (heterogeneous medium, mixed faces)."""
    p = mms_case(n=21, mesh=mesh, hetero=True)
    o = oracle_lib.OracleDomain(p)
    u0 = o.mms_exact(0.0)
    o.set_fields(u0)
    g = _domain(p, nsteps_hint=10)
    g.set_fields(u0)
    dt = p.dt()
    o.run(10, dt=dt)
    g.run(10, dt=dt)
    assert rel_l2(g.fields(), o.fields()) < 1e-11


@pytest.mark.parametrize("mesh", ["cartesian", "curvilinear"])
def test_mms_convergence_order(wql3d_lib, oracle_lib, mesh):
    """Relative L2 error of all nine fields at t = 0.1 on 21^3, 41^3, 81^3:
    order > 3.9 between each pair (6th-order interior, 3rd-order closures)."""
    errs = []
    for n in (21, 41, 81):
        p = mms_case(n=n, mesh=mesh)
        o = oracle_lib.OracleDomain(p) if n <= 21 else None
        exact0 = o.mms_exact(0.0) if o is not None else None
        g = _domain(p, nsteps_hint=p.nt() + 2)
        if exact0 is None:
            exact0 = _exact_host(p, 0.0)
        g.set_fields(exact0)
        nt = p.nt()
        dt = p.t_final / nt
        g.run(nt, dt=dt)
        errs.append(mms_error(g.fields(), _exact_host(p, nt * dt)))
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert min(rates) > 3.9, (errs, rates)


def _exact_host(p, t):
    """u* of src/mms.f90:136-148 on the block's coordinates (nt = 2, nx = ny = nz = 1)."""
    b = p.blocks[0]
    nq, nr, ns = b.nqrs
    if b.coords is not None:
        X = b.coords
    else:
        x = np.linspace(b.aqrs[0], b.bqrs[0], nq)[None, None, :]
        y = np.linspace(b.aqrs[1], b.bqrs[1], nr)[None, :, None]
        z = np.linspace(b.aqrs[2], b.bqrs[2], ns)[:, None, None]
        X = np.broadcast_arrays(x, y, z)
    m = p.mms
    ct = np.cos(m.nt * np.pi * t)
    a = np.sin(m.nx * np.pi * X[0]) * np.sin(m.ny * np.pi * X[1]) * np.sin(m.nz * np.pi * X[2])
    c = np.cos(m.nx * np.pi * X[0]) * np.cos(m.ny * np.pi * X[1]) * np.cos(m.nz * np.pi * X[2])
    u = np.empty((9, ns, nr, nq))
    u[:3] = ct * a
    u[3:] = ct * c
    return u
