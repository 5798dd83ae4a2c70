"""The oracle's rate-and-state interface (TPV101 / TPV102) on CPU: the run
stays finite with the state evolving and slip accumulating, the initial
velocity and state follow init_vel_state, and TPV101 and TPV102 (the same
law and prestress in the reference) give the same run."""
import numpy as np

from cases import tpv101_case


def test_rate_state_runs_and_evolves(oracle_lib):
    p = tpv101_case()
    o = oracle_lib.OracleDomain(p)
    o.run(6)
    W = o.fault("state")
    S = o.fault("S")
    Uhat = o.fault("Uhat")
    F = [o.fields(b) for b in (0, 1)]
    assert all(np.isfinite(f).all() for f in F)
    assert np.isfinite(W).all() and np.abs(W).max() > 0
    assert np.isfinite(S).all() and S[3].max() > 0          # slip accumulates
    # with the state at 0 the fault slides everywhere: slip rates are positive
    Svel = o.fault("Svel")
    assert np.sqrt(Svel[1] ** 2 + Svel[2] ** 2).min() > 0


def test_initial_state_and_velocity(oracle_lib):
    """init_vel_state (src/Interface_Condition.f90:2722-2786): block 1's v_z is
    -Vin/2 and the state is the steady value of the background traction,
    W = a log(2 sinh(T0_l / (a sigma_n))) - a log(Vin / V0) with T0_l = 75,
    sigma_n = 120, a = 0.008 inside the velocity-weakening patch."""
    p = tpv101_case()
    o = oracle_lib.OracleDomain(p)
    F1 = o.fields(0)
    assert np.all(F1[2] == -0.5e-12) and np.all(o.fields(1) == 0.0)
    a, Vin, V0 = 0.008, 1e-12, 1e-6
    W0 = a * np.log(2 * np.sinh(75.0 / (a * 120.0))) - a * np.log(Vin / V0)
    W = o.fault("state")
    assert np.allclose(W, W0, rtol=0, atol=1e-12)


def test_tpv101_equals_tpv102(oracle_lib):
    a = oracle_lib.OracleDomain(tpv101_case(problem="TPV101"))
    b = oracle_lib.OracleDomain(tpv101_case(problem="TPV102"))
    a.run(3)
    b.run(3)
    for k in (0, 1):
        assert np.array_equal(a.fields(k), b.fields(k))
    assert np.array_equal(a.fault("state"), b.fault("state"))
