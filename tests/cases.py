"""Shared test problems.

``pin_case`` is inputfile/test_elastic_traditional_o6.in of the reference:
41^3 Cartesian block on [-2,2]^3, traditional order 6, rho_s_p = (2.7,
3.464, 6), all faces absorbing, Cos-Bell source (t0 = 0.05, M_xz = -10) at
the origin with the 9-point delta, CFL 0.2, t_final 0.02 (6 steps).  Its
published final state is ``Elastic final state: max|field|=1.6623128367649574E+02``
(PHASE5_TRADITIONAL_CARTESIAN_RHS.md:35 of the reference).
"""
import numpy as np

from waveqlab3d_q_gpu_b200.problem import AnelasticParams, Block, Problem, Source

PIN_MAX_FIELD = 1.6623128367649574e02

# inputfile/test_elastic_locked_interface_o6.in: published per-block maxima of
# the final state, 5 digits (CODEX_PUNAKHA_HANDOFF.md:142-143,
# PHASE2_SCRATCH_MEMORY_AUDIT.md:222-223 of the reference)
LOCKED_PIN_BLOCK_MAX = (2.0699e03, 1.6389e03)

# inputfile/test_anelastic_Q8_dynamic.in / test_anelastic_Q4_dynamic.in
# (upwind order 4): published final max|field| and max|memory variable|,
# 5 digits (ACCELERATOR_RUNTIME.md:176-177, NVHPC_shutdown_regression_fix.md:35-41)
UPWIND4_PIN = {"anelastic-Q8": (1.8221e02, 1.4544e01), "anelastic-Q4": (1.8221e02, 1.1049e01)}

# inputfile/test_elastic_upwind_o6.in / test_elastic_upwind_drp_o6.in: the
# 41^3 case of ``pin_case`` with fd_type 'upwind' / 'upwind_drp', order 6;
# published final max|field|, 5 digits (PHASE2_SCRATCH_MEMORY_AUDIT.md:190-191)
ORDER6_PIN = {("upwind", 6): 1.6563e02, ("upwind_drp", 6): 1.6567e02}


def pin_case(**kw):
    b = Block(nqrs=(41, 41, 41), aqrs=(-2.0, -2.0, -2.0), bqrs=(2.0, 2.0, 2.0), rho_s_p=(2.7, 3.464, 6.0),
              sources=[Source("Cos-Bell", 0.0, 0.05, 0.0, 0.0, 0.0, 0.0, -10.0, 0.0, 0.0, 0.0, 0.0)])
    return Problem(blocks=[b], t_final=0.02, CFL=0.2, source_order=4, source_alpha=0, **kw)


def locked_pin_case(**kw):
    """inputfile/test_elastic_locked_interface_o6.in of the reference: two 41^3
    Cartesian traditional-6 blocks on [-2,0] x [-1,1]^2 and [0,2] x [-1,1]^2
    meeting at x = 0 with a locked interface, absorbing SATs on every outer
    face, rho_s_p = (2.7, 3.464, 6); the tensor_listU row of block 1,
    'Cos-Bell' 0 0.05 -0.25 0 0 0 -10 0 0 0 0 0, is a Cos-Bell moment
    (t_init 0.05, M_xx = -0.25, M_xz = -10) at the origin, a node of block 1's
    interface face, with the 9-point delta (alpha 0); block 2 has no source.
    CFL 0.2, t_final 0.15: 103 steps, long enough for the wave to cross the
    interface and reach the outer y / z faces."""
    src = [Source("Cos-Bell", 0.0, 0.05, -0.25, 0.0, 0.0, 0.0, -10.0, 0.0, 0.0, 0.0, 0.0)]
    b1 = Block(nqrs=(41, 41, 41), aqrs=(-2.0, -1.0, -1.0), bqrs=(0.0, 1.0, 1.0), rho_s_p=(2.7, 3.464, 6.0),
               lqrs=(1, 1, 1), rqrs=(0, 1, 1), sources=src)
    b2 = Block(nqrs=(41, 41, 41), aqrs=(0.0, -1.0, -1.0), bqrs=(2.0, 1.0, 1.0), rho_s_p=(2.7, 3.464, 6.0),
               lqrs=(0, 1, 1), rqrs=(1, 1, 1))
    from waveqlab3d_q_gpu_b200.problem import InterfaceParams
    return Problem(blocks=[b1, b2], t_final=0.15, CFL=0.2, source_order=4, source_alpha=0,
                   interface=InterfaceParams(coupling="locked"), **kw)


def upwind4_pin_case(response="anelastic-Q8", **kw):
    """inputfile/test_anelastic_Q8_dynamic.in (and its Q4 twin) of the reference:
    the 41^3 block, absorbing faces and Cos-Bell M_xz source of ``pin_case``
    with fd_type = 'upwind', order = 4, CFL 0.25, t_final 0.02 (5 steps) and
    Qs0 = 100, Qp0 = 50, fref = 1 (default band 0.05-20 Hz)."""
    b = Block(nqrs=(41, 41, 41), aqrs=(-2.0, -2.0, -2.0), bqrs=(2.0, 2.0, 2.0), rho_s_p=(2.7, 3.464, 6.0),
              sources=[Source("Cos-Bell", 0.0, 0.05, 0.0, 0.0, 0.0, 0.0, -10.0, 0.0, 0.0, 0.0, 0.0)])
    return Problem(blocks=[b], response=response, t_final=0.02, CFL=0.25, source_order=4, source_alpha=0,
                   anelastic=AnelasticParams(Qs0=100.0, Qp0=50.0, fref=1.0), fd_type="upwind", order=4, **kw)


def round_sig(v, digits=5):
    """v rounded to `digits` significant digits (the reference prints ES11.4 / 5 digits)."""
    return float("%.*E" % (digits - 1, v))


def curvilinear_coords(nq, nr, ns, L=(2.0, 2.4, 2.2), amp=0.04, seed=0):
    """Smooth non-orthogonal mapping of the unit cube (x fastest; shape (3, ns, nr, nq))."""
    q = np.linspace(0.0, 1.0, nq)[None, None, :]
    r = np.linspace(0.0, 1.0, nr)[None, :, None]
    s = np.linspace(0.0, 1.0, ns)[:, None, None]
    x = L[0] * q + amp * np.sin(2 * np.pi * r) * np.sin(np.pi * s)
    y = L[1] * r + amp * np.sin(np.pi * q) * np.cos(np.pi * s) + 0.3 * amp * q * s
    z = L[2] * s + amp * np.sin(2 * np.pi * q) * np.sin(np.pi * r) + 0.5 * amp * np.cos(np.pi * q * r)
    shape = (ns, nr, nq)
    return np.stack([np.broadcast_to(x, shape), np.broadcast_to(y, shape), np.broadcast_to(z, shape)]).copy()


def small_case(mesh="cartesian", response="elastic", pml=False, n=(21, 23, 25), bc=((2, 1, 3), (1, 3, 1)),
               sources=True, receivers=True, hetero=True, seed=1):
    rng = np.random.default_rng(seed)
    nq, nr, ns = n
    kw = {}
    if mesh == "curvilinear":
        kw["coords"] = curvilinear_coords(nq, nr, ns)
    if hetero:
        rho = 2.6 + 0.2 * rng.random((ns, nr, nq))
        cs = 3.3 + 0.3 * rng.random((ns, nr, nq))
        cp = np.sqrt(3.0) * cs
        kw["material"] = np.stack([rho * (cp ** 2 - 2 * cs ** 2), rho * cs ** 2, rho])
    srcs = []
    if sources:
        srcs = [Source("ricker", 8.0, 0.1, 1.0, 1.0, 1.0, 0.3, -0.2, 0.1, 0.9, 1.1, 1.05),
                Source("gaussian", 30.0, 0.05, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.25, 0.3, 0.35)]
    rec = None
    if receivers:
        rec = np.array([[0.0, 0.5, 0.5], [0.0, 1.0, 1.2], [1.0, 1.2, 1.1], [1.5, 0.2, 2.0]])
    b = Block(nqrs=n, aqrs=(0.0, 0.0, 0.0), bqrs=(2.0, 2.4, 2.2), rho_s_p=(2.67, 3.464, 6.0),
              lqrs=bc[0], rqrs=bc[1], sources=srcs, receivers=rec, **kw)
    if pml:
        b.pml_lqrs = (False, True, True)
        b.pml_rqrs = (True, True, True)
        b.npml = 7
        b.lqrs = (2, 1, 1)
        b.rqrs = (1, 1, 1)
    an = AnelasticParams(Qs0=40.0, Qp0=80.0, fref=1.0, fmin=0.05, fmax=20.0, gamma=0.6, f_transition=1.0)
    if response == "anelastic-fQ8":
        an.tau = list(np.exp(np.linspace(np.log(0.008), np.log(3.0), 8)))
        an.strength_s = list(0.004 + 0.001 * np.arange(8))
        an.strength_p = list(0.002 + 0.0007 * np.arange(8))
    p = Problem(blocks=[b], response=response, type_of_mesh=mesh, t_final=0.2, CFL=0.4, source_order=4,
                anelastic=an)
    return p


def random_state(problem, seed=3, scale=1.0):
    rng = np.random.default_rng(seed)
    out = []
    for b in problem.blocks:
        nq, nr, ns = b.nqrs
        F = scale * rng.standard_normal((9, ns, nr, nq))
        DF = scale * rng.standard_normal((9, ns, nr, nq))
        out.append((F, DF))
    return out


def rel_l2(a, b):
    a = np.asarray(a, float).ravel()
    b = np.asarray(b, float).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def tpv5_case(serial_shared=False, n=21, t_final=0.5):
    """test_problems/test_rup_cart_fric.in of the reference: two 21^3 Cartesian
    blocks on [-3,0] and [0,3] x [6,9] x [-1.5,1.5] meeting at x = 0, TPV5
    slip-weakening fault (prestress and strength of
    src/Interface_Condition.f90:1283-1294, 1822-1830), free surface at y = 6,
    absorbing elsewhere, CFL 0.5, stations at the fault centre on each side."""
    from waveqlab3d_q_gpu_b200.problem import InterfaceParams
    b1 = Block(nqrs=(n, n, n), aqrs=(-3.0, 6.0, -1.5), bqrs=(0.0, 9.0, 1.5), rho_s_p=(2.67, 3.464, 6.0),
               lqrs=(1, 2, 1), rqrs=(0, 1, 1), receivers=np.array([[-0.0, 7.5, 0.0]]))
    b2 = Block(nqrs=(n, n, n), aqrs=(0.0, 6.0, -1.5), bqrs=(3.0, 9.0, 1.5), rho_s_p=(2.67, 3.464, 6.0),
               lqrs=(0, 2, 1), rqrs=(1, 1, 1), receivers=np.array([[0.0, 7.5, 0.0]]))
    ip = InterfaceParams(coupling="slip-weakening_friction", problem="TPV5", serial_shared=serial_shared)
    return Problem(blocks=[b1, b2], response="elastic", type_of_mesh="cartesian", t_final=t_final, CFL=0.5,
                   interface=ip, w_stride=1)


def two_block_case(mesh="cartesian", coupling="locked", response="elastic", n=(15, 17, 19), seed=4,
                   serial_shared=False, pml=False):
    """Two blocks meeting at a q-direction interface, with a heterogeneous
    medium (different on each side) and, for 'curvilinear', a smooth
    non-orthogonal mapping that is continuous across the interface so the
    two face traces sit at the same points.  Friction laws get uniform
    prestress / strength maps that put part of the fault above strength."""
    from waveqlab3d_q_gpu_b200.problem import InterfaceParams
    rng = np.random.default_rng(seed)
    nq, nr, ns = n
    L = (2.0, 2.4, 2.2)
    blocks = []
    for side in range(2):
        kw = {}
        q = np.linspace(0.0, 1.0, nq)
        xi = 0.5 * q if side == 0 else 0.5 + 0.5 * q     # global q in [0, 1]
        if mesh == "curvilinear":
            xi3 = xi[None, None, :]
            r = np.linspace(0.0, 1.0, nr)[None, :, None]
            s = np.linspace(0.0, 1.0, ns)[:, None, None]
            amp = 0.04
            x = 2 * L[0] * xi3 - L[0] + amp * np.sin(2 * np.pi * r) * np.sin(np.pi * s) * np.sin(np.pi * xi3)
            y = L[1] * r + amp * np.sin(np.pi * xi3) * np.cos(np.pi * s)
            z = L[2] * s + amp * np.sin(2 * np.pi * xi3) * np.sin(np.pi * r)
            shape = (ns, nr, nq)
            kw["coords"] = np.stack([np.broadcast_to(x, shape), np.broadcast_to(y, shape),
                                     np.broadcast_to(z, shape)]).copy()
        rho = (2.6 + 0.15 * side) + 0.2 * rng.random((ns, nr, nq))
        cs = (3.2 + 0.2 * side) + 0.3 * rng.random((ns, nr, nq))
        cp = np.sqrt(3.0) * cs
        kw["material"] = np.stack([rho * (cp ** 2 - 2 * cs ** 2), rho * cs ** 2, rho])
        a = (-L[0], 0.0, 0.0) if side == 0 else (0.0, 0.0, 0.0)
        bq = (0.0, L[1], L[2]) if side == 0 else (L[0], L[1], L[2])
        lq = (1, 2, 1) if side == 0 else (0, 2, 1)
        rq = (0, 1, 3) if side == 0 else (1, 1, 3)
        srcs = [Source("ricker", 8.0, 0.1, 1.0, 0.8, 1.2, 0.3, -0.2, 0.1,
                       -0.9 if side == 0 else 0.8, 1.1, 1.05)]
        rec = np.array([[-0.5 if side == 0 else 0.5, 1.0, 1.2], [0.0, 1.2, 1.1]])
        b = Block(nqrs=n, aqrs=a, bqrs=bq, rho_s_p=(2.67, 3.464, 6.0), lqrs=lq, rqrs=rq, sources=srcs,
                  receivers=rec, **kw)
        if pml:
            b.pml_lqrs = (side == 0, False, False)
            b.pml_rqrs = (side == 1, True, False)
            b.npml = 5
        blocks.append(b)
    ip = InterfaceParams(coupling=coupling, serial_shared=serial_shared)
    if coupling != "locked":
        ip.tau0_n = np.full((ns, nr), -120.0)
        ip.tau0_m = np.full((ns, nr), 5.0)
        yy = np.linspace(0.0, 1.0, nr)[None, :]
        zz = np.linspace(0.0, 1.0, ns)[:, None]
        ip.tau0_l = 70.0 + 12.0 * np.exp(-((yy - 0.5) ** 2 + (zz - 0.5) ** 2) / 0.05)
        ip.fs_map = np.full((ns, nr), 0.677)
    an = AnelasticParams(Qs0=40.0, Qp0=80.0, fref=1.0, fmin=0.05, fmax=20.0)
    return Problem(blocks=blocks, response=response, type_of_mesh=mesh, t_final=0.2, CFL=0.4, source_order=4,
                   anelastic=an, interface=ip)


def mms_case(n=21, mesh="cartesian", bc=((2, 1, 3), (1, 3, 1)), t_final=0.1, hetero=False, seed=6):
    """Manufactured-solution problem (src/mms.f90:136-235, nt = 2, nx = ny = nz = 1)
    on the box [0.1, 1.1] x [0.2, 1.2] x [0.15, 1.15]: forcing in the rates,
    exact boundary data in the face SATs.  'curvilinear' perturbs the interior
    of the mesh smoothly (faces stay planar)."""
    from waveqlab3d_q_gpu_b200.problem import MMSParams
    kw = {}
    a, bq = (0.1, 0.2, 0.15), (1.1, 1.2, 1.15)
    if mesh == "curvilinear":
        q = np.linspace(0.0, 1.0, n)[None, None, :]
        r = np.linspace(0.0, 1.0, n)[None, :, None]
        s = np.linspace(0.0, 1.0, n)[:, None, None]
        bump = 0.03 * np.sin(np.pi * q) * np.sin(np.pi * r) * np.sin(np.pi * s)
        shape = (n, n, n)
        x = a[0] + q * (bq[0] - a[0]) + bump
        y = a[1] + r * (bq[1] - a[1]) + 0.7 * bump
        z = a[2] + s * (bq[2] - a[2]) - 0.5 * bump
        kw["coords"] = np.stack([np.broadcast_to(x, shape), np.broadcast_to(y, shape),
                                 np.broadcast_to(z, shape)]).copy()
    if hetero:
        rng = np.random.default_rng(seed)
        rho = 2.6 + 0.1 * rng.random((n, n, n))
        cs = 3.3 + 0.2 * rng.random((n, n, n))
        cp = np.sqrt(3.0) * cs
        kw["material"] = np.stack([rho * (cp ** 2 - 2 * cs ** 2), rho * cs ** 2, rho])
    b = Block(nqrs=(n, n, n), aqrs=a, bqrs=bq, rho_s_p=(2.67, 3.464, 6.0), lqrs=bc[0], rqrs=bc[1], **kw)
    return Problem(blocks=[b], response="elastic", type_of_mesh=mesh, t_final=t_final, CFL=0.5, mms=MMSParams())


def mms_error(fields, exact):
    return float(np.linalg.norm(fields - exact) / np.linalg.norm(exact))


def tpv101_case(serial_shared=False, n=21, t_final=0.5, problem="TPV101"):
    """The TPV5 geometry with the reference's rate-and-state law and TPV101 /
    TPV102 prestress (src/Interface_Condition.f90:386-436, 918-1263,
    2324-2385): uniform background stress (-120, 0, -120, 0, 75, 0), a
    nucleation patch of radius 3 at (y, z) = (7.5, 0) ramped in over 1 s, the
    state starting at 0 as the reference leaves it."""
    from waveqlab3d_q_gpu_b200.problem import InterfaceParams
    p = tpv5_case(serial_shared=serial_shared, n=n, t_final=t_final)
    p.interface = InterfaceParams(coupling="rate-and-state_friction", problem=problem, serial_shared=serial_shared)
    return p


def tpv28_case(grid, serial_shared=False, n=21, t_final=0.5):
    """test_problems/test_rup_curv_fric.in of the reference: two 21^3
    curvilinear blocks on [-3,0] and [0,3] x [6,9] x [-1.5,1.5] whose shared
    q-face carries the 'analytical_test_problem' fault profile (lc = 1 on
    block 1, rc = 1 on block 2; src/grid.f90:777-829), TPV28 slip-weakening
    prestress and strength (src/Interface_Condition.f90:1459-1474, 2049-2076),
    free surface at y = 6, absorbing elsewhere, CFL 0.5, stations at the fault
    centre on each side.  grid(surfaces, nqrs) builds the volume mesh (the
    oracle's or the device's transfinite interpolation)."""
    from waveqlab3d_q_gpu_b200.mesh import block_surfaces
    from waveqlab3d_q_gpu_b200.problem import InterfaceParams
    blocks = []
    for side in range(2):
        a = (-3.0, 6.0, -1.5) if side == 0 else (0.0, 6.0, -1.5)
        b = (0.0, 9.0, 1.5) if side == 0 else (3.0, 9.0, 1.5)
        lc, rc = (1.0, 0.0) if side == 0 else (0.0, 1.0)
        X = grid(block_surfaces((n, n, n), a, b, lc, rc, "analytical_test_problem"), (n, n, n))
        blocks.append(Block(nqrs=(n, n, n), aqrs=a, bqrs=b, rho_s_p=(2.67, 3.464, 6.0),
                            lqrs=(1, 2, 1) if side == 0 else (0, 2, 1), rqrs=(0, 1, 1) if side == 0 else (1, 1, 1),
                            coords=X, receivers=np.array([[0.0, 7.5, 0.0]])))
    ip = InterfaceParams(coupling="slip-weakening_friction", problem="TPV28", serial_shared=serial_shared)
    return Problem(blocks=blocks, response="elastic", type_of_mesh="curvilinear", t_final=t_final, CFL=0.5,
                   interface=ip, w_stride=1)
