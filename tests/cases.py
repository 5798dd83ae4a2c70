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


def pin_case(**kw):
    b = Block(nqrs=(41, 41, 41), aqrs=(-2.0, -2.0, -2.0), bqrs=(2.0, 2.0, 2.0), rho_s_p=(2.7, 3.464, 6.0),
              sources=[Source("Cos-Bell", 0.0, 0.05, 0.0, 0.0, 0.0, 0.0, -10.0, 0.0, 0.0, 0.0, 0.0)])
    return Problem(blocks=[b], t_final=0.02, CFL=0.2, source_order=4, source_alpha=0, **kw)


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
