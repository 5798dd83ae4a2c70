"""Synthetic workloads with the shapes of the benchmark configurations.

There is no public dataset behind these runs: every medium, mesh and source
is generated here from fixed seeds, in the reference's units (km, km/s,
g/cm^3, s).

* :func:`cartesian_101` -- plain FP64 single Cartesian block, 101^3 points at
  h = 0.1 km, homogeneous medium (Vp 6, Vs 3.464, rho 2.67), free surface on
  the q-min face (depth axis x), absorbing SAT elsewhere, explosive
  moment-tensor source at the centre node with a Ricker wavelet f0 = 2 Hz
  (delay 1.2/f0), CFL 0.5 (500 steps), 10 x 10 receivers on the free surface.
* :func:`curvilinear_q8` -- scaled-down or full curvilinear block with a
  Gaussian hill plus seeded bumps, 20-point PML on the sides and bottom,
  layered Vs, Q8 with per-point Qs = 50 Vs, Qp = 2 Qs.
"""
from __future__ import annotations

import math

import numpy as np

from .problem import AnelasticParams, Block, Problem, Source


def cartesian_101(n: int = 101, steps: int = 500) -> Problem:
    h = 0.1
    L = h * (n - 1)
    c = 0.5 * L
    src = Source("ricker", duration=2.0, t_init=1.2 / 2.0, mxx=1.0, myy=1.0, mzz=1.0, x=c, y=c, z=c)
    ys = np.linspace(0.05 * L, 0.95 * L, 10)
    rec = np.array([[0.0, y, z] for z in ys for y in ys])
    b = Block(nqrs=(n, n, n), aqrs=(0.0, 0.0, 0.0), bqrs=(L, L, L), rho_s_p=(2.67, 3.464, 6.0),
              lqrs=(2, 1, 1), rqrs=(1, 1, 1), sources=[src], receivers=rec)
    p = Problem(blocks=[b], response="elastic", type_of_mesh="cartesian", CFL=0.5, source_order=4,
                source_alpha=0, w_stride=1)
    p.t_final = steps * p.dt() * (1.0 + 1e-9)
    return p


def hill_coords(nq: int, nr: int, ns: int, h: float, seed: int = 2, amp: float = 0.8, sigma: float = 2.5,
                bump: float = 0.03) -> np.ndarray:
    """Curvilinear mesh: depth axis q (x = depth), surface x = -topography(y, z).

    Transfinite vertical stretch between the topographic surface and a flat
    bottom, as mesh_source = 'file' would supply (src/grid.f90:147-212).
    """
    rng = np.random.default_rng(seed)
    Ly, Lz, Lx = h * (nr - 1), h * (ns - 1), h * (nq - 1)
    y = np.linspace(0.0, Ly, nr)
    z = np.linspace(0.0, Lz, ns)
    Y, Z = np.meshgrid(y, z, indexing="xy")  # (ns, nr)
    topo = amp * np.exp(-((Y - 0.5 * Ly) ** 2 + (Z - 0.5 * Lz) ** 2) / (2.0 * sigma ** 2))
    # seeded smooth random bumps
    for _ in range(12):
        cy, cz = rng.uniform(0, Ly), rng.uniform(0, Lz)
        r = rng.uniform(0.5, 1.5)
        topo += bump * rng.standard_normal() * np.exp(-((Y - cy) ** 2 + (Z - cz) ** 2) / (2 * r * r))
    q = np.linspace(0.0, 1.0, nq)
    X = np.empty((3, ns, nr, nq))
    top = -topo[:, :, None]
    X[0] = top + (Lx - top) * q[None, None, :]
    X[1] = Y[:, :, None]
    X[2] = Z[:, :, None]
    return X


def curvilinear_q8(n: int = 201, h: float = 0.05, npml: int = 20, seed: int = 2) -> Problem:
    X = hill_coords(n, n, n, h, seed=seed)
    depth = X[0] - X[0][:, :, :1]
    vs = 2.0 + 1.5 * np.clip(depth / (h * (n - 1)), 0.0, 1.0)
    vp = math.sqrt(3.0) * vs
    rho = 1.7 + 0.2 * vp
    mat = np.stack([rho * (vp ** 2 - 2 * vs ** 2), rho * vs ** 2, rho])
    qs = 1.0 / (50.0 * vs)
    qp = 0.5 * qs
    rng = np.random.default_rng(seed)
    strike, dip, rake = rng.uniform(0, 2 * math.pi), rng.uniform(0.2, 1.4), rng.uniform(-math.pi, math.pi)
    ns_ = np.array([-math.sin(dip) * math.sin(strike), math.sin(dip) * math.cos(strike), -math.cos(dip)])
    ds_ = np.array([math.cos(rake) * math.cos(strike) + math.sin(rake) * math.cos(dip) * math.sin(strike),
                    math.cos(rake) * math.sin(strike) - math.sin(rake) * math.cos(dip) * math.cos(strike),
                    -math.sin(rake) * math.sin(dip)])
    M = np.outer(ns_, ds_) + np.outer(ds_, ns_)
    c = 0.5 * h * (n - 1)
    src = Source("ricker", duration=3.0, t_init=1.2 / 3.0, mxx=M[0, 0], myy=M[1, 1], mzz=M[2, 2], mxy=M[0, 1],
                 mxz=M[0, 2], myz=M[1, 2], x=c, y=c, z=c)
    b = Block(nqrs=(n, n, n), aqrs=(0.0, 0.0, 0.0), bqrs=(h * (n - 1),) * 3, rho_s_p=(2.7, 3.5, 6.06),
              lqrs=(2, 1, 1), rqrs=(1, 1, 1), pml_lqrs=(False, True, True), pml_rqrs=(True, True, True),
              npml=npml, coords=X, material=mat, qs_inv=qs, qp_inv=qp, sources=[src])
    an = AnelasticParams(Qs0=100.0, Qp0=200.0, fref=1.0, fmin=0.05, fmax=20.0)
    return Problem(blocks=[b], response="anelastic-Q8", type_of_mesh="curvilinear", CFL=0.5, source_order=4,
                   anelastic=an, t_final=1.0)


def hill_two_block_q8(n: int = 201, h: float = 0.05, npml: int = 20, seed: int = 2, steps: int = 1500,
                      nrec: int = 10) -> Problem:
    """Curvilinear two-block Q8 + PML workload: an n x n x n-point domain at
    spacing h split at mid-depth into two blocks of (n+1)/2 x n x n points
    that share the locked interface plane (the reference couples blocks only
    across q, the depth axis here).

    * Surface: Gaussian hill of 0.8 km amplitude (sigma 2.5 km) plus seeded
      random bumps of 0.03 km standard amplitude (:func:`hill_coords`); the
      interface plane is flat at half the depth extent, block 2 below it.
    * Vs layered 2.0 -> 3.5 km/s with depth, Vp = sqrt(3) Vs,
      rho = 1.7 + 0.2 Vp (g/cm^3).
    * Q8 with per-point Qs = 50 Vs[km/s], Qp = 2 Qs.
    * Free surface on top, 20-point PML on the four sides of both blocks
      and on the bottom of block 2 (absorbing SAT on those faces).
    * Seeded random double-couple with a Ricker wavelet f0 = 3 Hz at 3/10 of
      the depth below the centre of the surface, nrec x nrec surface stations.
    """
    if n % 2 == 0:
        raise ValueError("n must be odd so that the interface is a grid plane")
    nb = (n + 1) // 2
    Lx = h * (n - 1)
    X = hill_coords(n, n, n, h, seed=seed)
    top = X[0][:, :, :1]
    blocks = []
    rng = np.random.default_rng(seed)
    strike, dip, rake = rng.uniform(0, 2 * math.pi), rng.uniform(0.2, 1.4), rng.uniform(-math.pi, math.pi)
    ns_ = np.array([-math.sin(dip) * math.sin(strike), math.sin(dip) * math.cos(strike), -math.cos(dip)])
    ds_ = np.array([math.cos(rake) * math.cos(strike) + math.sin(rake) * math.cos(dip) * math.sin(strike),
                    math.cos(rake) * math.sin(strike) - math.sin(rake) * math.cos(dip) * math.cos(strike),
                    -math.sin(rake) * math.sin(dip)])
    M = np.outer(ns_, ds_) + np.outer(ds_, ns_)
    c = 0.5 * h * (n - 1)
    src = Source("ricker", duration=3.0, t_init=1.2 / 3.0, mxx=M[0, 0], myy=M[1, 1], mzz=M[2, 2], mxy=M[0, 1],
                 mxz=M[0, 2], myz=M[1, 2], x=0.3 * Lx, y=c, z=c)
    ys = np.linspace(0.05 * Lx, 0.95 * Lx, nrec)
    for side in range(2):
        q = np.linspace(0.0, 1.0, nb)[None, None, :]
        Xb = np.empty((3, n, n, nb))
        if side == 0:
            Xb[0] = top * (1.0 - q) + (0.5 * Lx) * q
            Xb[0][:, :, -1] = 0.5 * Lx
        else:
            Xb[0] = 0.5 * Lx + (0.5 * Lx) * q
            Xb[0][:, :, 0] = 0.5 * Lx
        Xb[1] = X[1][:, :, :nb]
        Xb[2] = X[2][:, :, :nb]
        depth = Xb[0] - top
        vs = 2.0 + 1.5 * np.clip(depth / Lx, 0.0, 1.0)
        vp = math.sqrt(3.0) * vs
        rho = 1.7 + 0.2 * vp
        mat = np.stack([rho * (vp ** 2 - 2 * vs ** 2), rho * vs ** 2, rho])
        qs = 1.0 / (50.0 * vs)
        qp = 0.5 * qs
        if side == 0:
            a, bq = (0.0, 0.0, 0.0), (0.5 * Lx, Lx, Lx)
            lq, rq = (2, 1, 1), (0, 1, 1)
            pl, pr = (False, True, True), (False, True, True)
            srcs = [src] if src.x <= 0.5 * Lx else []
            rec = np.array([[0.0, y, z] for z in ys for y in ys])
        else:
            a, bq = (0.5 * Lx, 0.0, 0.0), (Lx, Lx, Lx)
            lq, rq = (0, 1, 1), (1, 1, 1)
            pl, pr = (False, True, True), (True, True, True)
            srcs = [src] if src.x > 0.5 * Lx else []
            rec = None
        blocks.append(Block(nqrs=(nb, n, n), aqrs=a, bqrs=bq, rho_s_p=(2.7, 3.5, 6.06), lqrs=lq, rqrs=rq,
                            pml_lqrs=pl, pml_rqrs=pr, npml=npml, coords=Xb, material=mat, qs_inv=qs, qp_inv=qp,
                            sources=srcs, receivers=rec))
    from .problem import InterfaceParams
    an = AnelasticParams(Qs0=100.0, Qp0=200.0, fref=1.0, fmin=0.05, fmax=20.0)
    p = Problem(blocks=blocks, response="anelastic-Q8", type_of_mesh="curvilinear", CFL=0.5, source_order=4,
                anelastic=an, interface=InterfaceParams(coupling="locked"), w_stride=1)
    p.t_final = steps * p.dt() * (1.0 + 1e-9)
    return p


def von_karman_field(shape, h: float, a: float = 1.0, hurst: float = 0.2, std: float = 0.05,
                     seed: int = 3) -> np.ndarray:
    """Seeded von Karman random field (3-D power spectrum proportional to
    (1 + k^2 a^2)^-(H + 3/2), correlation length a, Hurst exponent H) with
    zero mean and the given standard deviation, on a grid of spacing h."""
    import scipy.fft as sf
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape).astype(np.float32)
    W = sf.rfftn(w, workers=-1)
    del w
    k = [2.0 * math.pi * sf.fftfreq(n, d=h).astype(np.float32) for n in shape[:-1]]
    k.append(2.0 * math.pi * sf.rfftfreq(shape[-1], d=h).astype(np.float32))
    k2 = (k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2)
    W *= np.power(1.0 + k2 * (a * a), -(hurst + 1.5) / 2.0).astype(np.float32)
    del k2
    f = sf.irfftn(W, s=shape, workers=-1)
    del W
    f -= f.mean()
    f *= std / max(float(f.std()), 1e-30)
    return f.astype(np.float64)


def planar_fault_fq8(nq: int = 512, nr: int = 512, ns: int = 384, h: float = 0.1, seed: int = 3,
                     steps: int = 2000, nrec: int = 4) -> Problem:
    """Two Cartesian blocks of nq/2 x nr x ns points (q the fault-normal axis)
    sharing a planar vertical slip-weakening interface.

    * Medium: Vp 6, Vs 3.464, rho 2.67 perturbed by one seeded von Karman
      field (Hurst 0.2, correlation length 1 km, 5 % standard deviation),
      continuous across the fault.
    * fQ8 anelasticity, Q0 = 100 (Qp0 = 200), gamma = 0.6 above 1 Hz.
    * Linear slip weakening mu_s = 0.70, mu_d = 0.50, Dc = 0.3 m under a
      normal traction of -120 MPa; shear traction 70 MPa with seeded smooth
      5 MPa heterogeneity, and a 3 km square nucleation patch at the fault
      centre loaded to 85 MPa, above the 84 MPa static strength.
    * Absorbing SATs on the outer faces; nrec x nrec stations on each side of
      the fault, one grid plane from it.
    """
    from .problem import InterfaceParams
    if nq % 2:
        raise ValueError("nq must be even: two blocks of nq / 2 points")
    nb = nq // 2
    Lq = h * (2 * nb - 2)
    Lr, Ls = h * (nr - 1), h * (ns - 1)
    d = von_karman_field((ns, nr, 2 * nb - 1), h, seed=seed)
    rng = np.random.default_rng(seed + 1)
    # smooth shear heterogeneity on the fault plane (Gaussian filter of white noise)
    import scipy.ndimage as nd
    het = nd.gaussian_filter(rng.standard_normal((ns, nr)), sigma=max(1.0, 2.0 / h), mode="wrap")
    het *= 5.0 / max(float(het.std()), 1e-30)
    yy = np.arange(nr)[None, :] * h
    zz = np.arange(ns)[:, None] * h
    patch = (np.abs(yy - 0.5 * Lr) <= 1.5) & (np.abs(zz - 0.5 * Ls) <= 1.5)
    tl = np.where(patch, 85.0, 70.0 + het)
    blocks = []
    for side in range(2):
        sl = slice(0, nb) if side == 0 else slice(nb - 1, 2 * nb - 1)
        db = d[:, :, sl]
        vp, vs, rho = 6.0 * (1.0 + db), 3.464 * (1.0 + db), 2.67 * (1.0 + db)
        mat = np.stack([rho * (vp ** 2 - 2 * vs ** 2), rho * vs ** 2, rho])
        x0 = 0.0 if side == 0 else 0.5 * Lq
        xr = (0.5 * Lq - h) if side == 0 else (0.5 * Lq + h)
        ys = np.linspace(0.3 * Lr, 0.7 * Lr, nrec)
        zs = np.linspace(0.3 * Ls, 0.7 * Ls, nrec)
        rec = np.array([[xr, y, z] for z in zs for y in ys])
        blocks.append(Block(nqrs=(nb, nr, ns), aqrs=(x0, 0.0, 0.0), bqrs=(x0 + 0.5 * Lq, Lr, Ls),
                            rho_s_p=(2.67, 3.464, 6.0), lqrs=(1, 1, 1) if side == 0 else (0, 1, 1),
                            rqrs=(0, 1, 1) if side == 0 else (1, 1, 1), material=mat, receivers=rec))
    ip = InterfaceParams(coupling="slip-weakening_friction", fs=0.70, fd=0.50, Dc=0.3,
                         tau0_n=np.full((ns, nr), -120.0), tau0_m=np.zeros((ns, nr)), tau0_l=tl,
                         fs_map=np.full((ns, nr), 0.70))
    an = AnelasticParams(Qs0=100.0, Qp0=200.0, fref=1.0, fmin=0.05, fmax=20.0, gamma=0.6, f_transition=1.0)
    p = Problem(blocks=blocks, response="anelastic-fQ8", type_of_mesh="cartesian", CFL=0.5, source_order=4,
                anelastic=an, interface=ip, w_stride=1)
    p.t_final = steps * p.dt() * (1.0 + 1e-9)
    return p


def adjoint_block(nq: int = 201, nr: int = 201, ns: int = 101, h: float = 0.1, seed: int = 5, nrec: int = 20,
                  anomaly: bool = False, steps: int = 1200) -> Problem:
    """Curvilinear block of the adjoint / gradient configuration: nq x nr x ns
    points at spacing h with the depth axis q (x = depth below a smooth
    seeded topography), smooth layered background Vs 2.0 -> 3.5 km/s with
    depth, Vp = sqrt(3) Vs, rho = 1.7 + 0.2 Vp, optionally a 3 % Gaussian Vs
    anomaly of radius 1.5 km centred 4 km below the surface; one seeded
    double-couple Ricker source (3 Hz) at 2 km depth and nrec x nrec surface
    stations.  Elastic with absorbing SATs on every face except the free
    surface: the discrete adjoint covers elastic blocks without PML."""
    rng = np.random.default_rng(seed)
    Ly, Lz, Lx = h * (nr - 1), h * (ns - 1), h * (nq - 1)
    y = np.linspace(0.0, Ly, nr)
    z = np.linspace(0.0, Lz, ns)
    Y, Z = np.meshgrid(y, z, indexing="xy")
    topo = 0.3 * np.exp(-((Y - 0.5 * Ly) ** 2 + (Z - 0.5 * Lz) ** 2) / (2.0 * (0.25 * Ly) ** 2))
    q = np.linspace(0.0, 1.0, nq)
    X = np.empty((3, ns, nr, nq))
    top = -topo[:, :, None]
    X[0] = top + (Lx - top) * q[None, None, :]
    X[1] = Y[:, :, None]
    X[2] = Z[:, :, None]
    depth = X[0] - X[0][:, :, :1]
    vs = 2.0 + 1.5 * np.clip(depth / Lx, 0.0, 1.0)
    if anomaly:
        r2 = (depth - 4.0) ** 2 + (X[1] - 0.5 * Ly) ** 2 + (X[2] - 0.5 * Lz) ** 2
        vs = vs * (1.0 + 0.03 * np.exp(-r2 / (1.5 ** 2)))
    vp = math.sqrt(3.0) * vs
    rho = 1.7 + 0.2 * vp
    mat = np.stack([rho * (vp ** 2 - 2 * vs ** 2), rho * vs ** 2, rho])
    strike, dip, rake = rng.uniform(0, 2 * math.pi), rng.uniform(0.2, 1.4), rng.uniform(-math.pi, math.pi)
    ns_ = np.array([-math.sin(dip) * math.sin(strike), math.sin(dip) * math.cos(strike), -math.cos(dip)])
    ds_ = np.array([math.cos(rake) * math.cos(strike) + math.sin(rake) * math.cos(dip) * math.sin(strike),
                    math.cos(rake) * math.sin(strike) - math.sin(rake) * math.cos(dip) * math.cos(strike),
                    -math.sin(rake) * math.sin(dip)])
    M = np.outer(ns_, ds_) + np.outer(ds_, ns_)
    src = Source("ricker", duration=3.0, t_init=1.2 / 3.0, mxx=M[0, 0], myy=M[1, 1], mzz=M[2, 2], mxy=M[0, 1],
                 mxz=M[0, 2], myz=M[1, 2], x=2.0, y=0.4 * Ly, z=0.6 * Lz)
    ys = np.linspace(0.05 * Ly, 0.95 * Ly, nrec)
    zs = np.linspace(0.05 * Lz, 0.95 * Lz, nrec)
    rec = np.array([[0.0, yy, zz] for zz in zs for yy in ys])
    b = Block(nqrs=(nq, nr, ns), aqrs=(0.0, 0.0, 0.0), bqrs=(Lx, Ly, Lz), rho_s_p=(2.7, 3.5, 6.06),
              lqrs=(2, 1, 1), rqrs=(1, 1, 1), coords=X, material=mat, sources=[src], receivers=rec)
    p = Problem(blocks=[b], response="elastic", type_of_mesh="curvilinear", CFL=0.5, source_order=4, w_stride=1)
    p.t_final = steps * p.dt() * (1.0 + 1e-9)
    return p
