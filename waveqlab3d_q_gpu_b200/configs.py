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
