"""Batched independent shots on one device.

Each shot is its own one-block problem with its own domain and CUDA stream;
:class:`ShotBatch` replays every shot's captured step graph in turn, in
chunks, so the shots' kernels run concurrently on the GPU.  Nothing is
exchanged between shots (across GPUs the batch splits into replicas).

:func:`random_shots` builds the batched-shot workload: Cartesian blocks of
seeded sizes between ``nmin`` and ``nmax`` points per axis, each with its own
seeded layered medium (Vs 1.5 -> 3.5 km/s, Vp = sqrt(3) Vs, rho = 1.7 + 0.2
Vp), elastic or Q4 (Qs = 50 Vs, Qp = 2 Qs), a seeded moment-tensor source
(position and mechanism) with a Ricker wavelet of 1-4 Hz, a free surface on
top, absorbing faces elsewhere and a line of surface stations.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

import numpy as np

from .problem import AnelasticParams, Block, Problem, Source


def random_shot(seed: int, nmin: int = 64, nmax: int = 192, h: float = 0.1, steps: int = 800,
                response: Optional[str] = None, nrec: int = 10) -> Problem:
    rng = np.random.default_rng(seed)
    nq, nr, ns = (int(rng.integers(nmin, nmax + 1)) for _ in range(3))
    if response is None:
        response = "elastic" if rng.random() < 0.5 else "anelastic-Q4"
    Lq, Lr, Ls = h * (nq - 1), h * (nr - 1), h * (ns - 1)
    # layered medium along depth q: a few seeded layers between 1.5 and 3.5 km/s
    nl = int(rng.integers(2, 6))
    tops = np.sort(rng.uniform(0.0, Lq, nl - 1))
    vsl = np.sort(rng.uniform(1.5, 3.5, nl))
    depth = np.arange(nq) * h
    vs_q = vsl[np.searchsorted(tops, depth)]
    vs = np.broadcast_to(vs_q[None, None, :], (ns, nr, nq)).copy()
    vp = math.sqrt(3.0) * vs
    rho = 1.7 + 0.2 * vp
    mat = np.stack([rho * (vp ** 2 - 2 * vs ** 2), rho * vs ** 2, rho])
    strike, dip, rake = rng.uniform(0, 2 * math.pi), rng.uniform(0.2, 1.4), rng.uniform(-math.pi, math.pi)
    nv = np.array([-math.sin(dip) * math.sin(strike), math.sin(dip) * math.cos(strike), -math.cos(dip)])
    dv = np.array([math.cos(rake) * math.cos(strike) + math.sin(rake) * math.cos(dip) * math.sin(strike),
                   math.cos(rake) * math.sin(strike) - math.sin(rake) * math.cos(dip) * math.cos(strike),
                   -math.sin(rake) * math.sin(dip)])
    M = np.outer(nv, dv) + np.outer(dv, nv)
    f0 = float(rng.uniform(1.0, 4.0))
    pos = [rng.uniform(0.3, 0.7) * L for L in (Lq, Lr, Ls)]
    src = Source("ricker", duration=f0, t_init=1.2 / f0, mxx=M[0, 0], myy=M[1, 1], mzz=M[2, 2], mxy=M[0, 1],
                 mxz=M[0, 2], myz=M[1, 2], x=pos[0], y=pos[1], z=pos[2])
    ys = np.linspace(0.1 * Lr, 0.9 * Lr, nrec)
    rec = np.array([[0.0, y, 0.5 * Ls] for y in ys])
    kw = {}
    if response == "anelastic-Q4":
        qs = 1.0 / (50.0 * vs)
        kw = {"qs_inv": qs, "qp_inv": 0.5 * qs}
    b = Block(nqrs=(nq, nr, ns), aqrs=(0.0, 0.0, 0.0), bqrs=(Lq, Lr, Ls), rho_s_p=(1.7 + 0.2 * math.sqrt(3.0) * 3.5,
              3.5, math.sqrt(3.0) * 3.5), lqrs=(2, 1, 1), rqrs=(1, 1, 1), material=mat, sources=[src],
              receivers=rec, **kw)
    an = AnelasticParams(Qs0=100.0, Qp0=200.0, fref=1.0, fmin=0.05, fmax=20.0)
    p = Problem(blocks=[b], response=response, type_of_mesh="cartesian", CFL=0.5, source_order=4, anelastic=an,
                w_stride=1)
    p.t_final = steps * p.dt() * (1.0 + 1e-9)
    return p


def random_shots(n: int = 48, seed: int = 7, nmin: int = 64, nmax: int = 192, h: float = 0.1,
                 steps: int = 800) -> List[Problem]:
    """The batched-shot workload: n seeded shots (see :func:`random_shot`)."""
    return [random_shot(seed * 1000 + i, nmin=nmin, nmax=nmax, h=h, steps=steps) for i in range(n)]


class ShotBatch:
    """Independent shots on one device.

    mode 'batched' (default): one launch per kernel kind and RK stage for
    every shot (``wql3d_batch_*``: shot x tile work lists, the step pair in one
    CUDA graph, interior tiles autotuned over the first steps).  mode
    'streams': each shot a domain on its own stream, its step graph replayed
    round-robin.  The shots share one time step (same spacing and rho_s_p, as
    :func:`random_shots` builds them)."""

    def __init__(self, problems: Sequence[Problem], precision: str = "fp64", nsteps_hint: Optional[int] = None,
                 mode: str = "batched"):
        import ctypes as C
        from . import _lib
        from .domain import Domain
        self.domains = [Domain(p, precision=precision, nsteps_hint=nsteps_hint) for p in problems]
        self.mode = mode
        self.batch = None
        self.dt = problems[0].dt()
        self.w_stride = problems[0].w_stride
        if any(abs(p.dt() - self.dt) > 1e-15 * self.dt for p in problems):
            raise ValueError("the shots of a batch share one time step")
        if mode == "batched":
            arr = (C.c_void_p * len(self.domains))(*[d.handle.value for d in self.domains])
            h = C.c_void_p()
            _lib.check(_lib.load().wql3d_batch_create(arr, len(self.domains), C.byref(h)), "wql3d_batch_create")
            self.batch = h

    @property
    def npoints(self) -> int:
        return sum(b.npoints for d in self.domains for b in d.blocks)

    def run(self, nsteps: int, chunk: int = 2):
        """nsteps on every shot.  Batched: one call; streams: each shot's step
        graph replayed ``chunk`` steps at a time, round-robin over the shots,
        so that all streams have work queued at once."""
        from . import _lib
        if self.batch is not None:
            _lib.check(_lib.load().wql3d_batch_run(self.batch, float(self.dt), int(nsteps), int(self.w_stride)),
                       "wql3d_batch_run")
            for d in self.domains:
                d.n += nsteps
            return
        done = 0
        while done < nsteps:
            k = min(chunk, nsteps - done)
            for d in self.domains:
                d.run(k)
            done += k

    def tuning(self):
        """(chosen z-chunk, [(candidate, ms per step), ...]) of the batch's tile autotuner."""
        import ctypes as C
        from . import _lib
        z, n = C.c_int32(), C.c_int32()
        zs = (C.c_int32 * 16)()
        ms = (C.c_float * 16)()
        _lib.check(_lib.load().wql3d_batch_tuning(self.batch, C.byref(z), C.byref(n), zs, ms), "wql3d_batch_tuning")
        return z.value, [(zs[i], ms[i]) for i in range(n.value)]

    def kernel_launches(self) -> int:
        import ctypes as C
        from . import _lib
        if self.batch is None:
            return sum(d.kernel_launches() for d in self.domains)
        v = C.c_int64()
        _lib.check(_lib.load().wql3d_batch_launches(self.batch, C.byref(v)), "wql3d_batch_launches")
        return v.value

    def synchronize(self):
        from . import _lib
        if self.batch is not None:
            _lib.check(_lib.load().wql3d_batch_synchronize(self.batch), "wql3d_batch_synchronize")
        for d in self.domains:
            d.synchronize()

    def seismograms(self) -> List[np.ndarray]:
        return [d.seismograms(0) for d in self.domains]

    def close(self):
        from . import _lib
        if self.batch is not None:
            _lib.load().wql3d_batch_destroy(self.batch)
            self.batch = None
        for d in self.domains:
            d.close()
        self.domains = []
