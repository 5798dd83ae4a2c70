"""Waveform-misfit gradients through the discrete adjoint of the CUDA stage.

The reference has no adjoint.  This module differentiates the misfit

    chi = 1/2 sum_n sum_r |v_r(t_n) - d_r(t_n)|^2

of the stage-1 station samples (src/time_step.f90:137) of an N-step run
from rest with respect to the material lambda, mu, rho of every point and
the moment tensors of the sources, for one FP64 elastic block without PML
(traditional-6 operator, face SATs, moment-tensor sources).  The adjoint
kernels are the transposes of the stage operator, the sources and the
Kennedy-Carpenter (5,4) low-storage update (``wql3d_adjoint_*`` in
include/wql3d.h).

Memory: sqrt(N)-step checkpointing with recomputation.  The forward run
stores the fields every K steps on the device; the reverse sweep restores
each checkpoint, recomputes its K steps once while recording every step's
five stage inputs and, for a curvilinear block, their derivative terms
(written by the stage kernel as it computes them) into a device segment
buffer (``wql3d_record_step``), and reverses those steps from the records
(``wql3d_adjoint_step_recorded``), so that the adjoint pass does not re-derive
the stage inputs for the material gradient.  Device storage is ceil(N/K) + 10 K
field states (K = ceil(sqrt(N / 10)) by default, the minimum) instead of 10 N;
the forward work is done twice.  With ``record_stages=False`` the segment
holds one state per step and every adjoint step recomputes its four inner
stages (ceil(N/K) + K states, K = ceil(sqrt(N)), the forward work done
almost three times).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from .domain import Domain, _ptr
from .problem import Problem


class AdjointSolver:
    """Forward runs and adjoint sweeps of one elastic block on the current CUDA device."""

    def __init__(self, problem: Problem, nsteps: int, checkpoint_every: Optional[int] = None,
                 record_stages: bool = True):
        if len(problem.blocks) != 1 or problem.response != "elastic":
            raise ValueError("the adjoint covers one elastic block")
        self.problem = problem
        self.nsteps = int(nsteps)
        # storage is ceil(N / K) checkpoints + K recorded steps of `per` field
        # volumes each: K = sqrt(N / per) minimises it (every step is still
        # recomputed exactly once in the reverse sweep, whatever K)
        per = _lib.RECORD_FIELDS if record_stages else 1
        self.K = (int(checkpoint_every) if checkpoint_every
                  else max(1, math.ceil(math.sqrt(self.nsteps / per))))
        self.dt = problem.dt()
        self.domain = Domain(problem, precision="fp64", max_samples=self.nsteps + 2)
        L = _lib.load()
        self.L = L
        self.h = self.domain.handle
        _lib.check(L.wql3d_adjoint_enable(self.h), "wql3d_adjoint_enable")
        ne = C.c_int64()
        _lib.check(L.wql3d_field_volume(self.h, 0, C.byref(ne)), "wql3d_field_volume")
        self.nchk = math.ceil(self.nsteps / self.K)
        self.ckpt = torch.empty((self.nchk, ne.value), dtype=torch.float64, device="cuda")
        self.record = bool(record_stages)
        self.ne = ne.value
        self.seg = torch.empty((self.K, per * ne.value), dtype=torch.float64, device="cuda")
        blk = problem.blocks[0]
        self.nrec = 0 if blk.receivers is None else len(blk.receivers)
        self.nsrc = len(blk.sources)
        self.shape = tuple(reversed(blk.nqrs))

    # ------------------------------------------------------------ parameters
    def set_parameters(self, material: Optional[np.ndarray] = None, moment: Optional[np.ndarray] = None):
        """material (3, ns, nr, nq) lambda, mu, rho; moment (nsrc, 6) mxx myy mzz mxy mxz myz."""
        if material is not None:
            m = np.ascontiguousarray(material, dtype=np.float64)
            _lib.check(self.L.wql3d_set_material(self.h, 0, _ptr(m)), "wql3d_set_material")
        if moment is not None and self.nsrc:
            m6 = np.ascontiguousarray(moment, dtype=np.float64).reshape(self.nsrc, 6)
            _lib.check(self.L.wql3d_set_moment(self.h, 0, _ptr(m6)), "wql3d_set_moment")

    def _ptr(self, t: torch.Tensor):
        return C.c_void_p(t.data_ptr())

    # ---------------------------------------------------------------- forward
    def forward(self) -> np.ndarray:
        """N steps from rest with checkpoints; returns the station velocities (N, nrec, 3)."""
        d = self.domain
        d.set_fields(np.zeros((9,) + self.shape))
        d.t = 0.0
        d.n = 1
        _lib.check(self.L.wql3d_reset_samples(self.h), "wql3d_reset_samples")
        for k in range(self.nchk):
            _lib.check(self.L.wql3d_store_fields(self.h, 0, self._ptr(self.ckpt[k])), "wql3d_store_fields")
            steps = min(self.K, self.nsteps - k * self.K)
            d.run(steps)
        seis = d.seismograms()[:self.nsteps, :, 1:4]
        return np.ascontiguousarray(seis)

    # --------------------------------------------------------------- backward
    def backward(self, residual: np.ndarray):
        """Reverse sweep for the misfit derivative residual (N, nrec, 3) with
        respect to the station samples; returns (d/d(lambda, mu, rho) as
        (3, ns, nr, nq), d/dM as (nsrc, 6))."""
        d, L, h = self.domain, self.L, self.h
        res = np.ascontiguousarray(residual, dtype=np.float64)
        _lib.check(L.wql3d_adjoint_reset(h), "wql3d_adjoint_reset")
        for k in range(self.nchk - 1, -1, -1):
            first = k * self.K
            steps = min(self.K, self.nsteps - first)
            # recompute the segment's states F_n, n = first .. first + steps - 1 (0-based)
            _lib.check(L.wql3d_load_fields(h, 0, self._ptr(self.ckpt[k])), "wql3d_load_fields")
            d.t = first * self.dt
            for j in range(steps):
                if self.record:
                    _lib.check(L.wql3d_record_step(h, float(self.dt), first + j + 1, int(self.problem.w_stride),
                                                   self._ptr(self.seg[j])), "wql3d_record_step")
                    continue
                _lib.check(L.wql3d_store_fields(h, 0, self._ptr(self.seg[j])), "wql3d_store_fields")
                if j + 1 < steps:
                    d.time_step_RK(first + j + 1)
            for j in range(steps - 1, -1, -1):
                n = first + j
                if self.record:
                    _lib.check(L.wql3d_adjoint_step_recorded(h, n + 1, float(self.dt), n * self.dt,
                                                             self._ptr(self.seg[j])), "wql3d_adjoint_step_recorded")
                else:
                    _lib.check(L.wql3d_load_fields(h, 0, self._ptr(self.seg[j])), "wql3d_load_fields")
                    d.t = n * self.dt
                    _lib.check(L.wql3d_adjoint_step(h, n + 1, float(self.dt)), "wql3d_adjoint_step")
                if self.nrec:
                    r = np.ascontiguousarray(res[n])
                    _lib.check(L.wql3d_adjoint_add_receivers(h, 0, _ptr(r)), "wql3d_adjoint_add_receivers")
        gmat = np.zeros((3,) + self.shape)
        gM = np.zeros((max(self.nsrc, 1), 6))
        _lib.check(L.wql3d_get_adjoint_gradient(h, 0, _ptr(gmat), _ptr(gM)), "wql3d_get_adjoint_gradient")
        return gmat, gM[:self.nsrc]

    def adjoint_fields(self) -> np.ndarray:
        a = np.zeros((9,) + self.shape)
        _lib.check(self.L.wql3d_get_adjoint_fields(self.h, 0, _ptr(a)), "wql3d_get_adjoint_fields")
        return a

    def close(self):
        self.domain.close()


class WaveformMisfit(torch.autograd.Function):
    """chi(material, moment) = 1/2 ||v(material, moment) - observed||^2 with the
    gradient from the discrete adjoint (one forward run with checkpoints in
    forward(), the recomputing reverse sweep in backward())."""

    @staticmethod
    def forward(ctx, material: torch.Tensor, moment: torch.Tensor, solver: AdjointSolver, observed: np.ndarray):
        solver.set_parameters(material.detach().cpu().numpy(), moment.detach().cpu().numpy())
        seis = solver.forward()
        res = seis - observed
        ctx.solver = solver
        ctx.res = res
        ctx.dev = material.device
        return torch.tensor(0.5 * float(np.sum(res * res)), dtype=torch.float64, device=material.device)

    @staticmethod
    def backward(ctx, gout):
        gmat, gM = ctx.solver.backward(ctx.res)
        g = float(gout)
        return (torch.from_numpy(g * gmat).to(ctx.dev), torch.from_numpy(g * gM).to(ctx.dev), None, None)


def waveform_misfit(material: torch.Tensor, moment: torch.Tensor, solver: AdjointSolver,
                    observed: np.ndarray) -> torch.Tensor:
    return WaveformMisfit.apply(material, moment, solver, observed)


def _solve_shot(problem: Problem, observed: np.ndarray, material: np.ndarray, checkpoint_every=None):
    """chi, d chi / d(lambda, mu, rho), d chi / dM of one shot on this GPU."""
    sol = AdjointSolver(problem, observed.shape[0], checkpoint_every)
    try:
        sol.set_parameters(material=material)
        seis = sol.forward()
        res = seis - observed
        gmat, gM = sol.backward(res)
        return 0.5 * float(np.sum(res * res)), gmat, gM
    finally:
        sol.close()


def gradient_over_shots(shots: Sequence, material: np.ndarray, *, group=None, solve=None):
    """Misfit and gradients summed over the shots of a gradient
    configuration, the shots dealt round-robin to the ranks of a
    torch.distributed process group (one GPU each): rank r solves shots r,
    r + W, ...; then one all-reduce (SUM) over the group of [chi, the material
    gradient field, the stacked per-shot moment-tensor gradients] (NCCL on
    device buffers, or gloo on host buffers).  shots: (problem, observed)
    pairs, observed (N, nrec, 3); material (3, ns, nr, nq).  Returns (chi,
    gradient (3, ns, nr, nq), [per-shot (nsrc, 6)]), the same on every rank.
    solve(problem, observed, material) -> (chi, gmat, gM) stands in for the
    per-shot forward + adjoint (tests on hosts without a GPU)."""
    solve = solve or _solve_shot
    try:
        import torch.distributed as dist
        dist_on = dist.is_available() and dist.is_initialized()
    except ImportError:
        dist_on = False
    rank = dist.get_rank(group) if dist_on else 0
    world = dist.get_world_size(group) if dist_on else 1
    nsrc = [len(p.blocks[0].sources) for p, _ in shots]
    offs = np.concatenate([[0], np.cumsum([6 * k for k in nsrc])]).astype(int)
    nmat = int(np.prod(material.shape))
    flat = np.zeros(1 + nmat + int(offs[-1]))
    for i, (p, obs) in enumerate(shots):
        if i % world != rank:
            continue
        chi, gmat, gM = solve(p, obs, material)
        flat[0] += chi
        flat[1:1 + nmat] += np.asarray(gmat, dtype=np.float64).ravel()
        flat[1 + nmat + offs[i]:1 + nmat + offs[i + 1]] = np.asarray(gM, dtype=np.float64).ravel()
    if world > 1:
        backend = dist.get_backend(group)
        t = torch.from_numpy(flat)
        if backend == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        flat = t.cpu().numpy()
    gms = [flat[1 + nmat + offs[i]:1 + nmat + offs[i + 1]].reshape(nsrc[i], 6) for i in range(len(shots))]
    return float(flat[0]), flat[1:1 + nmat].reshape(material.shape), gms
