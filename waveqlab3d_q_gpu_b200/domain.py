"""Host-side domain: the reference's domain / time_step interface on the GPU.

Mirrors the Fortran driver's public operations (paths relative to the
reference project root):

=====================================  ===========================================
reference                               this module
=====================================  ===========================================
``init_domain`` domain.f90:30-330       :class:`Domain` (``Domain(problem)``)
``init_RK`` time_step.f90:20-65         :func:`init_RK`
``time_step_RK`` time_step.f90:68-150   :meth:`Domain.time_step_RK`
``scale_rates`` domain.f90:922-949      :meth:`Domain.scale_rates`
``set_rates`` domain.f90:951-979        :meth:`Domain.set_rates`
``enforce_bound_iface_conditions``      :meth:`Domain.enforce_bound_iface_conditions`
``update_fields`` domain.f90:982-1017   :meth:`Domain.update_fields`
``exchange_fields`` domain.f90:682-694  :meth:`Domain.exchange_fields` (one GPU: no-op)
``close_domain`` domain.f90:505-613     :meth:`Domain.close_domain`
=====================================  ===========================================

All numerical work runs in libwql3d.so (sm_100a); this module only prepares
setup-time arrays (material with the anelastic modulus correction, source
and receiver tables) and moves data across the C ABI.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

from . import _lib
from .problem import COUPLINGS, FAULT_PROBLEMS, RESPONSES, RK_A, RK_B, RK_C, STF_CODES, Problem


@dataclass
class RK:
    """Low-storage RK coefficients (RK_type, time_step.f90:12-17)."""

    nstage: int
    A: Tuple[float, ...]
    B: Tuple[float, ...]
    C: Tuple[float, ...]


def init_RK() -> RK:
    """Kennedy-Carpenter (5,4), the reference's hard-coded order 4 (time_step.f90:20-65)."""
    return RK(5, RK_A, RK_B, RK_C)


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_lib.dp)


class Domain:
    """One or two blocks resident on the current CUDA device."""

    def __init__(self, problem: Problem, precision: str = "fp64", max_samples: Optional[int] = None,
                 nsteps_hint: Optional[int] = None, remote_block: Optional[int] = None, slab=None):
        """``remote_block`` = r holds only block r of a two-block problem; the
        other block lives in another process and the interface face is
        exchanged every stage (see :mod:`waveqlab3d_q_gpu_b200.distributed`).
        ``slab`` (a :class:`waveqlab3d_q_gpu_b200.slabs.SlabPart`) makes this
        domain one s-slab of a larger block whose ghost planes are exchanged
        every stage (see :mod:`waveqlab3d_q_gpu_b200.slabs`)."""
        from . import anelastic as an

        L = _lib.load()
        self.problem = problem
        self.precision = precision
        self._keep: List[np.ndarray] = []
        if remote_block is not None:
            if len(problem.blocks) != 2 or remote_block not in (0, 1):
                raise ValueError("remote_block needs a two-block problem and r in (0, 1)")
            self.blocks = [problem.blocks[remote_block]]
        else:
            self.blocks = list(problem.blocks)
        self.remote_block = remote_block
        nb = len(self.blocks)
        if nb not in (1, 2):
            raise ValueError("one or two blocks")
        d = _lib.DomainDesc()
        d.abi_version = _lib.ABI_VERSION
        d.nblocks = nb
        d.remote_side = 0 if remote_block is None else remote_block + 1
        d.precision = 0 if precision == "fp64" else 1
        d.response = RESPONSES[problem.response]
        d.coarse_grain = 1 if (problem.response == "anelastic-fQ8" and problem.anelastic.coarse_grain == 2) else 0
        d.Qs0 = problem.anelastic.Qs0
        d.Qp0 = problem.anelastic.Qp0
        if problem.response != "elastic":
            tau, c1, c2 = an.coefficients(problem.response, problem.anelastic)
            for k in range(len(tau)):
                d.tau[k] = float(tau[k])
                if problem.response == "anelastic-fQ8":
                    d.strength_s[k] = float(c1[k])
                    d.strength_p[k] = float(c2[k])
                else:
                    d.weight[k] = float(c1[k])
        ip = problem.interface
        d.coupling = COUPLINGS[ip.coupling]
        d.serial_shared = 1 if ip.serial_shared else 0
        d.fault_problem = FAULT_PROBLEMS[ip.problem]
        d.fs, d.fd, d.Dc = ip.fs, ip.fd, ip.Dc
        if ip.stress is not None:
            d.fault_stress[:] = [float(v) for v in ip.stress]
        if nb == 2 or remote_block is not None:
            nq, nr, ns = problem.blocks[0].nqrs
            if ip.tau0_n is not None or ip.tau0_m is not None or ip.tau0_l is not None:
                t0 = np.zeros((3, ns, nr))
                for k, a in enumerate((ip.tau0_n, ip.tau0_m, ip.tau0_l)):
                    if a is not None:
                        t0[k] = a
                self._keep.append(t0)
                d.iface_tau0 = _ptr(t0)
            if ip.fs_map is not None:
                fm = np.ascontiguousarray(ip.fs_map, dtype=np.float64)
                self._keep.append(fm)
                d.iface_fs = _ptr(fm)
        if max_samples is None:
            nt = nsteps_hint if nsteps_hint is not None else problem.nt()
            max_samples = max(1, (nt + max(problem.w_stride, 1) - 1) // max(problem.w_stride, 1) + 1)
        d.max_samples = int(max_samples)
        self.slab = slab
        if slab is not None:
            d.slab_z0 = int(slab.z0)
            d.slab_ns_global = int(slab.ns_global)
            if slab.ghost_coords is not None:
                gc = np.ascontiguousarray(slab.ghost_coords, dtype=np.float64)
                self._keep.append(gc)
                d.slab_ghost_coords = _ptr(gc)
        if problem.mms is not None:
            d.mms = 1
            d.mms_nt, d.mms_nx, d.mms_ny, d.mms_nz = problem.mms.nt, problem.mms.nx, problem.mms.ny, problem.mms.nz
        for i, b in enumerate(self.blocks):
            bd = d.block[i]
            bd.nq, bd.nr, bd.ns = b.nqrs
            bd.mesh = 1 if problem.type_of_mesh == "curvilinear" else 0
            bd.f32_literal = 1 if problem.closure_f32_literal else 0
            for k, v in enumerate(b.bc()):
                bd.bc[k] = int(v)
            for k, v in enumerate(b.pml()):
                bd.pml[k] = int(v)
            bd.npml = int(b.npml)
            for k in range(3):
                bd.aqrs[k], bd.bqrs[k] = b.aqrs[k], b.bqrs[k]
            bd.tau0 = problem.sat_penalty()
            bd.fd_operator = problem.fd_operator()
            bd.host_nb = 0
            if problem.type_of_mesh == "curvilinear":
                if b.coords is None:
                    raise ValueError("curvilinear blocks need coordinates")
                xyz = np.ascontiguousarray(b.coords, dtype=np.float64)
                self._keep.append(xyz)
                bd.coords = _ptr(xyz)
            mat = np.ascontiguousarray(an.corrected_material(problem, b), dtype=np.float64)
            self._keep.append(mat)
            bd.material = _ptr(mat)
            if problem.response in ("anelastic-Q4", "anelastic-Q8"):
                qs, qp = an.q_inverse(problem, b)
                self._keep += [qs, qp]
                bd.qs_inv, bd.qp_inv = _ptr(qs), _ptr(qp)
            bd.nsrc = len(b.sources)
            bd.src_order = problem.source_order
            bd.src_alpha = problem.source_alpha
            if b.sources:
                st = np.array([STF_CODES[s.stf] for s in b.sources], dtype=np.int32)
                sp = np.array([s.params() for s in b.sources], dtype=np.float64).ravel()
                self._keep += [st, sp]
                bd.src_type = st.ctypes.data_as(_lib.ip)
                bd.src_par = _ptr(sp)
            if b.receivers is not None and len(b.receivers):
                rx = np.ascontiguousarray(b.receivers, dtype=np.float64).ravel()
                self._keep.append(rx)
                bd.nrec = len(b.receivers)
                bd.rec_xyz = _ptr(rx)
        h = C.c_void_p()
        _lib.check(L.wql3d_domain_create(C.byref(d), C.byref(h)), "wql3d_domain_create")
        self.handle = h
        self.nblocks = nb
        self.dt = problem.dt() if slab is None else slab.dt
        self.RK = init_RK()
        self.n = 1

    # ------------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "handle", None):
            _lib.load().wql3d_domain_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ time
    @property
    def t(self) -> float:
        v = C.c_double()
        _lib.check(_lib.load().wql3d_get_time(self.handle, C.byref(v)), "wql3d_get_time")
        return v.value

    @t.setter
    def t(self, value: float):
        _lib.check(_lib.load().wql3d_set_time(self.handle, float(value)), "wql3d_set_time")

    def time_step_RK(self, n: Optional[int] = None, dt: Optional[float] = None):
        """Advance one time step with the 5-stage low-storage RK (time_step.f90:68-150)."""
        n = self.n if n is None else n
        dt = self.dt if dt is None else dt
        _lib.check(_lib.load().wql3d_time_step(self.handle, float(dt), int(n), int(self.problem.w_stride)),
                   "wql3d_time_step")
        self.n = n + 1

    def stage(self, stage: int, dt: Optional[float] = None):
        """One RK stage of the whole domain (time_step.f90:109-147 loop body)."""
        dt = self.dt if dt is None else dt
        _lib.check(_lib.load().wql3d_stage(self.handle, int(stage), float(dt)), "wql3d_stage")

    def run(self, nsteps: int, dt: Optional[float] = None):
        """Advance ``nsteps`` steps through the graph-captured step loop."""
        dt = self.dt if dt is None else dt
        _lib.check(_lib.load().wql3d_run(self.handle, float(dt), int(self.n), int(nsteps),
                                         int(self.problem.w_stride)), "wql3d_run")
        self.n += nsteps

    # split stage operations (domain.f90)
    def exchange_fields(self):
        """Halo exchange between ranks; a single-GPU domain has none."""

    def scale_rates(self, A: float):
        _lib.check(_lib.load().wql3d_scale_rates(self.handle, float(A)), "wql3d_scale_rates")

    def set_rates(self):
        _lib.check(_lib.load().wql3d_set_rates_rhs(self.handle), "wql3d_set_rates_rhs")

    def enforce_bound_iface_conditions(self, stage: int = 1):
        _lib.check(_lib.load().wql3d_enforce_bound_iface_conditions(self.handle, int(stage)),
                   "wql3d_enforce_bound_iface_conditions")

    def update_fields(self, dt: float):
        _lib.check(_lib.load().wql3d_update_fields(self.handle, float(dt)), "wql3d_update_fields")

    def check_status(self) -> int:
        """Waits for the queued work; raises Wql3dError (ENONFINITE) when a station
        sample so far was not finite (src/seismogram.f90:516-524), or (ECUDA)
        when a bounded device wait of a stage kernel gave up."""
        bad = C.c_int32()
        _lib.check(_lib.load().wql3d_check_status(self.handle, C.byref(bad)), "wql3d_check_status")
        return bad.value

    def synchronize(self):
        _lib.check(_lib.load().wql3d_synchronize(self.handle), "wql3d_synchronize")

    # ------------------------------------------------------------------ data
    def _shape(self, b: int, ncomp: int, host_nb: int = 0):
        nq, nr, ns = self.blocks[b].nqrs
        return (ncomp, ns + 2 * host_nb, nr + 2 * host_nb, nq + 2 * host_nb)

    def fields(self, b: int = 0, host_nb: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        a = np.zeros(self._shape(b, 9, host_nb)) if out is None else out
        _lib.check(_lib.load().wql3d_get_fields(self.handle, b, _ptr(a), host_nb), "wql3d_get_fields")
        return a

    def set_fields(self, F: np.ndarray, b: int = 0, host_nb: int = 0):
        a = np.ascontiguousarray(F, dtype=np.float64)
        _lib.check(_lib.load().wql3d_set_fields(self.handle, b, _ptr(a), host_nb), "wql3d_set_fields")

    def rates(self, b: int = 0, host_nb: int = 0) -> np.ndarray:
        a = np.zeros(self._shape(b, 9, host_nb))
        _lib.check(_lib.load().wql3d_get_rates(self.handle, b, _ptr(a), host_nb), "wql3d_get_rates")
        return a

    def set_rates_array(self, DF: np.ndarray, b: int = 0, host_nb: int = 0):
        a = np.ascontiguousarray(DF, dtype=np.float64)
        _lib.check(_lib.load().wql3d_set_rates(self.handle, b, _ptr(a), host_nb), "wql3d_set_rates")

    def eta(self, b: int = 0) -> np.ndarray:
        nm = self.problem.nmech
        nq, nr, ns = self.blocks[b].nqrs
        a = np.zeros((6, nm, ns, nr, nq))
        _lib.check(_lib.load().wql3d_get_memory_variables(self.handle, b, _ptr(a)), "wql3d_get_memory_variables")
        return a

    def metrics(self, b: int = 0) -> np.ndarray:
        a = np.zeros(self._shape(b, 10))
        _lib.check(_lib.load().wql3d_get_metrics(self.handle, b, _ptr(a)), "wql3d_get_metrics")
        return a

    def interface(self) -> np.ndarray:
        nq, nr, ns = self.blocks[0].nqrs
        a = np.zeros((ns, nr, 7))
        _lib.check(_lib.load().wql3d_get_interface(self.handle, _ptr(a)), "wql3d_get_interface")
        return a

    # stage-by-stage driving and the remote interface side
    def begin_step(self, n: Optional[int] = None):
        """Step counter and stage-1 receiver sample (time_step.f90:137) before wql3d_stage calls."""
        n = self.n if n is None else n
        _lib.check(_lib.load().wql3d_begin_step(self.handle, int(n), int(self.problem.w_stride)), "wql3d_begin_step")

    def interface_buffers(self):
        """(send_ptr, recv_ptr, count, elem_bytes) of a remote interface side."""
        snd, rcv = C.c_void_p(), C.c_void_p()
        cnt, eb = C.c_int64(), C.c_int32()
        _lib.check(_lib.load().wql3d_interface_buffers(self.handle, C.byref(snd), C.byref(rcv), C.byref(cnt),
                                                       C.byref(eb)), "wql3d_interface_buffers")
        return snd.value, rcv.value, cnt.value, eb.value

    def pack_interface(self):
        _lib.check(_lib.load().wql3d_pack_interface(self.handle), "wql3d_pack_interface")

    # ghost planes of an s-slab domain (kind 0: fields, 1: metric)
    def halo_buffers(self, kind: int = 0):
        """(send_ptr, recv_ptr, count per face, elem_bytes) of the ghost-plane buffers."""
        snd, rcv = C.c_void_p(), C.c_void_p()
        cnt, eb = C.c_int64(), C.c_int32()
        _lib.check(_lib.load().wql3d_halo_buffers(self.handle, int(kind), C.byref(snd), C.byref(rcv), C.byref(cnt),
                                                  C.byref(eb)), "wql3d_halo_buffers")
        return snd.value, rcv.value, cnt.value, eb.value

    def pack_halo(self, kind: int = 0):
        _lib.check(_lib.load().wql3d_pack_halo(self.handle, int(kind)), "wql3d_pack_halo")

    def unpack_halo(self, kind: int = 0):
        _lib.check(_lib.load().wql3d_unpack_halo(self.handle, int(kind)), "wql3d_unpack_halo")

    def interface_material(self) -> np.ndarray:
        nq, nr, ns = self.blocks[0].nqrs
        a = np.zeros((3, ns, nr))
        _lib.check(_lib.load().wql3d_get_interface_material(self.handle, _ptr(a)), "wql3d_get_interface_material")
        return a

    def set_interface_remote_material(self, M: np.ndarray):
        a = np.ascontiguousarray(M, dtype=np.float64)
        _lib.check(_lib.load().wql3d_set_interface_remote_material(self.handle, _ptr(a)),
                   "wql3d_set_interface_remote_material")

    FAULT_KINDS = {"S": (0, 4), "Svel": (1, 3), "Uhat": (2, 6), "Vhat": (3, 6), "state": (4, 1), "trup": (5, 1)}

    def fault(self, name: str) -> np.ndarray:
        """One fault output (``S``, ``Svel``, ``Uhat``, ``Vhat``, ``state``, ``trup``) as
        (ncomp, ns, nr), the layout of the reference's ``_interface.*`` files
        (src/fault_output.f90:73-122); ``Uface`` / ``Vface`` come from :meth:`fields`."""
        kind, nc = self.FAULT_KINDS[name]
        nq, nr, ns = self.blocks[0].nqrs
        a = np.zeros((nc, ns, nr))
        _lib.check(_lib.load().wql3d_get_fault_output(self.handle, kind, _ptr(a)), "wql3d_get_fault_output")
        return a

    def plane(self, b: int, axis: int, index: int, c0: int = 0, ncomp: int = 9) -> np.ndarray:
        """Field components c0 .. c0 + ncomp - 1 of block b on the plane of
        1-based ``index`` normal to ``axis`` (1: q, 2: r, 3: s), gathered on
        the device (wql3d_get_plane): (ncomp, n2, n1), n1 the first in-plane
        axis (q, or r for axis 1)."""
        nq, nr, ns = self.blocks[b].nqrs
        n1 = nr if axis == 1 else nq
        n2 = nr if axis == 3 else ns
        a = np.zeros((ncomp, n2, n1))
        _lib.check(_lib.load().wql3d_get_plane(self.handle, b, int(axis), int(index), int(c0), int(ncomp), _ptr(a)),
                   "wql3d_get_plane")
        return a

    def seismograms(self, b: int = 0) -> np.ndarray:
        blk = self.blocks[b]
        nrec = 0 if blk.receivers is None else len(blk.receivers)
        ns = C.c_int32()
        _lib.check(_lib.load().wql3d_get_seismograms(self.handle, b, None, C.byref(ns)), "wql3d_get_seismograms")
        a = np.zeros((max(ns.value, 1), max(nrec, 1), 4))
        if ns.value and nrec:
            _lib.check(_lib.load().wql3d_get_seismograms(self.handle, b, _ptr(a), C.byref(ns)),
                       "wql3d_get_seismograms")
        return a[:ns.value, :nrec]

    def receiver_index(self, b: int = 0) -> np.ndarray:
        blk = self.blocks[b]
        n = 0 if blk.receivers is None else len(blk.receivers)
        a = np.zeros((max(n, 1), 3), dtype=np.int32)
        _lib.check(_lib.load().wql3d_receiver_index(self.handle, b, a.ctypes.data_as(_lib.ip)), "wql3d_receiver_index")
        return a[:n]

    def final_state(self):
        mf, me = C.c_double(), C.c_double()
        mb = (C.c_double * 2)()
        _lib.check(_lib.load().wql3d_final_state(self.handle, C.byref(mf), C.byref(me), mb), "wql3d_final_state")
        return mf.value, me.value, (mb[0], mb[1])

    def close_domain(self, verbose: bool = True):
        """Final-state diagnostics with the reference's 16-digit format (domain.f90:573-587)."""
        mf, me, mb = self.final_state()
        lines = []
        r = self.problem.response
        if r == "elastic":
            lines.append("Elastic final state: max|field|=%24.16E" % mf)
            if self.nblocks == 2:
                lines.append("Elastic block maxima: block1=%24.16E, block2=%24.16E" % mb)
        else:
            tag = {"anelastic-Q4": "Q4", "anelastic-Q8": "Q8", "anelastic-fQ8": "fQ8"}[r]
            lines.append("%s final state: max|field|=%24.16E, max|memory|=%24.16E" % (tag, mf, me))
        if verbose:
            for ln in lines:
                print(ln)
        return mf, me, mb

    def stream_handle(self) -> int:
        """The domain's cudaStream_t as an integer (for CUDA events / torch.cuda.ExternalStream)."""
        v = C.c_void_p()
        _lib.check(_lib.load().wql3d_get_stream(self.handle, C.byref(v)), "wql3d_get_stream")
        return int(v.value or 0)

    def device_bytes(self) -> int:
        v = C.c_int64()
        _lib.check(_lib.load().wql3d_device_bytes(self.handle, C.byref(v)), "wql3d_device_bytes")
        return v.value

    def kernel_launches(self) -> int:
        v = C.c_int64()
        _lib.check(_lib.load().wql3d_kernel_launches(self.handle, C.byref(v)), "wql3d_kernel_launches")
        return v.value
