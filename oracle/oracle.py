"""ctypes driver for the CPU oracle (test infrastructure only).

The oracle (``wql3d_oracle.c``) restates the reference solver's hot path in
plain C.  Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs
of bench.py use it, always as the checker.  Build it with ``oracle/build.sh``
(``__graft_entry__.build()`` calls that too).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class OrcDesc(C.Structure):
    _fields_ = [
        ("nq", C.c_int), ("nr", C.c_int), ("ns", C.c_int),
        ("mesh", C.c_int), ("f32lit", C.c_int),
        ("bc", C.c_int * 6), ("pml", C.c_int * 6), ("npml", C.c_int),
        ("response", C.c_int), ("coarse", C.c_int),
        ("aqrs", C.c_double * 3), ("bqrs", C.c_double * 3), ("rho_s_p", C.c_double * 3),
        ("coords", C.POINTER(C.c_double)), ("material", C.POINTER(C.c_double)),
        ("qsinv", C.POINTER(C.c_double)), ("qpinv", C.POINTER(C.c_double)),
        ("tau", C.c_double * 8), ("weight", C.c_double * 8), ("sstr", C.c_double * 8), ("pstr", C.c_double * 8),
        ("tau0", C.c_double),
        ("nsrc", C.c_int), ("src_order", C.c_int), ("src_alpha", C.c_int),
        ("src_type", C.POINTER(C.c_int)), ("src_par", C.POINTER(C.c_double)),
        ("nrec", C.c_int), ("rec_xyz", C.POINTER(C.c_double)),
        ("mms", C.c_int), ("mms_nt", C.c_double), ("mms_nx", C.c_double), ("mms_ny", C.c_double),
        ("mms_nz", C.c_double), ("fd", C.c_int),
    ]


class OrcIface(C.Structure):
    _fields_ = [
        ("coupling", C.c_int), ("double_ds", C.c_int), ("problem", C.c_int),
        ("fs", C.c_double), ("fd", C.c_double), ("Dc", C.c_double), ("alpha_lin", C.c_double),
        ("tau0_n", C.POINTER(C.c_double)), ("tau0_l", C.POINTER(C.c_double)),
        ("tau0_m", C.POINTER(C.c_double)), ("fs_map", C.POINTER(C.c_double)),
        ("s0", C.c_double * 6),
    ]


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libwql3d_oracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.c_int, C.POINTER(OrcDesc), C.POINTER(OrcIface)]
        L.orc_destroy.argtypes = [vp]
        L.orc_time.restype = C.c_double
        L.orc_time.argtypes = [vp]
        L.orc_set_time.argtypes = [vp, C.c_double]
        L.orc_run.restype = C.c_int
        L.orc_run.argtypes = [vp, C.c_double, C.c_int, C.c_int, dp, dp]
        L.orc_stage.argtypes = [vp, C.c_int, C.c_double]
        for name in ("orc_get_fields", "orc_set_fields", "orc_get_rates", "orc_set_rates", "orc_get_metrics",
                     "orc_get_material", "orc_set_eta"):
            getattr(L, name).argtypes = [vp, C.c_int, dp]
        L.orc_get_eta.restype = C.c_int
        L.orc_get_eta.argtypes = [vp, C.c_int, dp]
        L.orc_get_pml.argtypes = [vp, C.c_int, C.c_int, dp]
        L.orc_get_normals.argtypes = [vp, C.c_int, C.c_int, dp]
        L.orc_get_iface.argtypes = [vp, dp]
        L.orc_get_fault.argtypes = [vp, C.c_int, dp]
        L.orc_mms_exact.argtypes = [vp, C.c_int, C.c_double, dp]
        L.orc_receiver_index.argtypes = [vp, C.c_int, ip]
        L.orc_final_state.argtypes = [vp, dp, dp, dp]
        L.orc_q4_coefficients.argtypes = [C.c_double, C.c_double, dp, dp]
        L.orc_q8_coefficients.argtypes = [C.c_double, C.c_double, dp, dp]
        L.orc_modulus_correction.argtypes = [C.c_int, dp, dp, C.c_double, C.c_long, dp, dp, dp, dp, dp]
        L.orc_adjoint_rhs.restype = C.c_int
        L.orc_adjoint_rhs.argtypes = [vp, C.c_int, dp, dp, dp]
        L.orc_adjoint_moment.argtypes = [vp, C.c_int, C.c_double, dp, dp]
        L.orc_tfi_grid.argtypes = [dp, C.c_int, C.c_int, C.c_int, dp]
        L.orc_upwind_row.restype = C.c_int
        L.orc_upwind_row.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, ip, dp]
        _LIB = L
    return _LIB


def build() -> str:
    """Compile the oracle with gcc (no fused multiply-add, OpenMP over z)."""
    import subprocess
    src = os.path.join(_HERE, "wql3d_oracle.c")
    out = os.path.join(_HERE, "libwql3d_oracle.so")
    cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fopenmp", "-o", out, src, "-lm"]
    subprocess.check_call(cmd)
    return out


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleDomain:
    """One or two blocks advanced by the oracle's time_step_RK."""

    def __init__(self, problem, *, material_override=None, threads: Optional[int] = None):
        from waveqlab3d_q_gpu_b200.problem import COUPLINGS, FAULT_PROBLEMS, RESPONSES, STF_CODES
        from waveqlab3d_q_gpu_b200 import anelastic as an

        if threads is not None:
            os.environ["OMP_NUM_THREADS"] = str(threads)
        self.problem = problem
        self._keep: List[np.ndarray] = []
        nb = len(problem.blocks)
        descs = (OrcDesc * nb)()
        resp = RESPONSES[problem.response]
        tau = weight = sstr = pstr = None
        if resp:
            tau, c1, c2 = an.coefficients(problem.response, problem.anelastic)
            if problem.response == "anelastic-fQ8":
                sstr, pstr = c1, c2
            else:
                weight = c1
        for i, b in enumerate(problem.blocks):
            d = descs[i]
            d.nq, d.nr, d.ns = b.nqrs
            d.mesh = 1 if problem.type_of_mesh == "curvilinear" else 0
            d.f32lit = 1 if problem.closure_f32_literal else 0
            for k, v in enumerate(b.bc()):
                d.bc[k] = int(v)
            for k, v in enumerate(b.pml()):
                d.pml[k] = int(v)
            d.npml = int(b.npml)
            d.response = resp
            d.coarse = 1 if (problem.response == "anelastic-fQ8" and problem.anelastic.coarse_grain == 2) else 0
            for k in range(3):
                d.aqrs[k], d.bqrs[k], d.rho_s_p[k] = b.aqrs[k], b.bqrs[k], b.rho_s_p[k]
            if b.coords is not None:
                arr = np.ascontiguousarray(b.coords, dtype=np.float64)
                self._keep.append(arr)
                d.coords = _dptr(arr)
            mat = None
            if material_override is not None:
                mat = material_override[i]
            elif resp:
                mat = an.corrected_material(problem, b)
            elif b.material is not None:
                mat = b.material
            if mat is not None:
                arr = np.ascontiguousarray(mat, dtype=np.float64)
                self._keep.append(arr)
                d.material = _dptr(arr)
            if resp and problem.response != "anelastic-fQ8":
                qs, qp = an.q_inverse(problem, b)
                qs = np.ascontiguousarray(qs, dtype=np.float64)
                qp = np.ascontiguousarray(qp, dtype=np.float64)
                self._keep += [qs, qp]
                d.qsinv, d.qpinv = _dptr(qs), _dptr(qp)
            if tau is not None:
                for k, v in enumerate(tau):
                    d.tau[k] = v
            if weight is not None:
                for k, v in enumerate(weight):
                    d.weight[k] = v
            if sstr is not None:
                for k in range(len(sstr)):
                    d.sstr[k], d.pstr[k] = sstr[k], pstr[k]
            d.tau0 = problem.sat_penalty()
            d.fd = problem.fd_operator()
            if problem.mms is not None:
                d.mms = 1
                d.mms_nt, d.mms_nx, d.mms_ny, d.mms_nz = (problem.mms.nt, problem.mms.nx, problem.mms.ny,
                                                          problem.mms.nz)
            d.nsrc = len(b.sources)
            d.src_order = problem.source_order
            d.src_alpha = problem.source_alpha
            if b.sources:
                st = np.array([STF_CODES[s.stf] for s in b.sources], dtype=np.int32)
                sp = np.array([s.params() for s in b.sources], dtype=np.float64).ravel()
                self._keep += [st, sp]
                d.src_type = st.ctypes.data_as(C.POINTER(C.c_int))
                d.src_par = _dptr(sp)
            if b.receivers is not None and len(b.receivers):
                rx = np.ascontiguousarray(b.receivers, dtype=np.float64).ravel()
                self._keep.append(rx)
                d.nrec = len(b.receivers)
                d.rec_xyz = _dptr(rx)
        self._iface = None
        if nb == 2:
            ip = problem.interface
            I = OrcIface()
            I.coupling = COUPLINGS[ip.coupling]
            I.double_ds = 1 if ip.serial_shared else 0
            I.problem = FAULT_PROBLEMS[ip.problem]
            I.fs, I.fd, I.Dc = ip.fs, ip.fd, ip.Dc
            if ip.stress is not None:
                I.s0[:] = [float(v) for v in ip.stress]
            for name in ("tau0_n", "tau0_l", "tau0_m", "fs_map"):
                a = getattr(ip, name)
                if a is not None:
                    a = np.ascontiguousarray(a, dtype=np.float64)
                    self._keep.append(a)
                    setattr(I, name, _dptr(a))
            self._iface = I
        self.nb = nb
        self.handle = lib().orc_create(nb, descs, C.byref(self._iface) if self._iface is not None else None)

    def close(self):
        if getattr(self, "handle", None):
            lib().orc_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    @property
    def t(self) -> float:
        return lib().orc_time(self.handle)

    @t.setter
    def t(self, v: float):
        lib().orc_set_time(self.handle, float(v))

    def run(self, nsteps: int, dt: Optional[float] = None, w_stride: Optional[int] = None):
        """Advance ``nsteps`` steps; returns seismograms per block, shape (nsamples, nrec, 4)."""
        dt = self.problem.dt() if dt is None else dt
        ws = self.problem.w_stride if w_stride is None else w_stride
        nsamp = (nsteps + ws - 1) // ws if ws > 0 else 0
        out = []
        ptrs = []
        for b in self.problem.blocks[:2]:
            nrec = 0 if b.receivers is None else len(b.receivers)
            a = np.zeros((max(nsamp, 1), max(nrec, 1), 4))
            out.append(a)
            ptrs.append(_dptr(a) if nrec else None)
        while len(ptrs) < 2:
            ptrs.append(None)
        lib().orc_run(self.handle, float(dt), int(nsteps), int(ws), ptrs[0], ptrs[1])
        res = []
        for b, a in zip(self.problem.blocks, out):
            nrec = 0 if b.receivers is None else len(b.receivers)
            res.append(a[:nsamp, :nrec])
        return res

    def stage(self, stage: int, dt: float):
        lib().orc_stage(self.handle, int(stage), float(dt))

    def adjoint_rhs(self, R: np.ndarray, b: int = 0):
        """Transpose of the elastic right-hand side at the current fields:
        (L^T R, (dL/d(lambda, mu, rho) F)^T R) as arrays (9, ns, nr, nq) and
        (3, ns, nr, nq)."""
        Rr = np.ascontiguousarray(R, dtype=np.float64)
        Fb = np.zeros(self._shape(b, 9))
        g = np.zeros(self._shape(b, 3))
        rc = lib().orc_adjoint_rhs(self.handle, b, _dptr(Rr), _dptr(Fb), _dptr(g))
        if rc != 0:
            raise ValueError("the oracle adjoint covers single elastic blocks without PML or interface")
        return Fb, g

    def misfit_gradient(self, observed: np.ndarray, nsteps: int):
        """FP64 discrete adjoint of the waveform misfit chi = 1/2 sum_n sum_r
        |v_r(t_n) - observed[n, r]|^2 over the stage-1 station samples of
        nsteps steps from rest (one elastic block).  Stores every step's state,
        recomputes each step's stage inputs, and reverses the stages with
        adjoint_rhs / adjoint_moment.  Returns (chi, seismograms,
        d chi / d(lambda, mu, rho) as (3, ns, nr, nq), d chi / dM as (nsrc, 6))."""
        from waveqlab3d_q_gpu_b200.problem import RK_A, RK_B, RK_C
        dt = self.problem.dt()
        shape9 = self._shape(0, 9)
        t_start = self.t
        states, seis = [], []
        ridx = self.receiver_index()
        for n in range(nsteps):
            states.append(self.fields())
            F = states[-1]
            seis.append(np.stack([F[c][ridx[:, 2] - 1, ridx[:, 1] - 1, ridx[:, 0] - 1] for c in range(3)], axis=1))
            self.run(1)
        seis = np.array(seis)
        res = seis - observed
        chi = 0.5 * float(np.sum(res * res))
        Fb = np.zeros(shape9)
        gmat = np.zeros(self._shape(0, 3))
        gM = np.zeros((len(self.problem.blocks[0].sources), 6))
        for n in range(nsteps - 1, -1, -1):
            tn = t_start + n * dt
            # stage inputs F^(0..4) of step n
            self.set_fields(states[n])
            self.set_rates(np.zeros(shape9))
            inputs = [states[n]]
            for st in range(1, 5):
                self.t = tn + RK_C[st - 1] * dt
                self.stage(st, dt)
                inputs.append(self.fields())
            DFb = np.zeros(shape9)
            for st in range(5, 0, -1):
                R = DFb + RK_B[st - 1] * dt * Fb
                self.set_fields(inputs[st - 1])
                fb, g = self.adjoint_rhs(R)
                Fb = Fb + fb
                gmat += g
                if len(gM):
                    gM += self.adjoint_moment(tn + RK_C[st - 1] * dt, R)
                DFb = RK_A[st - 1] * R
            for c in range(3):
                np.add.at(Fb[c], (ridx[:, 2] - 1, ridx[:, 1] - 1, ridx[:, 0] - 1), res[n][:, c])
        return chi, seis, gmat, gM

    def adjoint_moment(self, t: float, R: np.ndarray, b: int = 0) -> np.ndarray:
        """Moment-tensor adjoint of the sources at time t for rate adjoint R: (nsrc, 6)."""
        nsrc = len(self.problem.blocks[b].sources)
        g = np.zeros((max(nsrc, 1), 6))
        Rr = np.ascontiguousarray(R, dtype=np.float64)
        lib().orc_adjoint_moment(self.handle, b, float(t), _dptr(Rr), _dptr(g))
        return g[:nsrc]

    def _shape(self, b: int, ncomp: int):
        nq, nr, ns = self.problem.blocks[b].nqrs
        return (ncomp, ns, nr, nq)

    def fields(self, b: int = 0) -> np.ndarray:
        a = np.zeros(self._shape(b, 9))
        lib().orc_get_fields(self.handle, b, _dptr(a))
        return a

    def set_fields(self, F: np.ndarray, b: int = 0):
        a = np.ascontiguousarray(F, dtype=np.float64)
        lib().orc_set_fields(self.handle, b, _dptr(a))

    def rates(self, b: int = 0) -> np.ndarray:
        a = np.zeros(self._shape(b, 9))
        lib().orc_get_rates(self.handle, b, _dptr(a))
        return a

    def set_rates(self, DF: np.ndarray, b: int = 0):
        a = np.ascontiguousarray(DF, dtype=np.float64)
        lib().orc_set_rates(self.handle, b, _dptr(a))

    def metrics(self, b: int = 0) -> np.ndarray:
        a = np.zeros(self._shape(b, 10))
        lib().orc_get_metrics(self.handle, b, _dptr(a))
        return a

    def material(self, b: int = 0) -> np.ndarray:
        a = np.zeros(self._shape(b, 3))
        lib().orc_get_material(self.handle, b, _dptr(a))
        return a

    def eta(self, b: int = 0) -> np.ndarray:
        nm = self.problem.nmech
        nq, nr, ns = self.problem.blocks[b].nqrs
        a = np.zeros((6, max(nm, 1), ns, nr, nq))
        if nm:
            lib().orc_get_eta(self.handle, b, _dptr(a))
        return a[:, :nm]

    def set_eta(self, eta: np.ndarray, b: int = 0):
        a = np.ascontiguousarray(eta, dtype=np.float64)
        lib().orc_set_eta(self.handle, b, _dptr(a))

    def pml(self, face: int, b: int = 0) -> np.ndarray:
        blk = self.problem.blocks[b]
        nq, nr, ns = blk.nqrs
        n = blk.npml
        dims = [ns, nr, nq]
        axis = face // 2  # 0: q, 1: r, 2: s
        dims[2 - axis] = n
        a = np.zeros((9,) + tuple(dims))
        lib().orc_get_pml(self.handle, b, face, _dptr(a))
        return a

    def normals(self, face: int, b: int = 0) -> np.ndarray:
        nq, nr, ns = self.problem.blocks[b].nqrs
        axis = face // 2
        d0 = nr if axis == 0 else nq
        d1 = nr if axis == 2 else ns
        a = np.zeros((9, d1, d0))
        lib().orc_get_normals(self.handle, b, face, _dptr(a))
        return a

    def iface(self) -> np.ndarray:
        nq, nr, ns = self.problem.blocks[0].nqrs
        a = np.zeros((ns, nr, 7))
        lib().orc_get_iface(self.handle, _dptr(a))
        return a

    FAULT_KINDS = {"S": (0, 4), "Svel": (1, 3), "Uhat": (2, 6), "Vhat": (3, 6), "state": (4, 1), "trup": (5, 1)}

    def fault(self, name: str) -> np.ndarray:
        """One fault output (src/fault_output.f90:73-122), shape (ncomp, ns, nr)."""
        kind, nc = self.FAULT_KINDS[name]
        nq, nr, ns = self.problem.blocks[0].nqrs
        a = np.zeros((nc, ns, nr))
        lib().orc_get_fault(self.handle, kind, _dptr(a))
        return a

    def mms_exact(self, t: float, b: int = 0) -> np.ndarray:
        """Manufactured solution at time t on block b's grid, shape (9, ns, nr, nq)."""
        a = np.zeros(self._shape(b, 9))
        lib().orc_mms_exact(self.handle, b, float(t), _dptr(a))
        return a

    def receiver_index(self, b: int = 0) -> np.ndarray:
        blk = self.problem.blocks[b]
        n = 0 if blk.receivers is None else len(blk.receivers)
        a = np.zeros((max(n, 1), 3), dtype=np.int32)
        if n:
            lib().orc_receiver_index(self.handle, b, a.ctypes.data_as(C.POINTER(C.c_int)))
        return a[:n]

    def final_state(self):
        mf, me = C.c_double(), C.c_double()
        mb = (C.c_double * 2)()
        lib().orc_final_state(self.handle, C.byref(mf), C.byref(me), mb)
        return mf.value, me.value, (mb[0], mb[1])


def tfi_grid(faces: np.ndarray, nqrs) -> np.ndarray:
    """Transfinite-interpolation block mesh (Gen3_Curve_Mesh of
    src/grid.f90:2292-2418) from packed surfaces; (3, ns, nr, nq)."""
    nq, nr, ns = nqrs
    f = np.ascontiguousarray(faces, dtype=np.float64)
    out = np.zeros((3, ns, nr, nq))
    lib().orc_tfi_grid(_dptr(f), int(nq), int(nr), int(ns), _dptr(out))
    return out


def upwind_row(fd: int, plus: bool, i: int, n: int):
    """(indices, coefficients) of row i (1-based) of the upwind operator fd's
    D+ (plus) or D- on n points."""
    idx = np.zeros(16, dtype=np.int32)
    c = np.zeros(16)
    k = lib().orc_upwind_row(int(fd), 1 if plus else 0, int(i), int(n),
                             idx.ctypes.data_as(C.POINTER(C.c_int)), _dptr(c))
    return idx[:k].copy(), c[:k].copy()
