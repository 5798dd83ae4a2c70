"""Problem description mirroring the reference's input namelists.

The reference reads ``&problem_list``, ``&block_list``, ``&moment_list``,
the anelastic lists and the ``!---begin:tensor_listU---`` source rows
(src/input_preflight.f90:21-211, src/simulation_config.f90:10-48,
src/moment_tensor.f90:125-133).  This module holds the same information as
plain dataclasses so that a run can be described once and handed to the
CUDA product (``waveqlab3d_q_gpu_b200.domain``) or to the CPU oracle.

Units follow the reference: km, km/s, g/cm^3 (moduli in GPa), seconds.
Arrays are numpy arrays in Fortran point order (q/x fastest), i.e. numpy
C-order shape ``(ns, nr, nq)`` per component.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

# source-time-function names of src/moment_tensor.f90:813-873; 'ricker' is
# an addition of this library (the reference has no Ricker wavelet)
STF_CODES = {
    "gaussian": 0,
    "LOH_discontinuity": 1,
    "Brune": 2,
    "Cos-Bell": 3,
    "cosine": 4,
    "LOH_moment_time_history": 5,
    "sine_moment_time_history": 6,
    "ricker": 7,
}

RESPONSES = {"elastic": 0, "anelastic-Q4": 1, "anelastic-Q8": 2, "anelastic-fQ8": 3}

COUPLINGS = {"locked": 0, "slip-weakening_friction": 1, "linear_friction": 2, "rate-and-state_friction": 3}
# fault prestress / strength: per-point maps, or the reference's TPV5 / TPV28
# formulas; TPV101 / TPV102: prestress and rate-and-state parameters of the reference
FAULT_PROBLEMS = {None: 0, "maps": 0, "TPV5": 1, "TPV101": 2, "TPV102": 3, "TPV28": 4}

# derivative operators (fd_type, order) -> WQL3D_FD_* and their SAT penalties
# (src/RHS_Interior.f90:36-128, src/block.f90:242-300)
FD_OPERATORS = {("traditional", 6): 0, ("upwind", 4): 1, ("upwind", 6): 2, ("upwind_drp", 6): 3}
SAT_PENALTY = {1: 144.0 / 49.0, 2: 42300.0 / 13613.0, 3: 3.39644507697204}

# Kennedy-Carpenter (5,4) low-storage coefficients, src/time_step.f90:53-62
RK_A = (
    0.0,
    -567301805773.0 / 1357537059087.0,
    -2404267990393.0 / 2016746695238.0,
    -3550918686646.0 / 2091501179385.0,
    -1275806237668.0 / 842570457699.0,
)
RK_B = (
    1432997174477.0 / 9575080441755.0,
    5161836677717.0 / 13612068292357.0,
    1720146321549.0 / 2090206949498.0,
    3134564353537.0 / 4481467310338.0,
    2277821191437.0 / 14882151754819.0,
)
RK_C = (
    0.0,
    1432997174477.0 / 9575080441755.0,
    2526269341429.0 / 6820363962896.0,
    2006345519317.0 / 3224310063776.0,
    2802321613138.0 / 2924317926251.0,
    1.0,
)

# SAT penalty of the traditional-6 operator, src/block.f90:242
TAU0_TRADITIONAL6 = 1.0 / 0.315949074074074


@dataclass
class Source:
    """One row of ``tensor_listU``: type, duration, t_init, moment tensor, location."""

    stf: str = "Cos-Bell"
    duration: float = 0.0
    t_init: float = 0.0
    mxx: float = 0.0
    myy: float = 0.0
    mzz: float = 0.0
    mxy: float = 0.0
    mxz: float = 0.0
    myz: float = 0.0
    x: float = 0.0
    y: float = 0.0
    z: float = 0.0

    def params(self) -> List[float]:
        return [self.duration, self.t_init, self.mxx, self.myy, self.mzz, self.mxy, self.mxz, self.myz,
                self.x, self.y, self.z]


@dataclass
class Block:
    """One ``btp(i)`` entry of ``&block_list`` plus optional arrays."""

    nqrs: Tuple[int, int, int]
    aqrs: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    bqrs: Tuple[float, float, float] = (1.0, 1.0, 1.0)
    rho_s_p: Tuple[float, float, float] = (2.67, 3.464, 6.0)
    lqrs: Tuple[int, int, int] = (1, 1, 1)   # type_of_bc on q-, r-, s-min faces
    rqrs: Tuple[int, int, int] = (1, 1, 1)   # type_of_bc on q-, r-, s-max faces
    pml_lqrs: Tuple[bool, bool, bool] = (False, False, False)
    pml_rqrs: Tuple[bool, bool, bool] = (False, False, False)
    npml: int = 0
    coords: Optional[np.ndarray] = None      # (3, ns, nr, nq) physical coordinates (mesh_source='file')
    material: Optional[np.ndarray] = None    # (3, ns, nr, nq) lambda, mu, rho (material_source='file')
    qs_inv: Optional[np.ndarray] = None      # (ns, nr, nq) per-point 1/Qs (Q4/Q8)
    qp_inv: Optional[np.ndarray] = None
    sources: List[Source] = field(default_factory=list)
    receivers: Optional[np.ndarray] = None   # (nrec, 3) physical coordinates

    @property
    def npoints(self) -> int:
        return int(self.nqrs[0]) * int(self.nqrs[1]) * int(self.nqrs[2])

    def bc(self) -> List[int]:
        """type_of_bc per face in the order Lx, Rx, Ly, Ry, Lz, Rz (src/BoundaryConditions.f90:15-48)."""
        return [self.lqrs[0], self.rqrs[0], self.lqrs[1], self.rqrs[1], self.lqrs[2], self.rqrs[2]]

    def pml(self) -> List[int]:
        """PML flags in face order 1..6 (src/block.f90:198-205)."""
        return [int(self.pml_lqrs[0]), int(self.pml_rqrs[0]), int(self.pml_lqrs[1]), int(self.pml_rqrs[1]),
                int(self.pml_lqrs[2]), int(self.pml_rqrs[2])]


@dataclass
class AnelasticParams:
    """Q4 / Q8 / fQ8 parameters (src/anelastic_q4_model.f90, q8, fq8)."""

    Qs0: float = 50.0
    Qp0: float = 100.0
    fref: float = 1.0
    fmin: float = 0.05
    fmax: float = 20.0
    gamma: float = 0.0
    f_transition: float = 1.0
    coarse_grain: int = 0
    coefficient_method: Optional[str] = None   # fQ8: 'conventional-nnls' or 'withers-2015'
    weight_policy: Optional[str] = None        # fQ8: 'table-exact' or 'nonnegative-refit'
    tau: Optional[Sequence[float]] = None        # overrides the builders when given
    weight: Optional[Sequence[float]] = None
    strength_s: Optional[Sequence[float]] = None
    strength_p: Optional[Sequence[float]] = None


@dataclass
class InterfaceParams:
    """Interface friction parameters (src/Interface_Condition.f90)."""

    coupling: str = "locked"
    fs: float = 0.677
    fd: float = 0.525
    Dc: float = 0.4
    tau0_n: Optional[np.ndarray] = None   # (ns, nr) initial normal traction
    tau0_m: Optional[np.ndarray] = None   # (ns, nr) initial shear traction along m
    tau0_l: Optional[np.ndarray] = None   # (ns, nr) initial shear traction along l
    fs_map: Optional[np.ndarray] = None   # (ns, nr) static friction map
    # True: both sides' interface solves add to the slip rate, as in the
    # reference's one-process two-block run (src/domain.f90:615-644 calls
    # Interface_RHS once per block on one shared iface); False: once per
    # stage, as in its one-rank-per-block run, which the archived rupture
    # output (test_problems/truth/1) follows.
    serial_shared: bool = False
    problem: Optional[str] = None         # 'TPV5': prestress and strength of src/Interface_Condition.f90
    # 'TPV28': background stress (sxx, syy, szz, sxy, sxz, syz) projected on
    # each fault point's (n, m, l) basis; None: the tensor of
    # src/initial_stress_condition.f90:78-84, (-60, 0, 60, 0, 29.38, 0)
    stress: Optional[tuple] = None


@dataclass
class MMSParams:
    """Manufactured solution of src/mms.f90:136-235: v = cos(nt pi t) sin sin sin,
    sigma = cos(nt pi t) cos cos cos (wavenumbers nx, ny, nz times pi).  When a
    problem carries one, the rates get the forcing u*_t - L(u*) and the face
    SATs the exact boundary data (src/BoundaryConditions.f90:84-88)."""

    nt: float = 2.0
    nx: float = 1.0
    ny: float = 1.0
    nz: float = 1.0


@dataclass
class Problem:
    """``&problem_list`` plus blocks."""

    blocks: List[Block]
    response: str = "elastic"
    type_of_mesh: str = "cartesian"
    t_final: float = 1.0
    CFL: float = 0.5
    w_stride: int = 1
    source_order: int = 2
    source_alpha: int = 0
    # SBP row-4 literal 0.013435342414630 carries no kind suffix in the
    # reference: double under gfortran -fdefault-real-8 (cpu-release), single
    # under nvfortran without -r8.  Both reproduce the published 16-digit pin.
    closure_f32_literal: bool = False
    anelastic: AnelasticParams = field(default_factory=AnelasticParams)
    interface: InterfaceParams = field(default_factory=InterfaceParams)
    tau0: float = TAU0_TRADITIONAL6
    mms: Optional[MMSParams] = None
    # derivative operator of &problem_list: fd_type 'traditional' (order 6),
    # 'upwind' (order 4 or 6) or 'upwind_drp' (order 6); the upwind pairs take
    # the forward operator on the velocities, the backward on the stresses
    # (src/JU_xJU_yJU_z6.f90:1439-3688, 10556-12058)
    fd_type: str = "traditional"
    order: int = 6

    def fd_operator(self) -> int:
        """Operator code of the C descriptors: 0 traditional-6, 1 upwind-4,
        2 upwind-6, 3 upwind-DRP-6."""
        code = FD_OPERATORS.get((self.fd_type, self.order))
        if code is None:
            raise ValueError("unsupported operator fd_type=%r order=%r" % (self.fd_type, self.order))
        return code

    def sat_penalty(self) -> float:
        """SAT penalty tau0 of the operator, src/block.f90:242-300:
        1/0.315949074074074 for traditional-6, 144/49 for upwind-4,
        42300/13613 for upwind-6, 3.39644507697204 for upwind-DRP-6."""
        return SAT_PENALTY.get(self.fd_operator(), self.tau0)

    def dt(self) -> float:
        """Global time step, src/domain.f90:150-171 and src/block.f90:495-510.

        Uses only the scalar ``rho_s_p`` of each block (not the material arrays),
        exactly like the reference.  Q4/Q8/fQ8 runs add the relaxation limit
        2*min(tau) (src/anelastic_q4_model.f90:143-149).
        """
        dtmin = math.inf
        for b in self.blocks:
            spat = [(b.bqrs[i] - b.aqrs[i]) / float(b.nqrs[i] - 1) for i in range(3)]
            h = min(spat)
            dtmin = min(dtmin, self.CFL * h / math.sqrt(b.rho_s_p[1] ** 2 + b.rho_s_p[2] ** 2))
        if self.response != "elastic":
            from .anelastic import coefficients
            tau, _, _ = coefficients(self.response, self.anelastic)
            dtmin = min(dtmin, 2.0 * min(tau))
        return dtmin

    def nt(self) -> int:
        """Number of time steps, src/domain.f90:230."""
        return int(math.floor(self.t_final / self.dt()))

    @property
    def nmech(self) -> int:
        return {"elastic": 0, "anelastic-Q4": 4, "anelastic-Q8": 8, "anelastic-fQ8": 8}[self.response]
