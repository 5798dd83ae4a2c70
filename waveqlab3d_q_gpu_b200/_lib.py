"""ctypes binding of libwql3d.so (the C ABI declared in include/wql3d.h).

The shared library is built in-tree by :func:`waveqlab3d_q_gpu_b200.build.build`.
Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwql3d.so")

ABI_VERSION = 4
RECORD_FIELDS = 10   # WQL3D_RECORD_FIELDS: field volumes per recorded step
OK = 0
ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "ENONFINITE", -5: "ESTATE"}

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)


class BlockDesc(C.Structure):
    _fields_ = [
        ("nq", C.c_int32), ("nr", C.c_int32), ("ns", C.c_int32),
        ("mesh", C.c_int32), ("f32_literal", C.c_int32),
        ("bc", C.c_int32 * 6), ("pml", C.c_int32 * 6), ("npml", C.c_int32),
        ("aqrs", C.c_double * 3), ("bqrs", C.c_double * 3),
        ("tau0", C.c_double),
        ("host_nb", C.c_int32),
        ("coords", dp), ("material", dp), ("qs_inv", dp), ("qp_inv", dp),
        ("nsrc", C.c_int32), ("src_order", C.c_int32), ("src_alpha", C.c_int32),
        ("src_type", ip), ("src_par", dp),
        ("nrec", C.c_int32), ("rec_xyz", dp),
        ("fd_operator", C.c_int32),
    ]


class DomainDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("nblocks", C.c_int32), ("precision", C.c_int32),
        ("response", C.c_int32), ("coarse_grain", C.c_int32),
        ("Qs0", C.c_double), ("Qp0", C.c_double),
        ("tau", C.c_double * 8), ("weight", C.c_double * 8),
        ("strength_s", C.c_double * 8), ("strength_p", C.c_double * 8),
        ("coupling", C.c_int32), ("fault_problem", C.c_int32), ("serial_shared", C.c_int32),
        ("fs", C.c_double), ("fd", C.c_double), ("Dc", C.c_double),
        ("iface_tau0", dp), ("iface_fs", dp), ("fault_stress", C.c_double * 6),
        ("max_samples", C.c_int32),
        ("mms", C.c_int32), ("mms_nt", C.c_double), ("mms_nx", C.c_double), ("mms_ny", C.c_double),
        ("mms_nz", C.c_double),
        ("remote_side", C.c_int32),
        ("slab_z0", C.c_int32), ("slab_ns_global", C.c_int32), ("slab_ghost_coords", dp),
        ("block", BlockDesc * 2),
    ]


# every exported symbol with its argument types (restype is int unless noted)
SIGNATURES = {
    "wql3d_domain_create": [C.POINTER(DomainDesc), C.POINTER(C.c_void_p)],
    "wql3d_domain_destroy": [C.c_void_p],
    "wql3d_set_fields": [C.c_void_p, C.c_int, dp, C.c_int32],
    "wql3d_get_fields": [C.c_void_p, C.c_int, dp, C.c_int32],
    "wql3d_set_rates": [C.c_void_p, C.c_int, dp, C.c_int32],
    "wql3d_get_rates": [C.c_void_p, C.c_int, dp, C.c_int32],
    "wql3d_get_memory_variables": [C.c_void_p, C.c_int, dp],
    "wql3d_get_metrics": [C.c_void_p, C.c_int, dp],
    "wql3d_get_interface": [C.c_void_p, dp],
    "wql3d_get_fault_output": [C.c_void_p, C.c_int, dp],
    "wql3d_get_plane": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp],
    "wql3d_set_time": [C.c_void_p, C.c_double],
    "wql3d_get_time": [C.c_void_p, dp],
    "wql3d_stage": [C.c_void_p, C.c_int, C.c_double],
    "wql3d_time_step": [C.c_void_p, C.c_double, C.c_int, C.c_int],
    "wql3d_run": [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int],
    "wql3d_begin_step": [C.c_void_p, C.c_int, C.c_int],
    "wql3d_interface_buffers": [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                C.POINTER(C.c_int32)],
    "wql3d_pack_interface": [C.c_void_p],
    "wql3d_halo_buffers": [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                           C.POINTER(C.c_int32)],
    "wql3d_pack_halo": [C.c_void_p, C.c_int],
    "wql3d_unpack_halo": [C.c_void_p, C.c_int],
    "wql3d_get_interface_material": [C.c_void_p, dp],
    "wql3d_set_interface_remote_material": [C.c_void_p, dp],
    "wql3d_scale_rates": [C.c_void_p, C.c_double],
    "wql3d_set_rates_rhs": [C.c_void_p],
    "wql3d_enforce_bound_iface_conditions": [C.c_void_p, C.c_int],
    "wql3d_update_fields": [C.c_void_p, C.c_double],
    "wql3d_try_traditional_rhs": [C.c_void_p, C.POINTER(C.c_int)],
    "wql3d_scale_rate_array": [C.c_void_p, C.c_int64, C.c_double, C.c_void_p],
    "wql3d_traditional_cartesian_rhs": [C.c_void_p] * 6 + [C.c_int32] * 11 + [C.c_double] * 3 + [C.c_void_p],
    "wql3d_update_state_array": [C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.c_void_p],
    "wql3d_get_seismograms": [C.c_void_p, C.c_int, dp, ip],
    "wql3d_receiver_index": [C.c_void_p, C.c_int, ip],
    "wql3d_final_state": [C.c_void_p, dp, dp, dp],
    "wql3d_synchronize": [C.c_void_p],
    "wql3d_get_stream": [C.c_void_p, C.POINTER(C.c_void_p)],
    "wql3d_device_bytes": [C.c_void_p, C.POINTER(C.c_int64)],
    "wql3d_kernel_launches": [C.c_void_p, C.POINTER(C.c_int64)],
    "wql3d_last_error": [],
    "wql3d_max_abs_noalloc": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p],
    "wql3d_reset_samples": [C.c_void_p],
    "wql3d_tfi_grid": [dp, C.c_int32, C.c_int32, C.c_int32, dp],
    "wql3d_batch_create": [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)],
    "wql3d_batch_run": [C.c_void_p, C.c_double, C.c_int32, C.c_int32],
    "wql3d_batch_tuning": [C.c_void_p, ip, ip, ip, C.POINTER(C.c_float)],
    "wql3d_batch_launches": [C.c_void_p, C.POINTER(C.c_int64)],
    "wql3d_batch_synchronize": [C.c_void_p],
    "wql3d_batch_destroy": [C.c_void_p],
    "wql3d_check_status": [C.c_void_p, ip],
    "wql3d_set_material": [C.c_void_p, C.c_int, dp],
    "wql3d_set_moment": [C.c_void_p, C.c_int, dp],
    "wql3d_field_volume": [C.c_void_p, C.c_int, C.POINTER(C.c_int64)],
    "wql3d_store_fields": [C.c_void_p, C.c_int, C.c_void_p],
    "wql3d_load_fields": [C.c_void_p, C.c_int, C.c_void_p],
    "wql3d_adjoint_enable": [C.c_void_p],
    "wql3d_adjoint_reset": [C.c_void_p],
    "wql3d_adjoint_step": [C.c_void_p, C.c_int, C.c_double],
    "wql3d_adjoint_add_receivers": [C.c_void_p, C.c_int, dp],
    "wql3d_record_step": [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_void_p],
    "wql3d_adjoint_step_recorded": [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_void_p],
    "wql3d_adjoint_rhs": [C.c_void_p, C.c_int, dp, dp, dp],
    "wql3d_get_adjoint_fields": [C.c_void_p, C.c_int, dp],
    "wql3d_get_adjoint_gradient": [C.c_void_p, C.c_int, dp, dp],
}

_LIB = None


class Wql3dError(RuntimeError):
    pass


def load() -> C.CDLL:
    """Load the in-tree libwql3d.so (raises when it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise Wql3dError(f"{LIB_PATH} is missing: build it with waveqlab3d_q_gpu_b200.build.build()")
    L = C.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_char_p if name == "wql3d_last_error" else C.c_int
    _LIB = L
    return L


def check(rc: int, what: str = ""):
    if rc != OK:
        msg = load().wql3d_last_error().decode(errors="replace")
        raise Wql3dError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")
