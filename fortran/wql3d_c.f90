! ISO_C_BINDING interface of libwql3d.so (include/wql3d.h) for the reference's
! Fortran driver.  The bind(C) derived types mirror wql3d_block_desc and
! wql3d_domain_desc field for field (tests/test_fortran_binding.py checks the
! field lists against the C header); the interfaces cover the entry points a
! driver calls.  Not compiled here: the image has no Fortran compiler.
module wql3d_c
  use iso_c_binding
  implicit none
  integer(c_int), parameter :: WQL3D_ABI_VERSION = 4
  integer(c_int), parameter :: WQL3D_FP64 = 0, WQL3D_FP32_COMPENSATED = 1
  integer(c_int), parameter :: WQL3D_FD_TRADITIONAL6 = 0, WQL3D_FD_UPWIND4 = 1, WQL3D_FD_UPWIND6 = 2, &
                                WQL3D_FD_UPWIND_DRP6 = 3
  integer(c_int), parameter :: WQL3D_MESH_CARTESIAN = 0, WQL3D_MESH_CURVILINEAR = 1
  integer(c_int), parameter :: WQL3D_IFACE_LOCKED = 0, WQL3D_IFACE_SLIP_WEAKENING = 1, WQL3D_IFACE_LINEAR = 2
  integer(c_int), parameter :: WQL3D_IFACE_RATE_STATE = 3
  integer(c_int), parameter :: WQL3D_FAULT_MAPS = 0, WQL3D_FAULT_TPV5 = 1, WQL3D_FAULT_TPV101 = 2, WQL3D_FAULT_TPV102 = 3, &
                                WQL3D_FAULT_TPV28 = 4

  type, bind(C) :: wql3d_block_desc
     integer(c_int32_t) :: nq, nr, ns, mesh, f32_literal
     integer(c_int32_t) :: bc(6), pml(6), npml
     real(c_double)     :: aqrs(3), bqrs(3), tau0
     integer(c_int32_t) :: host_nb
     type(c_ptr)        :: coords, material, qs_inv, qp_inv
     integer(c_int32_t) :: nsrc, src_order, src_alpha
     type(c_ptr)        :: src_type, src_par
     integer(c_int32_t) :: nrec
     type(c_ptr)        :: rec_xyz
     integer(c_int32_t) :: fd_operator
  end type

  type, bind(C) :: wql3d_domain_desc
     integer(c_int32_t) :: abi_version, nblocks, precision, response, coarse_grain
     real(c_double)     :: Qs0, Qp0, tau(8), weight(8), strength_s(8), strength_p(8)
     integer(c_int32_t) :: coupling, fault_problem, serial_shared
     real(c_double)     :: fs, fd, Dc
     type(c_ptr)        :: iface_tau0, iface_fs
     real(c_double)     :: fault_stress(6)
     integer(c_int32_t) :: max_samples
     integer(c_int32_t) :: mms
     real(c_double)     :: mms_nt, mms_nx, mms_ny, mms_nz
     integer(c_int32_t) :: remote_side
     integer(c_int32_t) :: slab_z0, slab_ns_global
     type(c_ptr)        :: slab_ghost_coords
     type(wql3d_block_desc) :: block(2)
  end type

  interface
     integer(c_int) function wql3d_domain_create(desc, d) bind(C)
       import; type(wql3d_domain_desc), intent(in) :: desc; type(c_ptr) :: d
     end function
     integer(c_int) function wql3d_domain_destroy(d) bind(C)
       import; type(c_ptr), value :: d
     end function
     integer(c_int) function wql3d_set_fields(d, block, F, host_nb) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: block, host_nb
       real(c_double), intent(in) :: F(*)
     end function
     integer(c_int) function wql3d_get_fields(d, block, F, host_nb) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: block, host_nb
       real(c_double), intent(out) :: F(*)
     end function
     integer(c_int) function wql3d_time_step(d, dt, n, w_stride) bind(C)
       import; type(c_ptr), value :: d; real(c_double), value :: dt; integer(c_int), value :: n, w_stride
     end function
     integer(c_int) function wql3d_run(d, dt, n_first, nsteps, w_stride) bind(C)
       import; type(c_ptr), value :: d; real(c_double), value :: dt
       integer(c_int), value :: n_first, nsteps, w_stride
     end function
     integer(c_int) function wql3d_scale_rates(d, A) bind(C)
       import; type(c_ptr), value :: d; real(c_double), value :: A
     end function
     integer(c_int) function wql3d_set_rates_rhs(d) bind(C)
       import; type(c_ptr), value :: d
     end function
     integer(c_int) function wql3d_enforce_bound_iface_conditions(d, stage) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: stage
     end function
     integer(c_int) function wql3d_update_fields(d, dt) bind(C)
       import; type(c_ptr), value :: d; real(c_double), value :: dt
     end function
     integer(c_int) function wql3d_scale_rate_array(rate, n, a, stream) bind(C)
       import; type(c_ptr), value :: rate, stream; integer(c_int64_t), value :: n; real(c_double), value :: a
     end function
     integer(c_int) function wql3d_traditional_cartesian_rhs(field, rate, metricx, metricy, metricz, material, &
          n1, n2, n3, nm, nmat, xlo, xhi, ylo, yhi, zlo, zhi, hq, hr, hs, stream) bind(C)
       import; type(c_ptr), value :: field, rate, metricx, metricy, metricz, material, stream
       integer(c_int32_t), value :: n1, n2, n3, nm, nmat, xlo, xhi, ylo, yhi, zlo, zhi
       real(c_double), value :: hq, hr, hs
     end function
     integer(c_int) function wql3d_update_state_array(state, rate, n, dt, stream) bind(C)
       import; type(c_ptr), value :: state, rate, stream; integer(c_int64_t), value :: n; real(c_double), value :: dt
     end function
     integer(c_int) function wql3d_get_seismograms(d, block, out, nsamples) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: block
       real(c_double), intent(out) :: out(*); integer(c_int32_t), intent(out) :: nsamples
     end function
     integer(c_int) function wql3d_get_fault_output(d, kind, out) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: kind; real(c_double), intent(out) :: out(*)
     end function
     integer(c_int) function wql3d_get_plane(d, block, axis, index, c0, ncomp, out) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: block, axis, index, c0, ncomp
       real(c_double), intent(out) :: out(*)
     end function
     integer(c_int) function wql3d_final_state(d, max_field, max_memory, block_max) bind(C)
       import; type(c_ptr), value :: d; real(c_double), intent(out) :: max_field, max_memory, block_max(*)
     end function
     integer(c_int) function wql3d_begin_step(d, n, w_stride) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: n, w_stride
     end function
     integer(c_int) function wql3d_stage(d, stage, dt) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: stage; real(c_double), value :: dt
     end function
     integer(c_int) function wql3d_interface_buffers(d, send, recv, count, elem_bytes) bind(C)
       import; type(c_ptr), value :: d; type(c_ptr) :: send, recv
       integer(c_int64_t) :: count; integer(c_int32_t) :: elem_bytes
     end function
     integer(c_int) function wql3d_pack_interface(d) bind(C)
       import; type(c_ptr), value :: d
     end function
     integer(c_int) function wql3d_get_interface_material(d, M) bind(C)
       import; type(c_ptr), value :: d; real(c_double), intent(out) :: M(*)
     end function
     integer(c_int) function wql3d_set_interface_remote_material(d, M) bind(C)
       import; type(c_ptr), value :: d; real(c_double), intent(in) :: M(*)
     end function
     integer(c_int) function wql3d_halo_buffers(d, kind, send, recv, count, elem_bytes) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: kind; type(c_ptr) :: send, recv
       integer(c_int64_t) :: count; integer(c_int32_t) :: elem_bytes
     end function
     integer(c_int) function wql3d_pack_halo(d, kind) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: kind
     end function
     integer(c_int) function wql3d_unpack_halo(d, kind) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: kind
     end function
     integer(c_int) function wql3d_set_time(d, t) bind(C)
       import; type(c_ptr), value :: d; real(c_double), value :: t
     end function
     integer(c_int) function wql3d_set_material(d, block, M) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: block; real(c_double), intent(in) :: M(*)
     end function
     integer(c_int) function wql3d_set_moment(d, block, m6) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: block; real(c_double), intent(in) :: m6(*)
     end function
     integer(c_int) function wql3d_adjoint_enable(d) bind(C)
       import; type(c_ptr), value :: d
     end function
     integer(c_int) function wql3d_adjoint_reset(d) bind(C)
       import; type(c_ptr), value :: d
     end function
     integer(c_int) function wql3d_adjoint_step(d, n, dt) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: n; real(c_double), value :: dt
     end function
     integer(c_int) function wql3d_adjoint_add_receivers(d, block, res) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: block; real(c_double), intent(in) :: res(*)
     end function
     integer(c_int) function wql3d_get_adjoint_gradient(d, block, g_material, g_moment) bind(C)
       import; type(c_ptr), value :: d; integer(c_int), value :: block
       real(c_double), intent(out) :: g_material(*), g_moment(*)
     end function
     type(c_ptr) function wql3d_last_error() bind(C)
       import
     end function
  end interface
end module wql3d_c
