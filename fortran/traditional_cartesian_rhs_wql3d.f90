! Drop-in backend for the reference's try_traditional_cartesian_rhs seam
! (src/traditional_cartesian_rhs_cpu.f90:8-15, the OpenACC backend
! src/traditional_cartesian_rhs_openacc.f90): the strict-interior rates of a
! Cartesian elastic traditional-6 block without PML or memory variables,
! computed by libwql3d.so on the device copies of F%F%F, F%F%DF, the metrics and
! the material (an OpenACC data region).  The same applicability checks as the
! OpenACC backend decide whether the call is handled; otherwise handled is
! false and the reference's JJU_x6_interior runs.  Selected at build time in
! place of traditional_cartesian_rhs_openacc.f90 (src/CMakeLists.txt:20-38).
! Not compiled here: the image has no Fortran compiler.
module traditional_cartesian_rhs_backend
  use common, only : wp
  use iso_c_binding
  use datatypes, only : block_type, block_grid_t, block_material
  use wql3d_c, only : wql3d_traditional_cartesian_rhs
  implicit none
  private
  public :: try_traditional_cartesian_rhs

contains

  subroutine try_traditional_cartesian_rhs(F, G, M, type_of_mesh, handled)
    use mpi3dbasic, only : nprocs
    type(block_type), intent(inout) :: F
    type(block_grid_t), intent(in) :: G
    type(block_material), intent(inout) :: M
    character(len=*), intent(in) :: type_of_mesh
    logical, intent(out) :: handled
    integer :: n1, n2, n3, xlo, xhi, ylo, yhi, zlo, zhi
    integer(c_int) :: ierr
    handled = .false.
    if (nprocs /= 1) return
    if (trim(type_of_mesh) /= 'cartesian') return
    if (trim(F%fd_type) /= 'traditional' .or. F%order /= 6) return
    if (M%anelastic .or. M%anelastic_Q .or. M%anelastic_Q8 .or. M%anelastic_Qf .or. M%anelastic_Qf8 .or. &
        M%anelastic_const_Q_4M .or. M%anelastic_const_Q_8M) return
    if (any(F%PMLB(:)%pml)) return
    if (.not. allocated(F%F%F) .or. .not. allocated(F%F%DF) .or. .not. allocated(G%metricx) .or. &
        .not. allocated(G%metricy) .or. .not. allocated(G%metricz) .or. .not. allocated(M%M)) return
    if (size(F%F%F, 4) /= 9 .or. size(M%M, 4) < 3 .or. size(G%metricx, 4) < 3) return
    if (any(shape(F%F%DF) /= shape(F%F%F))) return
    if (any(lbound(F%F%DF) /= lbound(F%F%F))) return
    if (any(shape(G%metricx) /= shape(G%metricy)) .or. any(shape(G%metricx) /= shape(G%metricz))) return
    if (any(shape(G%metricx(:,:,:,1)) /= shape(F%F%F(:,:,:,1)))) return
    if (any(shape(M%M(:,:,:,1)) /= shape(F%F%F(:,:,:,1)))) return
    if (any(lbound(G%metricx(:,:,:,1)) /= lbound(F%F%F(:,:,:,1)))) return
    n1 = size(F%F%F, 1); n2 = size(F%F%F, 2); n3 = size(F%F%F, 3)
    if (n1 < 13 .or. n2 < 13 .or. n3 < 13) return
    ! strict interior 7 .. n - 6 in the arrays' own 1-based indices
    xlo = 7 - lbound(F%F%F, 1) + 1; xhi = G%C%nq - 6 - lbound(F%F%F, 1) + 1
    ylo = 7 - lbound(F%F%F, 2) + 1; yhi = G%C%nr - 6 - lbound(F%F%F, 2) + 1
    zlo = 7 - lbound(F%F%F, 3) + 1; zhi = G%C%ns - 6 - lbound(F%F%F, 3) + 1
    if (xlo < 4 .or. xhi > n1 - 3 .or. xlo > xhi .or. ylo < 4 .or. yhi > n2 - 3 .or. ylo > yhi .or. &
        zlo < 4 .or. zhi > n3 - 3 .or. zlo > zhi) return
    !$acc host_data use_device(F%F%F, F%F%DF, G%metricx, G%metricy, G%metricz, M%M)
    ierr = wql3d_traditional_cartesian_rhs(c_loc(F%F%F), c_loc(F%F%DF), c_loc(G%metricx), c_loc(G%metricy), &
         c_loc(G%metricz), c_loc(M%M), int(n1, c_int32_t), int(n2, c_int32_t), int(n3, c_int32_t), &
         int(size(G%metricx, 4), c_int32_t), int(size(M%M, 4), c_int32_t), int(xlo, c_int32_t), &
         int(xhi, c_int32_t), int(ylo, c_int32_t), int(yhi, c_int32_t), int(zlo, c_int32_t), &
         int(zhi, c_int32_t), real(G%hq, c_double), real(G%hr, c_double), real(G%hs, c_double), c_null_ptr)
    !$acc end host_data
    if (ierr /= 0) error stop 'wql3d_traditional_cartesian_rhs failed'
    handled = .true.
  end subroutine try_traditional_cartesian_rhs

end module traditional_cartesian_rhs_backend
