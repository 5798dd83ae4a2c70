! Drop-in backend for the reference's rk_vector seam (src/rk_vector_cpu.f90:7-18,
! src/rk_vector_openacc.f90:8-75): scale_rate_array / update_state_array on
! arrays that live on the device (an OpenACC data region), carried out by
! libwql3d.so's kernels through the device addresses of the arrays.
! Selected at build time in place of rk_vector_openacc.f90
! (src/CMakeLists.txt:20-38).  Not compiled here: the image has no Fortran
! compiler.
module rk_vector_backend
  use common, only : wp
  use iso_c_binding
  use wql3d_c, only : wql3d_scale_rate_array, wql3d_update_state_array, wql3d_last_error
  implicit none
  private
  public :: scale_rate_array, update_state_array

contains

  subroutine scale_rate_array(rate, coefficient)
    real(kind = wp), dimension(:,:,:,:), allocatable, intent(inout) :: rate
    real(kind = wp), intent(in) :: coefficient
    integer(c_int) :: ierr
    if (.not. allocated(rate)) return
    !$acc host_data use_device(rate)
    ierr = wql3d_scale_rate_array(c_loc(rate), int(size(rate), c_int64_t), real(coefficient, c_double), c_null_ptr)
    !$acc end host_data
    if (ierr /= 0) error stop 'wql3d_scale_rate_array failed'
  end subroutine scale_rate_array

  subroutine update_state_array(state, rate, increment)
    real(kind = wp), dimension(:,:,:,:), allocatable, intent(inout) :: state
    real(kind = wp), dimension(:,:,:,:), allocatable, intent(in) :: rate
    real(kind = wp), intent(in) :: increment
    integer(c_int) :: ierr
    if (.not. allocated(state)) return
    !$acc host_data use_device(state, rate)
    ierr = wql3d_update_state_array(c_loc(state), c_loc(rate), int(size(state), c_int64_t), &
                                    real(increment, c_double), c_null_ptr)
    !$acc end host_data
    if (ierr /= 0) error stop 'wql3d_update_state_array failed'
  end subroutine update_state_array

end module rk_vector_backend
