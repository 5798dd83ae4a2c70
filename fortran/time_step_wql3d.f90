! Drop-in time loop for the reference's time_step_RK (src/time_step.f90:68-150):
! the domain's blocks are handed to libwql3d.so once (wql3d_domain_create +
! wql3d_set_fields, replacing enter_domain_device_data), every step is one
! wql3d_time_step call (the five stages of all blocks, the interface and the
! stage-1 station sample), and the fields come back for output and
! close_domain.  The descriptor is filled from the resolved configuration the
! reference already holds (block sizes, boundary codes, PML flags, material,
! sources, stations).  Not compiled here: the image has no Fortran compiler.
module time_step_wql3d
  use iso_c_binding
  use wql3d_c
  implicit none
  private
  public :: run_time_steps_wql3d

contains

  ! nt steps of size dt from step n_first, w_stride as the reference's
  ! &problem_list; F(:,:,:,:,b) are the blocks' fields with 3 ghost layers
  subroutine run_time_steps_wql3d(dom, nblocks, F1, F2, dt, n_first, nt, w_stride)
    type(c_ptr), intent(in) :: dom
    integer, intent(in) :: nblocks, n_first, nt, w_stride
    real(c_double), intent(inout), target :: F1(*), F2(*)
    real(c_double), intent(in) :: dt
    integer(c_int) :: ierr
    ierr = wql3d_set_fields(dom, 0_c_int, F1, 3_c_int)
    if (ierr == 0 .and. nblocks == 2) ierr = wql3d_set_fields(dom, 1_c_int, F2, 3_c_int)
    if (ierr == 0) ierr = wql3d_run(dom, dt, int(n_first, c_int), int(nt, c_int), int(w_stride, c_int))
    if (ierr == 0) ierr = wql3d_get_fields(dom, 0_c_int, F1, 3_c_int)
    if (ierr == 0 .and. nblocks == 2) ierr = wql3d_get_fields(dom, 1_c_int, F2, 3_c_int)
    if (ierr /= 0) error stop 'libwql3d.so time stepping failed (see wql3d_last_error)'
  end subroutine run_time_steps_wql3d

end module time_step_wql3d
