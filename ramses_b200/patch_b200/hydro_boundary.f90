!###########################################################
! B200 replacement of hydro/hydro_boundary.f90 for the PATCH mechanism: the
! ghost octs of the wall and free boundary regions of level ilevel are filled
! on the GPU from their reference octs (rb_make_boundary_hydro), on the
! device-resident uold. Imposed boundaries (bound_type 3) are rejected by
! rb_set_boundary, and rb_b200_init stops on no_inflow = .true.
!###########################################################
subroutine make_boundary_hydro(ilevel)
  use amr_commons
  use hydro_commons
  use rb_b200
  implicit none
  integer::ilevel
  if(.not. simple_boundary)return
  call rb_b200_device
  call rb_b200_check(rb_make_boundary_hydro(rb_ctx, int(ilevel, c_int)), 'make_boundary_hydro')
end subroutine make_boundary_hydro
