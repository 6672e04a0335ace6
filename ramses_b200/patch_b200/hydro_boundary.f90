!###########################################################
! B200 replacement of hydro/hydro_boundary.f90 for the PATCH mechanism: the
! ghost octs of the wall and free boundary regions of level ilevel are filled
! on the GPU from their reference octs (rb_make_boundary_hydro). Imposed
! boundaries (bound_type 3) are rejected by rb_set_boundary, and no_inflow
! (.false. by default) is not applied.
!###########################################################
subroutine make_boundary_hydro(ilevel)
  use amr_commons
  use hydro_commons
  use rb_b200
  implicit none
  integer::ilevel
  if(.not. simple_boundary)return
  call rb_b200_push
  call rb_b200_check(rb_make_boundary_hydro(rb_ctx, int(ilevel, c_int)), 'make_boundary_hydro')
  call rb_b200_pull
end subroutine make_boundary_hydro
