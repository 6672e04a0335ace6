!###########################################################
! B200 replacement of hydro/godunov_fine.f90 for the PATCH mechanism:
! godunov_fine, set_unew and set_uold run on the GPU through rb_b200, on the
! device-resident uold (rb_b200_device before each call).
! Same call sites and semantics as the reference (pure hydro: no Poisson
! source terms, no pressure_fix, no momentum feedback, one MPI rank).
!###########################################################
subroutine godunov_fine(ilevel)
  use amr_commons
  use hydro_commons
  use rb_b200
  implicit none
  integer::ilevel
  if(numbtot(1,ilevel)==0)return
  if(static)return
  call rb_b200_device
  call rb_b200_check(rb_godunov_fine(rb_ctx, int(ilevel, c_int), real(dtnew(ilevel), c_double)), 'godunov_fine')
end subroutine godunov_fine
!###########################################################
subroutine set_unew(ilevel)
  use amr_commons
  use hydro_commons
  use rb_b200
  implicit none
  integer::ilevel
  if(numbtot(1,ilevel)==0)return
  call rb_b200_device
  call rb_b200_check(rb_set_unew(rb_ctx, int(ilevel, c_int)), 'set_unew')
end subroutine set_unew
!###########################################################
subroutine set_uold(ilevel)
  use amr_commons
  use hydro_commons
  use rb_b200
  implicit none
  integer::ilevel
  if(numbtot(1,ilevel)==0)return
  if(poisson .or. nener>0)then
     write(*,*)'rb_b200: gravity and non-thermal energy source terms are not supported'
     call clean_stop
  end if
  ! with pressure_fix, rb_set_uold adds the pdV term to enew and repairs the
  ! total energy on the device (add_pdv_source_terms and the fix of set_uold);
  ! uold stays on the device (amr_step's upload_fine that follows is wrapped
  ! to the device too, wrap_b200.f90)
  call rb_b200_device
  call rb_b200_check(rb_set_uold(rb_ctx, int(ilevel, c_int)), 'set_uold')
end subroutine set_uold
!###########################################################
subroutine add_gravity_source_terms(ilevel)
  implicit none
  integer::ilevel
  write(*,*)'rb_b200: add_gravity_source_terms is not supported', ilevel
  call clean_stop
end subroutine add_gravity_source_terms
!###########################################################
subroutine add_pdv_source_terms(ilevel)
  implicit none
  integer::ilevel
  write(*,*)'rb_b200: add_pdv_source_terms runs inside rb_set_uold', ilevel
  call clean_stop
end subroutine add_pdv_source_terms
