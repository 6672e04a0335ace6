!###########################################################
! B200 replacement of hydro/hydro_flag.f90 for the PATCH mechanism, for runs
! whose refinement uses the gradient criterion only (err_grad_d, err_grad_p,
! err_grad_u of &REFINE_PARAMS; no Jeans or geometric criterion, NENER=0):
! the criterion is evaluated on the device state and only the flags come
! back, one byte per cell of the level; uold stays on the device.
!###########################################################
subroutine hydro_flag(ilevel)
  use amr_commons
  use hydro_commons
  use rb_b200
  implicit none
  integer::ilevel
  type(rb_refine_params_t)::rp
  integer(c_int64_t)::nadd
  if(ilevel==nlevelmax)return
  if(numbtot(1,ilevel)==0)return
  if(err_grad_d==-1.0.and.err_grad_p==-1.0.and.err_grad_u==-1.0)return
  call rb_b200_device
  rp%err_grad_d=err_grad_d; rp%err_grad_p=err_grad_p; rp%err_grad_u=err_grad_u
  rp%floor_d=floor_d; rp%floor_u=floor_u; rp%floor_p=floor_p
  ! flag1 is allocated (0:ncell): pass flag1(0) so that C indexes by icell
  call rb_b200_check(rb_hydro_flag(rb_ctx, int(ilevel,c_int), rp, flag1(0:), nadd), 'hydro_flag')
  nflag=nflag+int(nadd)
end subroutine hydro_flag
