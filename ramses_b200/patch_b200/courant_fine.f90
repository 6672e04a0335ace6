!###########################################################
! B200 replacement of hydro/courant_fine.f90 for the PATCH mechanism: the CFL
! time step and the mass/energy totals of level ilevel's leaf cells are
! reduced on the GPU; the MPI reduction of the scalars is kept.
!###########################################################
subroutine courant_fine(ilevel)
  use amr_commons
  use hydro_commons
  use mpi_mod
  use rb_b200
  implicit none
#ifndef WITHOUTMPI
  integer::info
  real(kind=8),dimension(3)::comm_buffin,comm_buffout
#endif
  integer::ilevel
  real(c_double)::dt_loc,mass_loc,ekin_loc,eint_loc
  real(kind=8)::mass_all,ekin_all,eint_all,dt_all
  if(numbtot(1,ilevel)==0)return
  call rb_b200_device
  dt_loc=dtnew(ilevel)
  call rb_b200_check(rb_courant_fine(rb_ctx, int(ilevel, c_int), dt_loc, mass_loc, ekin_loc, eint_loc), &
       & 'courant_fine')
#ifndef WITHOUTMPI
  comm_buffin(1)=mass_loc
  comm_buffin(2)=ekin_loc
  comm_buffin(3)=eint_loc
  call MPI_ALLREDUCE(comm_buffin,comm_buffout,3,MPI_DOUBLE_PRECISION,MPI_SUM,MPI_COMM_WORLD,info)
  call MPI_ALLREDUCE(dt_loc,dt_all,1,MPI_DOUBLE_PRECISION,MPI_MIN,MPI_COMM_WORLD,info)
  mass_all=comm_buffout(1)
  ekin_all=comm_buffout(2)
  eint_all=comm_buffout(3)
#else
  mass_all=mass_loc
  ekin_all=ekin_loc
  eint_all=eint_loc
  dt_all=dt_loc
#endif
  mass_tot=mass_tot+mass_all
  ekin_tot=ekin_tot+ekin_all
  eint_tot=eint_tot+eint_all
  dtnew(ilevel)=MIN(dtnew(ilevel),dt_all)
end subroutine courant_fine
