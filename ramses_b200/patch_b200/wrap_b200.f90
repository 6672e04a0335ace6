!###########################################################
! Link-time wrappers (GNU ld --wrap, added by this directory's Makefile) of
! the reference routines that change the tree, read or write uold on the
! host, or restrict it, so that the device copy of uold stays authoritative
! without patching their source files. A call from another object file to
! refine_fine_ reaches __wrap_refine_fine_, which calls the original
! through __real_refine_fine_.
!   refine_fine  (amr/refine_utils.f90:332-585): the tree changes; the new
!                octs' state is prolonged on the device at the next device
!                call, the host's own interpolation (on a stale uold) is
!                never uploaded
!   load_balance, defrag (amr/load_balance.f90:5-280, 993-1608): move octs
!                and their uold on the host: the host copy is refreshed
!                first, then both the tree and uold are host-written
!   dump_all     (amr/output_amr.f90:5-206): reads uold: refreshed first
!   flag_fine    (amr/flag_utils.f90:57-106): the mass criterion (m_refine)
!                reads uold on the host: refreshed first when it is on
!   upload_fine  (hydro/interpol_hydro.f90:5-68): restriction on the device
!###########################################################
subroutine wrap_refine_fine(ilevel) bind(c, name='__wrap_refine_fine_')
  use rb_b200
  implicit none
  integer(c_int) :: ilevel
  interface
     subroutine real_refine_fine(ilevel) bind(c, name='__real_refine_fine_')
       import :: c_int
       integer(c_int) :: ilevel
     end subroutine real_refine_fine
  end interface
  call real_refine_fine(ilevel)
  call rb_b200_tree_changed
end subroutine wrap_refine_fine

subroutine wrap_load_balance() bind(c, name='__wrap_load_balance_')
  use rb_b200
  implicit none
  interface
     subroutine real_load_balance() bind(c, name='__real_load_balance_')
     end subroutine real_load_balance
  end interface
  call rb_b200_host
  call real_load_balance()
  call rb_b200_tree_changed
  call rb_b200_host_wrote
end subroutine wrap_load_balance

subroutine wrap_defrag() bind(c, name='__wrap_defrag_')
  use rb_b200
  implicit none
  interface
     subroutine real_defrag() bind(c, name='__real_defrag_')
     end subroutine real_defrag
  end interface
  call rb_b200_host
  call real_defrag()
  call rb_b200_tree_changed
  call rb_b200_host_wrote
end subroutine wrap_defrag

subroutine wrap_dump_all() bind(c, name='__wrap_dump_all_')
  use rb_b200
  implicit none
  interface
     subroutine real_dump_all() bind(c, name='__real_dump_all_')
     end subroutine real_dump_all
  end interface
  call rb_b200_host
  call real_dump_all()
end subroutine wrap_dump_all

subroutine wrap_flag_fine(ilevel, icount) bind(c, name='__wrap_flag_fine_')
  use amr_commons
  use rb_b200
  implicit none
  integer(c_int) :: ilevel, icount
  interface
     subroutine real_flag_fine(ilevel, icount) bind(c, name='__real_flag_fine_')
       import :: c_int
       integer(c_int) :: ilevel, icount
     end subroutine real_flag_fine
  end interface
  if (any(m_refine(1:nlevelmax) > -1.0d0)) call rb_b200_host
  call real_flag_fine(ilevel, icount)
end subroutine wrap_flag_fine

subroutine wrap_upload_fine(ilevel) bind(c, name='__wrap_upload_fine_')
  use amr_commons
  use rb_b200
  implicit none
  integer(c_int) :: ilevel
  if (ilevel == nlevelmax) return
  if (numbtot(1, ilevel) == 0) return
  call rb_b200_device
  call rb_b200_check(rb_upload_fine(rb_ctx, int(ilevel, c_int)), 'upload_fine')
end subroutine wrap_upload_fine
