!###########################################################
! rb_b200: ISO_C_BINDING layer between RAMSES's hydro call sites and the
! B200 library (include/ramses_b200.h). The Fortran host keeps its arrays
! (son, father, nbor, active, uold) and its &HYDRO_PARAMS namelist; this
! module mirrors them on the GPU and converts the namelist strings to codes.
!
! Residency protocol: the device copy of uold stays authoritative across
! hydro calls. The library knows which copy is newer (every device call that
! writes uold makes it the device's); the host says when it changed the
! tree or wrote uold:
!   rb_b200_device : before a device hydro call (courant_fine, set_unew,
!                    godunov_fine, set_uold, upload_fine, make_boundary_hydro,
!                    hydro_flag): re-synchronises the tree when the host
!                    changed it (the library prolongs the new octs on the
!                    device), uploads uold only when the host copy is newer;
!   rb_b200_host   : before host code reads uold (dump_all, load_balance,
!                    flag criteria evaluated on the host): downloads only when
!                    the device copy is newer;
!   rb_b200_tree_changed / rb_b200_host_wrote : called by the wrappers of
!                    refine_fine, load_balance and defrag (wrap_b200.f90,
!                    linked with -Wl,--wrap).
! unew lives on the device only between set_unew and set_uold.
!###########################################################
module rb_b200
  use iso_c_binding
  implicit none

  type, bind(c) :: rb_hydro_params_t
     real(c_double) :: gamma, smallr, smallc, courant_factor, slope_theta
     integer(c_int32_t) :: riemann, slope_type, scheme, interpol_var, interpol_type, pressure_fix
     real(c_double) :: difmag, beta_fix
     integer(c_int32_t) :: niter_riemann, pad_
  end type rb_hydro_params_t

  type, bind(c) :: rb_mesh_params_t
     integer(c_int32_t) :: nx, ny, nz, ncoarse, ngridmax, nlevelmax, levelmin, nvector
     real(c_double) :: boxlen
     integer(c_int32_t) :: nsubcycle(0:32)
     integer(c_int32_t) :: nx_loc, pad_
  end type rb_mesh_params_t

  type, bind(c) :: rb_refine_params_t
     real(c_double) :: err_grad_d, err_grad_p, err_grad_u
     real(c_double) :: floor_d, floor_u, floor_p
  end type rb_refine_params_t

  type(c_ptr), save :: rb_ctx = c_null_ptr

  interface
     integer(c_int) function rb_create(hp, mp, precision, ctx) bind(c, name='rb_create')
       import :: c_int, c_ptr, rb_hydro_params_t, rb_mesh_params_t
       type(rb_hydro_params_t), intent(in) :: hp
       type(rb_mesh_params_t), intent(in) :: mp
       integer(c_int), value :: precision
       type(c_ptr), intent(out) :: ctx
     end function rb_create
     integer(c_int) function rb_sync_tree(ctx, son, father, nbor, numbl, active) bind(c, name='rb_sync_tree')
       import :: c_int, c_ptr, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), intent(in) :: son(*), father(*), nbor(*), numbl(*), active(*)
     end function rb_sync_tree
     integer(c_int) function rb_set_boundary(ctx, nb, btype, numbb, igrid) bind(c, name='rb_set_boundary')
       import :: c_int, c_ptr, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: nb
       integer(c_int32_t), intent(in) :: btype(*), numbb(*), igrid(*)
     end function rb_set_boundary
     integer(c_int) function rb_make_boundary_hydro(ctx, ilevel) bind(c, name='rb_make_boundary_hydro')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: ilevel
     end function rb_make_boundary_hydro
     integer(c_int) function rb_upload_state(ctx, uold) bind(c, name='rb_upload_state')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: uold(*)
     end function rb_upload_state
     integer(c_int) function rb_download_state(ctx, uold) bind(c, name='rb_download_state')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(inout) :: uold(*)
     end function rb_download_state
     integer(c_int) function rb_set_unew(ctx, ilevel) bind(c, name='rb_set_unew')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: ilevel
     end function rb_set_unew
     integer(c_int) function rb_set_uold(ctx, ilevel) bind(c, name='rb_set_uold')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: ilevel
     end function rb_set_uold
     integer(c_int) function rb_upload_fine(ctx, ilevel) bind(c, name='rb_upload_fine')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: ilevel
     end function rb_upload_fine
     integer(c_int) function rb_godunov_fine(ctx, ilevel, dt) bind(c, name='rb_godunov_fine')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: ilevel
       real(c_double), value :: dt
     end function rb_godunov_fine
     integer(c_int) function rb_courant_fine(ctx, ilevel, dt, mass, ekin, eint) bind(c, name='rb_courant_fine')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: ilevel
       real(c_double), intent(inout) :: dt
       real(c_double), intent(out) :: mass, ekin, eint
     end function rb_courant_fine
     integer(c_int) function rb_hydro_flag(ctx, ilevel, rp, flag1, nflag_added) bind(c, name='rb_hydro_flag')
       import :: c_int, c_int32_t, c_int64_t, c_ptr, rb_refine_params_t
       type(c_ptr), value :: ctx
       integer(c_int), value :: ilevel
       type(rb_refine_params_t), intent(in) :: rp
       integer(c_int32_t), dimension(*) :: flag1
       integer(c_int64_t) :: nflag_added
     end function rb_hydro_flag
     integer(c_int) function rb_note_tree_changed(ctx) bind(c, name='rb_note_tree_changed')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function rb_note_tree_changed
     integer(c_int) function rb_note_host_state_written(ctx) bind(c, name='rb_note_host_state_written')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function rb_note_host_state_written
     integer(c_int) function rb_tree_needs_sync(ctx, needed) bind(c, name='rb_tree_needs_sync')
       import :: c_int, c_ptr, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), intent(out) :: needed
     end function rb_tree_needs_sync
     integer(c_int) function rb_ensure_device(ctx, son, father, nbor, numbl, active, nb, btype, numbb, bgrid, &
          & uold) bind(c, name='rb_ensure_device')
       import :: c_int, c_ptr, c_int32_t, c_double
       type(c_ptr), value :: ctx
       integer(c_int32_t), intent(in) :: son(*), father(*), nbor(*), numbl(*), active(*)
       integer(c_int32_t), value :: nb
       integer(c_int32_t), intent(in) :: btype(*), numbb(*), bgrid(*)
       real(c_double), intent(in) :: uold(*)
     end function rb_ensure_device
     integer(c_int) function rb_ensure_host(ctx, uold) bind(c, name='rb_ensure_host')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(inout) :: uold(*)
     end function rb_ensure_host
     type(c_ptr) function rb_last_error() bind(c, name='rb_last_error')
       import :: c_ptr
     end function rb_last_error
  end interface

contains

  subroutine rb_b200_check(rc, where)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: where
    character(kind=c_char), pointer :: msg(:)
    integer :: n
    if (rc == 0) return
    call c_f_pointer(rb_last_error(), msg, [1024])
    n = 0
    do while (n < 1024)
       if (msg(n+1) == c_null_char) exit
       n = n + 1
    end do
    write(*,*) 'rb_b200: ', where, ' failed with status ', rc, ': ', msg(1:n)
    call clean_stop
  end subroutine rb_b200_check

  subroutine rb_b200_init
    use amr_commons
    use hydro_commons
    type(rb_hydro_params_t) :: hp
    type(rb_mesh_params_t) :: mp
    integer :: l
    if (c_associated(rb_ctx)) return
    if (no_inflow) then
       write(*,*) 'rb_b200: no_inflow is not supported by the device boundary fill'
       call clean_stop
    end if
    hp%gamma = gamma; hp%smallr = smallr; hp%smallc = smallc
    hp%courant_factor = courant_factor; hp%slope_theta = slope_theta
    hp%slope_type = slope_type; hp%scheme = 0; hp%pressure_fix = 0
    hp%interpol_var = interpol_var; hp%interpol_type = interpol_type; hp%difmag = difmag
    hp%beta_fix = beta_fix
    hp%niter_riemann = niter_riemann; hp%pad_ = 0
    if (scheme == 'plmde') hp%scheme = 1
    if (scheme /= 'muscl' .and. scheme /= 'plmde') hp%scheme = -1
    if (pressure_fix) hp%pressure_fix = 1
    hp%riemann = 0
    if (riemann == 'llf') hp%riemann = 1
    if (riemann == 'hll') hp%riemann = 2
    if (riemann == 'hllc') hp%riemann = 3
    if (riemann == 'acoustic') hp%riemann = 4
    if (riemann == 'exact') hp%riemann = 5
    mp%nx = nx; mp%ny = ny; mp%nz = nz; mp%ncoarse = ncoarse; mp%ngridmax = ngridmax
    mp%nlevelmax = nlevelmax; mp%levelmin = levelmin; mp%nvector = nvector
    mp%boxlen = boxlen
    mp%nx_loc = icoarse_max - icoarse_min + 1; mp%pad_ = 0
    mp%nsubcycle = 2
    do l = 1, min(nlevelmax, 32)
       mp%nsubcycle(l) = nsubcycle(l)
    end do
    call rb_b200_check(rb_create(hp, mp, 0_c_int, rb_ctx), 'rb_create')
  end subroutine rb_b200_init

  ! before a device hydro call: the tree when the host changed it (the tree
  ! arrays are gathered only then), uold when the host copy is newer
  subroutine rb_b200_device
    use amr_commons
    use hydro_commons
    integer(c_int32_t), allocatable :: numbl(:), act(:), numbb(:,:), bgrid(:), btype(:)
    integer(c_int32_t) :: need, dummy(1)
    integer :: l, i, n, ib
    call rb_b200_init
    call rb_b200_check(rb_tree_needs_sync(rb_ctx, need), 'rb_tree_needs_sync')
    if (need == 0) then
       dummy = 0
       call rb_b200_check(rb_ensure_device(rb_ctx, son, father, nbor, dummy, dummy, 0_c_int32_t, dummy, &
            & dummy, dummy, uold), 'rb_ensure_device')
       return
    end if
    allocate(numbl(nlevelmax))
    n = 0
    do l = 1, nlevelmax
       numbl(l) = active(l)%ngrid
       n = n + active(l)%ngrid
    end do
    allocate(act(max(n, 1)))
    n = 0
    do l = 1, nlevelmax
       do i = 1, active(l)%ngrid
          n = n + 1
          act(n) = active(l)%igrid(i)
       end do
    end do
    ! physical boundaries: boundary(ibound,ilevel)%igrid, level by level
    allocate(numbb(max(nboundary, 1), nlevelmax))
    n = 0
    do l = 1, nlevelmax
       do ib = 1, nboundary
          numbb(ib, l) = boundary(ib, l)%ngrid
          n = n + boundary(ib, l)%ngrid
       end do
    end do
    allocate(bgrid(max(n, 1)), btype(max(nboundary, 1)))
    btype = 0
    if (nboundary > 0) btype(1:nboundary) = boundary_type(1:nboundary)
    n = 0
    do l = 1, nlevelmax
       do ib = 1, nboundary
          do i = 1, boundary(ib, l)%ngrid
             n = n + 1
             bgrid(n) = boundary(ib, l)%igrid(i)
          end do
       end do
    end do
    call rb_b200_check(rb_ensure_device(rb_ctx, son, father, nbor, numbl, act, int(nboundary, c_int32_t), &
         & btype, numbb, bgrid, uold), 'rb_ensure_device')
    deallocate(numbl, act, numbb, bgrid, btype)
  end subroutine rb_b200_device

  ! before host code reads uold
  subroutine rb_b200_host
    use hydro_commons
    if (.not. c_associated(rb_ctx)) return
    call rb_b200_check(rb_ensure_host(rb_ctx, uold), 'rb_ensure_host')
  end subroutine rb_b200_host

  ! the host changed son/father/nbor/active or the boundary lists
  subroutine rb_b200_tree_changed
    call rb_b200_init
    call rb_b200_check(rb_note_tree_changed(rb_ctx), 'rb_note_tree_changed')
  end subroutine rb_b200_tree_changed

  ! the host wrote uold
  subroutine rb_b200_host_wrote
    call rb_b200_init
    call rb_b200_check(rb_note_host_state_written(rb_ctx), 'rb_note_host_state_written')
  end subroutine rb_b200_host_wrote

end module rb_b200
