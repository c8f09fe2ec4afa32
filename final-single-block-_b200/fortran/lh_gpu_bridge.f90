! iso_c_binding bridge from the LittleHarsh Fortran driver to the B200
! engine (include/lh_gpu.h).  The Fortran main loop keeps its arrays and
! its set-up.  This module holds the bind(C) interfaces, the context and the
! whole-substep wrappers (gpu_*); lh_gpu_surface.f90 builds on it the
! external subroutines with the reference's own names and argument lists
! (four_to_phys_u, phys_to_four_du, LUsolU, LUsolP, LU_buildP, solveU,
! solveP), so littleharsh.f90 and FOU3D.f90 call sites stay as they are.  A
! non-zero status stops the run the way the reference stops on bad input
! (start.f90:203-204).
!
! Build (Fortran compiler and the engine library required; the declaration
! module of the reference first):
!   mpif90 -c declaration.f90 lh_gpu_bridge.f90 lh_gpu_surface.f90
!   mpif90 -o littleharsh lh_gpu_surface.o lh_gpu_bridge.o <reference objects> \
!          -Wl,--allow-multiple-definition \
!          -L<repo>/final-single-block-_b200/build -llh_gpu -lcudart
module lh_gpu_bridge
  use iso_c_binding
  implicit none

  type, bind(C) :: lh_grid_desc
    integer(c_int)  :: Nx, Nz, ny
    real(c_double)  :: Re, alp, bet, mpgx
    integer(c_int)  :: flag_ctpress, grid_type
    real(c_double)  :: dyq
    integer(c_int)  :: ppp
    real(c_double)  :: gamma
    integer(c_int)  :: dt_mode
    real(c_double)  :: CFL, dt
  end type lh_grid_desc

  interface
    integer(c_int) function lh_ctx_create(desc, ctx) bind(C, name="lh_ctx_create")
      import :: c_int, c_ptr, lh_grid_desc
      type(lh_grid_desc), intent(in) :: desc
      type(c_ptr), intent(out)       :: ctx
    end function
    integer(c_int) function lh_ctx_destroy(ctx) bind(C, name="lh_ctx_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function lh_upload_state(ctx, u1, u2, u3, p) bind(C, name="lh_upload_state")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: ctx
      complex(c_double_complex), intent(in) :: u1(*), u2(*), u3(*), p(*)
    end function
    integer(c_int) function lh_download_state(ctx, u1, u2, u3, p) bind(C, name="lh_download_state")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: ctx
      complex(c_double_complex), intent(out) :: u1(*), u2(*), u3(*), p(*)
    end function
    integer(c_int) function lh_substep(ctx, kRK) bind(C, name="lh_substep")
      import :: c_int, c_ptr
      type(c_ptr), value    :: ctx
      integer(c_int), value :: kRK
    end function
    integer(c_int) function lh_step(ctx, nsteps) bind(C, name="lh_step")
      import :: c_int, c_ptr
      type(c_ptr), value    :: ctx
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function lh_get_scalars(ctx, t, dt, iter, mpgx, qx) bind(C, name="lh_get_scalars")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: t, dt, mpgx, qx
      integer(c_int), intent(out) :: iter
    end function
    integer(c_int) function lh_four_to_phys(ctx, planes, n) bind(C, name="lh_four_to_phys")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value    :: ctx
      real(c_double)        :: planes(*)
      integer(c_int), value :: n
    end function
    integer(c_int) function lh_phys_to_four(ctx, planes, n) bind(C, name="lh_phys_to_four")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value    :: ctx
      real(c_double)        :: planes(*)
      integer(c_int), value :: n
    end function
    integer(c_int) function lh_lusolu(ctx, grid, kRK, dt, rhs, u) bind(C, name="lh_lusolu")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value    :: ctx
      integer(c_int), value :: grid, kRK
      real(c_double), value :: dt
      complex(c_double_complex), intent(in)  :: rhs(*)
      complex(c_double_complex), intent(out) :: u(*)
    end function
    integer(c_int) function lh_lusolp(ctx, x) bind(C, name="lh_lusolp")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: ctx
      complex(c_double_complex) :: x(*)
    end function
    integer(c_int) function lh_spectra_accumulate(ctx) bind(C, name="lh_spectra_accumulate")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function lh_stats_accumulate(ctx) bind(C, name="lh_stats_accumulate")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function lh_pressure_snapshot(ctx) bind(C, name="lh_pressure_snapshot")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function lh_omega_x(ctx, out, cap) bind(C, name="lh_omega_x")
      import :: c_int, c_ptr, c_double, c_size_t
      type(c_ptr), value       :: ctx
      real(c_double)           :: out(*)
      integer(c_size_t), value :: cap
    end function
    integer(c_int) function lh_get_stats(ctx, out, cap, count) bind(C, name="lh_get_stats")
      import :: c_int, c_ptr, c_double, c_size_t
      type(c_ptr), value       :: ctx
      real(c_double)           :: out(*)
      integer(c_size_t), value :: cap
      integer(c_int)           :: count
    end function
    integer(c_int) function lh_get_spectra(ctx, which, out, cap, count) bind(C, name="lh_get_spectra")
      import :: c_int, c_ptr, c_double, c_size_t
      type(c_ptr), value       :: ctx
      integer(c_int), value    :: which
      real(c_double)           :: out(*)
      integer(c_size_t), value :: cap
      integer(c_int)           :: count
    end function
    integer(c_int) function lh_synchronize(ctx) bind(C, name="lh_synchronize")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function lh_error_div(ctx, err) bind(C, name="lh_error_div")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: err
    end function
    integer(c_int) function lh_tridiag_factor(ctx, grid, kRK, dt, a, cap) bind(C, name="lh_tridiag_factor")
      import :: c_int, c_ptr, c_double, c_size_t
      type(c_ptr), value       :: ctx
      integer(c_int), value    :: grid, kRK
      real(c_double), value    :: dt
      real(c_double)           :: a(*)
      integer(c_size_t), value :: cap
    end function
    integer(c_int) function lh_tridiag_solve(ctx, grid, a, x) bind(C, name="lh_tridiag_solve")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value    :: ctx
      integer(c_int), value :: grid
      real(c_double), intent(in) :: a(*)
      complex(c_double_complex)  :: x(*)
    end function
    integer(c_int) function lh_set_dg(ctx, a) bind(C, name="lh_set_dg")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: a(*)
    end function
    integer(c_int) function lh_set_scalars(ctx, t, iter, mpgx) bind(C, name="lh_set_scalars")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value    :: ctx
      real(c_double), value :: t, mpgx
      integer(c_int), value :: iter
    end function
  end interface

  type(c_ptr), save :: gpu_ctx = c_null_ptr

contains

  subroutine gpu_check(rc, where)
    integer(c_int), intent(in) :: rc
    character(*), intent(in)   :: where
    if (rc /= 0) then
      write(*,*) 'lh_gpu error', rc, 'in ', where
      stop
    end if
  end subroutine

  ! After start(): describe the instance from the declaration module.
  subroutine gpu_start()
    use declaration
    type(lh_grid_desc) :: d
    d%Nx = Nspec_x; d%Nz = Nspec_z; d%ny = nyv + 2
    d%Re = Re; d%alp = alp; d%bet = bet; d%mpgx = mpgx
    d%flag_ctpress = flag_ctpress
    d%grid_type = 0; d%dyq = dyq; d%ppp = ppp; d%gamma = 0d0
    d%dt_mode = 0; d%CFL = CFL; d%dt = 0d0
    call gpu_check(lh_ctx_create(d, gpu_ctx), 'lh_ctx_create')
  end subroutine

  ! The context, created from the declaration module on first use by the
  ! reference-named routines of lh_gpu_surface.f90.
  subroutine gpu_ensure()
    if (.not. c_associated(gpu_ctx)) call gpu_start()
  end subroutine

  ! Column count and row counts of the declaration module (np = 1).
  integer(c_size_t) function gpu_cols()
    use declaration, only: columns_num
    gpu_cols = int(columns_num(0), c_size_t)
  end function

  ! After getini(): hand the initial state to the device, with the t, iter
  ! and mpgx getini left in the declaration module (zero / the input deck's
  ! for flag_init = 1, the restart file's for flag_init = 2,
  ! start.f90:1268-1282).
  subroutine gpu_getini(u1, u2, u3, p)
    use declaration, only: t, iter, mpgx
    complex(8), intent(in) :: u1(*), u2(*), u3(*), p(*)
    call gpu_check(lh_upload_state(gpu_ctx, u1, u2, u3, p), 'lh_upload_state')
    call gpu_check(lh_set_scalars(gpu_ctx, t, int(iter, c_int), mpgx), 'lh_set_scalars')
  end subroutine

  ! Refresh the declaration module's t, dt, iter, mpgx and Qx from the
  ! device (the main loop's do while (t < maxt) test, hist output).
  subroutine gpu_scalars()
    use declaration, only: t, dt, iter, mpgx, Qx
    integer(c_int) :: it
    call gpu_check(lh_get_scalars(gpu_ctx, t, dt, it, mpgx, Qx), 'lh_get_scalars')
    iter = it
  end subroutine

  ! error(div) (littleharsh.f90:370-409): max |div| of the current state
  subroutine gpu_error(err_out)
    real(8), intent(out) :: err_out
    call gpu_check(lh_error_div(gpu_ctx, err_out), 'lh_error_div')
  end subroutine

  ! The engine uses the caller's DG (start.f90:636) as its pressure factors.
  subroutine gpu_set_dg(DG_in)
    real(8), intent(in) :: DG_in(*)
    call gpu_check(lh_set_dg(gpu_ctx, DG_in), 'lh_set_dg')
  end subroutine

  ! Replaces the body of the substep loop, littleharsh.f90:169-220
  ! (RHS0_u1/2/3, nonlinear, solveU x3, meanflow_ctU, solveP, v_corr).
  subroutine gpu_substep(kRK_in)
    integer, intent(in) :: kRK_in
    call gpu_check(lh_substep(gpu_ctx, int(kRK_in, c_int)), 'lh_substep')
  end subroutine

  ! Bring the state back for record_out / stats on output steps.
  subroutine gpu_fetch(u1, u2, u3, p)
    complex(8), intent(out) :: u1(*), u2(*), u3(*), p(*)
    call gpu_check(lh_download_state(gpu_ctx, u1, u2, u3, p), 'lh_download_state')
  end subroutine

  ! spectra(u1,u2,u2_itp,u3,p,myid) at a flagged step (FOU3D.f90:137-141):
  ! the accumulation stays on the device
  subroutine gpu_spectra()
    call gpu_check(lh_spectra_accumulate(gpu_ctx), 'lh_spectra_accumulate')
  end subroutine

  ! Bring the accumulated spectra back before write_spect (spectra.f90)
  ! The capacities are the sizes of spU/spW/spUV (jlim(:,ugrid) rows), spV
  ! (vgrid rows) and spP (pgrid rows) times the columns (start.f90:641-645).
  subroutine gpu_fetch_spectra(spU_, spV_, spW_, spUV_, spP_)
    use declaration, only: nyu, nyv
    real(8) :: spU_(*), spV_(*), spW_(*), spUV_(*), spP_(*)
    integer(c_int) :: n, cnt
    integer(c_size_t) :: cu, cv, cp
    cu = int(nyu + 2, c_size_t) * gpu_cols()
    cv = int(nyv + 2, c_size_t) * gpu_cols()
    cp = int(nyu, c_size_t) * gpu_cols()
    n = lh_get_spectra(gpu_ctx, 0_c_int, spU_, cu, cnt)
    if (n < 0) call gpu_check(n, 'lh_get_spectra')
    n = lh_get_spectra(gpu_ctx, 1_c_int, spV_, cv, cnt)
    if (n < 0) call gpu_check(n, 'lh_get_spectra')
    n = lh_get_spectra(gpu_ctx, 2_c_int, spW_, cu, cnt)
    if (n < 0) call gpu_check(n, 'lh_get_spectra')
    n = lh_get_spectra(gpu_ctx, 3_c_int, spUV_, cu, cnt)
    if (n < 0) call gpu_check(n, 'lh_get_spectra')
    n = lh_get_spectra(gpu_ctx, 4_c_int, spP_, cp, cnt)
    if (n < 0) call gpu_check(n, 'lh_get_spectra')
  end subroutine

  ! stats(myid,status,ierr) at the flagst steps (FOU3D.f90:307-341), with
  ! omega_x formed on the device
  subroutine gpu_stats()
    call gpu_check(lh_stats_accumulate(gpu_ctx), 'lh_stats_accumulate')
  end subroutine

  ! ppPL = 0; modes_to_planes_UVP(ppPL, p, ...) on output steps (FOU3D.f90:149-152)
  subroutine gpu_pressure_planes()
    call gpu_check(lh_pressure_snapshot(gpu_ctx), 'lh_pressure_snapshot')
  end subroutine

  ! The plane sums acc(0:nyu+1, 13) = Um U2m Vm V2m Wm W2m UVm UWm VWm Pm P2m
  ! wxm wx2m, with the number of accumulations (istat)
  subroutine gpu_fetch_stats(acc, nstat_done)
    use declaration, only: nyu
    real(8) :: acc(*)
    integer :: nstat_done
    integer(c_int) :: n, cnt
    n = lh_get_stats(gpu_ctx, acc, 13_c_size_t * int(nyu + 2, c_size_t), cnt)
    if (n < 0) call gpu_check(n, 'lh_get_stats')
    nstat_done = cnt
  end subroutine

  ! omega_x at the v faces, wx(Nspec_x+2, Nspec_z, 0:nyu+1) in physical space
  subroutine gpu_omega_x(wx_out)
    use declaration, only: nyu, Nspec_x, Nspec_z
    real(8) :: wx_out(*)
    integer(c_int) :: n
    n = lh_omega_x(gpu_ctx, wx_out, int(nyu + 2, c_size_t) * int(Nspec_z, c_size_t) * int(Nspec_x + 2, c_size_t))
    if (n < 0) call gpu_check(n, 'lh_omega_x')
  end subroutine

  subroutine gpu_finalize()
    if (c_associated(gpu_ctx)) call gpu_check(lh_ctx_destroy(gpu_ctx), 'lh_ctx_destroy')
    gpu_ctx = c_null_ptr
  end subroutine

end module lh_gpu_bridge
