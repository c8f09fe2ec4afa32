! The reference's own subroutine surface over the B200 engine: external
! subroutines with the names and argument lists littleharsh.f90, FOU3D.f90
! and start.f90 call, so those call sites compile unchanged.  Module
! globals the reference reads inside these routines (kRK, dt, dti, aRK,
! bRK, jlim, columns_num) are forwarded to the C ABI explicitly.  Link this
! object before the reference's objects with -Wl,--allow-multiple-definition
! so its definitions are the ones used (GNU ld keeps the first), and build
! the reference without cross-procedure inlining (gfortran's default -O0,
! or -fno-inline) so FOU3D.f90's calls of four_to_phys_u / phys_to_four_du
! go through the symbols.  The engine context is created from the
! declaration module on the first call (gpu_ensure).
!
! Replaced (reference file:line):
!   four_to_phys_u(u1,u2,u3)          FOU3D.f90:653-679
!   four_to_phys_du(du)               FOU3D.f90:681-697
!   phys_to_four_du(duPL)             FOU3D.f90:1654-1672
!   LUsolU(u,rhsu,a,grid,myid)        tridLU_3D.f90:38-94
!   LUsolP(x,myid,nystart,nyend)      tridLU_3D.f90:98-132
!   LU_buildP(nystart,nyend,myid,a)   tridLU_3D.f90:224-297 (with LU_decP)
!   solveU(u,du,grid,a_grid,myid)     littleharsh.f90:863-894
!   solveP(p,psi,u1,u2,u3,div,myid)   littleharsh.f90:626-680

subroutine four_to_phys_u(u1, u2, u3)
  use declaration, only: Ngal_x, Ngal_z
  use lh_gpu_bridge
  implicit none
  real(8) u1(Ngal_x+2, Ngal_z), u2(Ngal_x+2, Ngal_z), u3(Ngal_x+2, Ngal_z)
  call gpu_ensure()
  ! lh_four_to_phys zeroes row Ngal_z/2+1 first, as four_to_phys_u does
  call gpu_check(lh_four_to_phys(gpu_ctx, u1, 1_c_int), 'lh_four_to_phys')
  call gpu_check(lh_four_to_phys(gpu_ctx, u2, 1_c_int), 'lh_four_to_phys')
  call gpu_check(lh_four_to_phys(gpu_ctx, u3, 1_c_int), 'lh_four_to_phys')
end subroutine

subroutine four_to_phys_du(du)
  use declaration, only: Ngal_x, Ngal_z
  use lh_gpu_bridge
  implicit none
  real(8) du(Ngal_x+2, Ngal_z)
  call gpu_ensure()
  call gpu_check(lh_four_to_phys(gpu_ctx, du, 1_c_int), 'lh_four_to_phys')
end subroutine

subroutine phys_to_four_du(duPL)
  use declaration, only: Ngal_x, Ngal_z
  use lh_gpu_bridge
  implicit none
  real(8) duPL(Ngal_x+2, Ngal_z)
  call gpu_ensure()
  ! lh_phys_to_four zeroes the oddball row Ngal_z/2+1 afterwards
  call gpu_check(lh_phys_to_four(gpu_ctx, duPL, 1_c_int), 'lh_phys_to_four')
end subroutine

! The a(3,:) work array of the reference (the factors of the last column)
! is not filled: no caller reads it after LUsolU returns.
subroutine LUsolU(u, rhsu, a, grid, myid)
  use declaration, only: jlim, columns_num, kRK, dt
  use lh_gpu_bridge
  implicit none
  integer grid, myid
  complex(8) :: u   (jlim(1,grid):jlim(2,grid), columns_num(myid))
  complex(8) :: rhsu(jlim(1,grid):jlim(2,grid), columns_num(myid))
  real(8)    :: a(3, jlim(1,grid):jlim(2,grid))
  call gpu_ensure()
  call gpu_check(lh_lusolu(gpu_ctx, int(grid, c_int), int(kRK, c_int), dt, rhsu, u), 'lh_lusolu')
end subroutine

subroutine LUsolP(x, myid, nystart, nyend)
  use declaration, only: jlim, columns_num, pgrid
  use lh_gpu_bridge
  implicit none
  integer myid, nystart, nyend
  complex(8) x(nystart:nyend, columns_num(myid))
  if (nystart /= jlim(1,pgrid) .or. nyend /= jlim(2,pgrid)) then
    write(*,*) 'LUsolP: the engine solves rows jlim(1:2,pgrid) only'
    stop
  end if
  call gpu_ensure()
  call gpu_check(lh_lusolp(gpu_ctx, x), 'lh_lusolp')
end subroutine

! DG as the engine forms it (LU_buildP + LU_decP restated in its set-up):
! start() keeps a host copy equal to the factors the device solves with.
subroutine LU_buildP(nystart, nyend, myid, a)
  use declaration, only: jlim, columns_num, pgrid
  use lh_gpu_bridge
  implicit none
  integer myid, nystart, nyend
  real(8) a(3, jlim(1,pgrid):jlim(2,pgrid), columns_num(myid))
  integer(c_int) :: n
  call gpu_ensure()
  n = lh_tridiag_factor(gpu_ctx, 3_c_int, 1_c_int, 0d0, a, int(size(a), c_size_t))
  if (n < 0) call gpu_check(n, 'lh_tridiag_factor')
end subroutine

subroutine solveU(u, du, grid, a_grid, myid)
  use declaration, only: jlim, columns_num, dt
  implicit none
  integer grid, myid, column, j
  complex(8) :: u ( jlim(1,grid):jlim(2,grid), columns_num(myid) )
  complex(8) :: du( jlim(1,grid):jlim(2,grid), columns_num(myid) )
  real(8)    :: a_grid(3, jlim(1,grid):jlim(2,grid))
  ! the right-hand side as littleharsh.f90:878-890 forms it, then the device solve
  do column = 1, columns_num(myid)
    du(jlim(1,grid), column) = 0d0
    do j = jlim(1,grid)+1, jlim(2,grid)-1
      du(j, column) = u(j, column) + dt*(du(j, column))
    end do
    du(jlim(2,grid), column) = 0d0
  end do
  call LUsolU(u, du, a_grid, grid, myid)
end subroutine

subroutine solveP(p, psi, u1, u2, u3, div, myid)
  use declaration, only: jlim, columns_num, ugrid, vgrid, pgrid, kRK, dti, aRK, bRK
  implicit none
  integer myid, column, j
  complex(8) :: u1 ( jlim(1,ugrid):jlim(2,ugrid), columns_num(myid) )
  complex(8) :: u2 ( jlim(1,vgrid):jlim(2,vgrid), columns_num(myid) )
  complex(8) :: u3 ( jlim(1,ugrid):jlim(2,ugrid), columns_num(myid) )
  complex(8) :: p  ( jlim(1,pgrid):jlim(2,pgrid), columns_num(myid) )
  complex(8) :: psi( jlim(1,pgrid):jlim(2,pgrid), columns_num(myid) )
  complex(8) :: div( jlim(1,pgrid):jlim(2,pgrid), columns_num(myid) )
  real(8) :: dtirk
  dtirk = dti/(aRK(kRK)+bRK(kRK))
  ! divergence (littleharsh.f90:242-278) stays the reference's routine
  call divergence(div, u1, u2, u3, myid)
  do column = 1, columns_num(myid)
    do j = jlim(1,pgrid), jlim(2,pgrid)
      psi(j, column) = dtirk*div(j, column)
    end do
  end do
  if (myid == 0) psi(jlim(1,pgrid), 1) = 0d0
  call LUsolP(psi, myid, jlim(1,pgrid), jlim(2,pgrid))
  do column = 1, columns_num(myid)
    do j = jlim(1,pgrid), jlim(2,pgrid)
      p(j, column) = p(j, column) + psi(j, column)
    end do
  end do
end subroutine
