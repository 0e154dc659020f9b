! ddcosmo_gpu.f90 -- Fortran drop-in for the reference's ddCOSMO interface.
!
! Provides `module ddcosmo` with the public variables and routines that the
! reference's host code uses (ddcosmo.f90:87-127 and main.f90:129-292), and
! the external routines `cosmo` (cosmo.f90:1), `forces_dd` (forces_dd.f90:1),
! `mkrhs` (mkrhs.f90:1) and `efld` (efld.f90:1), all implemented by calls into
! the CUDA library libddcosmo_gpu.so through its C ABI (include/ddcosmo_gpu.h).
! A host program written against the reference (e.g. its main.f90) compiles
! unchanged against this file:
!
!   gfortran -O2 ddcosmo_gpu.f90 main.f90 -L<lib> -lddcosmo_gpu -o main.exe
!
! Module arrays that the host reads directly after ddinit (ccav, csph, ui,
! grid, w) are host copies filled by ddinit.  Errors that the reference turns
! into `stop` stop here too, after printing the library's message.
!
module ddcosmo_c
  use, intrinsic :: iso_c_binding
  implicit none
  type, bind(c) :: ddc_params
    integer(c_int)  :: lmax, ngrid, iconv, igrad
    real(c_double)  :: eps, eta
    integer(c_int)  :: iprint, max_iter, ndiis, precision, guess, device, device_pointers
    type(c_ptr)     :: stream
    integer(c_int)  :: timing, pair_solves
  end type ddc_params
  type, bind(c) :: ddc_solve_info
    integer(c_int)  :: iterations, converged, diis_restarts, refinements
    real(c_double)  :: final_norm, seconds
    real(c_double)  :: norms(256)
  end type ddc_solve_info
  interface
    integer(c_int) function ddc_default_params(p) bind(c, name='ddc_default_params')
      import :: c_int, ddc_params
      type(ddc_params), intent(out) :: p
    end function
    integer(c_int) function ddc_create(p, ctx) bind(c, name='ddc_create')
      import :: c_int, c_ptr, ddc_params
      type(ddc_params), intent(in) :: p
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function ddc_destroy(ctx) bind(c, name='ddc_destroy')
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    type(c_ptr) function ddc_last_error(ctx) bind(c, name='ddc_last_error')
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function ddc_init(ctx, n, x, y, z, r) bind(c, name='ddc_init')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      real(c_double), intent(in) :: x(*), y(*), z(*), r(*)
    end function
    integer(c_int) function ddc_sizes(ctx, nsph, ncav, nylm, ngrid) bind(c, name='ddc_sizes')
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), intent(out) :: nsph, ncav, nylm, ngrid
    end function
    integer(c_int) function ddc_get_ccav(ctx, a) bind(c, name='ddc_get_ccav')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: a(*)
    end function
    integer(c_int) function ddc_get_ui(ctx, a) bind(c, name='ddc_get_ui')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: a(*)
    end function
    integer(c_int) function ddc_get_csph(ctx, a) bind(c, name='ddc_get_csph')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: a(*)
    end function
    integer(c_int) function ddc_get_grid(ctx, g, w) bind(c, name='ddc_get_grid')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: g(*), w(*)
    end function
    integer(c_int) function ddc_mkrhs(ctx, n, q, x, y, z, ncav, ccav, phi, nylm, psi) &
        bind(c, name='ddc_mkrhs')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: n, ncav, nylm
      real(c_double), intent(in) :: q(*), x(*), y(*), z(*), ccav(*)
      real(c_double), intent(out) :: phi(*), psi(*)
    end function
    integer(c_int) function ddc_cosmo(ctx, star, cart, phi, glm, psi, sigma, esolv, info) &
        bind(c, name='ddc_cosmo')
      import :: c_int, c_ptr, c_double, ddc_solve_info
      type(c_ptr), value :: ctx
      integer(c_int), value :: star, cart
      real(c_double), intent(in) :: phi(*), glm(*), psi(*)
      real(c_double), intent(inout) :: sigma(*)
      real(c_double), intent(inout) :: esolv
      type(ddc_solve_info), intent(out) :: info
    end function
    integer(c_int) function ddc_forces_dd(ctx, phi, sigma, s, fx) bind(c, name='ddc_forces_dd')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: phi(*), sigma(*), s(*)
      real(c_double), intent(out) :: fx(*)
    end function
    integer(c_int) function ddc_mkzeta(ctx, s, zeta) bind(c, name='ddc_mkzeta')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: s(*)
      real(c_double), intent(out) :: zeta(*)
    end function
    integer(c_int) function ddc_mkxi(ctx, s, xi) bind(c, name='ddc_mkxi')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: s(*)
      real(c_double), intent(out) :: xi(*)
    end function
    integer(c_int) function ddc_efld(ctx, nsrc, src, csrc, ntrg, ctrg, ef) bind(c, name='ddc_efld')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsrc, ntrg
      real(c_double), intent(in) :: src(*), csrc(*), ctrg(*)
      real(c_double), intent(out) :: ef(*)
    end function
  end interface
end module ddcosmo_c

module ddcosmo
  use, intrinsic :: iso_c_binding
  use ddcosmo_c
  implicit none
  ! constants and control variables as in ddcosmo.f90:87-107
  integer, parameter :: ndiis = 25, iout = 6, nngmax = 100
  real*8, parameter :: zero = 0.d0, pt5 = 0.5d0, one = 1.d0, two = 2.d0, four = 4.d0
  real*8, parameter :: se = -1.0d0
  real*8 :: pi, sq2
  integer :: iprint = 0, nproc = 0, lmax = 6, ngrid = 110, iconv = 7, igrad = 0
  real*8 :: eps = 78.3553d0, eta = 0.2d0
  integer :: nsph = 0, ncav = 0, nylm = 0
  ! host copies of the module arrays the reference's host code reads
  real*8, allocatable :: csph(:,:), ccav(:,:), ui(:,:), grid(:,:), w(:), rsph(:)
  logical :: grad
  type(c_ptr), save :: ddc_handle = c_null_ptr
contains
  subroutine ddc_check(st, where)
    integer(c_int), intent(in) :: st
    character(len=*), intent(in) :: where
    character(kind=c_char), pointer :: msg(:)
    integer :: k
    if (st == 0) return
    write(iout, '(1x,a,": ddcosmo_gpu status ",i3)') where, st
    if (c_associated(ddc_handle)) then
      call c_f_pointer(ddc_last_error(ddc_handle), msg, [1024])
      k = 1
      do while (k <= 1024)
        if (msg(k) == c_null_char) exit
        k = k + 1
      end do
      write(iout, '(1x,1024a)') msg(1:k-1)
    end if
    stop
  end subroutine ddc_check

  ! ddinit (ddcosmo.f90:159): the module state lives on the GPU; the arrays
  ! that the host reads are copied back here.
  subroutine ddinit(n, x, y, z, rvdw)
    integer, intent(in) :: n
    real*8, dimension(n), intent(in) :: x, y, z, rvdw
    type(ddc_params) :: p
    integer(c_int) :: st, a, b, c, d
    pi = four*atan(one)
    sq2 = sqrt(two)
    grad = igrad /= 0
    if (c_associated(ddc_handle)) call memfree
    st = ddc_default_params(p)
    p%lmax = lmax; p%ngrid = ngrid; p%iconv = iconv; p%igrad = igrad
    p%eps = eps; p%eta = eta; p%iprint = iprint
    call ddc_check(ddc_create(p, ddc_handle), 'ddinit')
    call ddc_check(ddc_init(ddc_handle, int(n, c_int), x, y, z, rvdw), 'ddinit')
    call ddc_check(ddc_sizes(ddc_handle, a, b, c, d), 'ddinit')
    nsph = a; ncav = b; nylm = c; ngrid = d
    allocate(csph(3,nsph), ccav(3,max(ncav,1)), ui(ngrid,nsph), grid(3,ngrid), w(ngrid), &
             rsph(nsph))
    rsph = rvdw
    call ddc_check(ddc_get_csph(ddc_handle, csph), 'ddinit')
    if (ncav > 0) call ddc_check(ddc_get_ccav(ddc_handle, ccav), 'ddinit')
    call ddc_check(ddc_get_ui(ddc_handle, ui), 'ddinit')
    call ddc_check(ddc_get_grid(ddc_handle, grid, w), 'ddinit')
  end subroutine ddinit

  ! memfree (ddcosmo.f90:491)
  subroutine memfree
    integer(c_int) :: st
    if (c_associated(ddc_handle)) st = ddc_destroy(ddc_handle)
    ddc_handle = c_null_ptr
    if (allocated(csph)) deallocate(csph)
    if (allocated(ccav)) deallocate(ccav)
    if (allocated(ui)) deallocate(ui)
    if (allocated(grid)) deallocate(grid)
    if (allocated(w)) deallocate(w)
    if (allocated(rsph)) deallocate(rsph)
  end subroutine memfree

  real*8 function sprod(n, u, v)
    integer, intent(in) :: n
    real*8, dimension(n), intent(in) :: u, v
    integer :: i
    sprod = zero
    do i = 1, n
      sprod = sprod + u(i)*v(i)
    end do
  end function sprod

  ! ddmkzeta / ddmkxi (ddcosmo.f90:1758-1806)
  subroutine ddmkzeta(s, zeta)
    real*8, dimension(nylm,nsph), intent(in) :: s
    real*8, dimension(ncav), intent(inout) :: zeta
    call ddc_check(ddc_mkzeta(ddc_handle, s, zeta), 'ddmkzeta')
  end subroutine ddmkzeta
  subroutine ddmkxi(s, xi)
    real*8, dimension(nylm,nsph), intent(in) :: s
    real*8, dimension(ncav), intent(inout) :: xi
    call ddc_check(ddc_mkxi(ddc_handle, s, xi), 'ddmkxi')
  end subroutine ddmkxi

  ! printing helpers with the reference's formats (ddcosmo.f90:667-780)
  subroutine ptcart(label, ncol, icol, x)
    character(len=*), intent(in) :: label
    integer, intent(in) :: ncol, icol
    real*8, dimension(ngrid,ncol), intent(in) :: x
    integer :: ig, noff, nprt, ic, j
    if (ncol == 1) then
      write(iout,'(3x,a,1x,"(column ",i4")")') label, icol
      do ig = 1, ngrid
        write(iout,'(1x,i5,f14.8)') ig, x(ig,1)
      end do
    else
      write(iout,'(3x,a)') label
      noff = mod(ncol,5)
      nprt = max(ncol - noff,0)
      do ic = 1, nprt, 5
        write(iout,'(6x,5i14)') (j, j = ic, ic+4)
        do ig = 1, ngrid
          write(iout,'(1x,i5,5f14.8)') ig, x(ig,ic:ic+4)
        end do
      end do
      write(iout,'(6x,5i14)') (j, j = nprt+1, nprt+noff)
      do ig = 1, ngrid
        write(iout,'(1x,i5,5f14.8)') ig, x(ig,nprt+1:nprt+noff)
      end do
    end if
  end subroutine ptcart

  subroutine prtsph(label, ncol, icol, x)
    character(len=*), intent(in) :: label
    integer, intent(in) :: ncol, icol
    real*8, dimension(nylm,ncol), intent(in) :: x
    integer :: l, m, ind, noff, nprt, ic, j
    if (ncol == 1) then
      write(iout,'(3x,a,1x,"(column ",i4")")') label, icol
      do l = 0, lmax
        ind = l*l + l + 1
        do m = -l, l
          write(iout,'(1x,i3,i4,f14.8)') l, m, x(ind+m,1)
        end do
      end do
    else
      write(iout,'(3x,a)') label
      noff = mod(ncol,5)
      nprt = max(ncol - noff,0)
      do ic = 1, nprt, 5
        write(iout,'(8x,5i14)') (j, j = ic, ic+4)
        do l = 0, lmax
          ind = l*l + l + 1
          do m = -l, l
            write(iout,'(1x,i3,i4,5f14.8)') l, m, x(ind+m,ic:ic+4)
          end do
        end do
      end do
      write(iout,'(8x,5i14)') (j, j = nprt+1, nprt+noff)
      do l = 0, lmax
        ind = l*l + l + 1
        do m = -l, l
          write(iout,'(1x,i3,i4,5f14.8)') l, m, x(ind+m,nprt+1:nprt+noff)
        end do
      end do
    end if
  end subroutine prtsph
end module ddcosmo

! cosmo(star, cart, phi, glm, psi, sigma, esolv)  (cosmo.f90:1)
subroutine cosmo(star, cart, phi, glm, psi, sigma, esolv)
  use ddcosmo
  implicit none
  logical, intent(in) :: star, cart
  real*8, dimension(ncav), intent(in) :: phi
  real*8, dimension(nylm,nsph), intent(in) :: glm, psi
  real*8, dimension(nylm,nsph), intent(inout) :: sigma
  real*8, intent(inout) :: esolv
  type(ddc_solve_info) :: info
  integer(c_int) :: st, istar, icart
  istar = 0; icart = 0
  if (star) istar = 1
  if (cart) icart = 1
  st = ddc_cosmo(ddc_handle, istar, icart, phi, glm, psi, sigma, esolv, info)
  if (st == 5) then
    if (star) then
      write(iout,'(" adjoint ddCOSMO did not converge! Aborting...")')
    else
      write(iout,'(" ddCOSMO did not converge! Aborting...")')
    end if
    stop
  end if
  call ddc_check(st, 'cosmo')
  if (iprint > 0) then
    write(iout,*)
    if (star) then
      write(iout,'(" solution time of ddCOSMO adjoint equations L^* \sigma = ",f8.3," secs.")') &
        info%seconds
    else
      write(iout,'(" solution time of ddCOSMO direct equations L \sigma = ",f8.3," secs.")') &
        info%seconds
    end if
    write(iout,*)
  end if
end subroutine cosmo

! forces_dd(n, phi, sigma, s, fx)  (forces_dd.f90:1)
subroutine forces_dd(n, phi, sigma, s, fx)
  use ddcosmo
  implicit none
  integer, intent(in) :: n
  real*8, dimension(ncav), intent(in) :: phi
  real*8, dimension(nylm,nsph), intent(in) :: sigma, s
  real*8, dimension(3,n), intent(inout) :: fx
  call ddc_check(ddc_forces_dd(ddc_handle, phi, sigma, s, fx), 'forces_dd')
end subroutine forces_dd

! mkrhs(n, charge, x, y, z, ncav, ccav, phi, nylm, psi)  (mkrhs.f90:1)
subroutine mkrhs(n, charge, x, y, z, ncav_, ccav_, phi, nylm_, psi)
  use ddcosmo, only: ddc_handle, ddc_check
  use ddcosmo_c
  implicit none
  integer, intent(in) :: n, ncav_, nylm_
  real*8, dimension(n), intent(in) :: charge, x, y, z
  real*8, dimension(3,ncav_), intent(in) :: ccav_
  real*8, dimension(ncav_), intent(inout) :: phi
  real*8, dimension(nylm_,n), intent(inout) :: psi
  call ddc_check(ddc_mkrhs(ddc_handle, int(n,c_int), charge, x, y, z, int(ncav_,c_int), ccav_, &
                           phi, int(nylm_,c_int), psi), 'mkrhs')
end subroutine mkrhs

! efld(nsrc, src, csrc, ntrg, ctrg, ef)  (efld.f90:1)
subroutine efld(nsrc, src, csrc, ntrg, ctrg, ef)
  use ddcosmo, only: ddc_handle, ddc_check
  use ddcosmo_c
  implicit none
  integer, intent(in) :: nsrc, ntrg
  real*8, dimension(nsrc), intent(in) :: src
  real*8, dimension(3,nsrc), intent(in) :: csrc
  real*8, dimension(3,ntrg), intent(in) :: ctrg
  real*8, dimension(3,ntrg), intent(inout) :: ef
  call ddc_check(ddc_efld(ddc_handle, int(nsrc,c_int), src, csrc, int(ntrg,c_int), ctrg, ef), &
                 'efld')
end subroutine efld
