!> GPU drop-in for PROGRESS's prg_sp2_mod (src/prg_sp2_mod.F90) over libsp2b.
!!
!! NOT COMPILED IN THIS REPOSITORY: the build image has no Fortran compiler (gfortran is
!! absent), so this file is source for a PROGRESS maintainer, checked only by reading.
!! It builds where PROGRESS builds (BML's Fortran modules on the include path) and links
!! with -lsp2b.
!!
!! The module keeps the name, the public routines and the dummy arguments of the
!! reference's prg_sp2_mod, so Fortran callers `use prg_sp2_mod` and call unchanged.
!! Each routine hands BML's own C pointer (h_bml%ptr, the component the reference's C
!! binding fills, src/prg_c_interface.F90:1113-1129) to the PROGRESS-named C export of
!! libsp2b, which reads and writes BML matrices through BML's C API.  pp and vv are
!! passed as the arrays they are; sp2conv goes as a NUL-terminated string.
!!
!! Behaviour kept from the reference: a solve that does not converge prints the
!! reference's message and stops (src/prg_sp2_mod.F90:360-363); other failures (no GPU,
!! bad input) print the library's message and stop.  prg_sp2_basic_tcore, the
!! reference's own tensor-core variant, is served by the same GPU path as prg_sp2_basic
!! (rhofull_bml receives the same density).
module prg_sp2_mod

  use iso_c_binding
  use bml

  implicit none

  private

  integer, parameter :: dp = kind(1.0d0)

  public :: prg_sp2_basic
  public :: prg_sp2_alg1
  public :: prg_sp2_alg1_genseq
  public :: prg_sp2_alg1_seq
  public :: prg_prg_sp2_alg1_seq_inplace
  public :: prg_sp2_alg2
  public :: prg_sp2_alg2_genseq
  public :: prg_sp2_alg2_seq
  public :: prg_prg_sp2_alg2_seq_inplace
  public :: prg_sp2_submatrix
  public :: prg_sp2_submatrix_inplace
  public :: prg_sp2_basic_tcore

  interface
    subroutine c_sp2_basic(h, rho, threshold, bndfil, minit, maxit, conv, idemtol, verbose) &
         bind(C, name="prg_sp2_basic")
      import :: c_ptr, c_int, c_double, c_char
      type(c_ptr), value :: h, rho
      real(c_double), value :: threshold, bndfil, idemtol
      integer(c_int), value :: minit, maxit, verbose
      character(kind=c_char), dimension(*) :: conv
    end subroutine c_sp2_basic

    subroutine c_sp2_alg1(h, rho, threshold, bndfil, minit, maxit, conv, idemtol, verbose) &
         bind(C, name="prg_sp2_alg1")
      import :: c_ptr, c_int, c_double, c_char
      type(c_ptr), value :: h, rho
      real(c_double), value :: threshold, bndfil, idemtol
      integer(c_int), value :: minit, maxit, verbose
      character(kind=c_char), dimension(*) :: conv
    end subroutine c_sp2_alg1

    subroutine c_sp2_alg2(h, rho, threshold, bndfil, minit, maxit, conv, idemtol, verbose) &
         bind(C, name="prg_sp2_alg2")
      import :: c_ptr, c_int, c_double, c_char
      type(c_ptr), value :: h, rho
      real(c_double), value :: threshold, bndfil, idemtol
      integer(c_int), value :: minit, maxit, verbose
      character(kind=c_char), dimension(*) :: conv
    end subroutine c_sp2_alg2

    subroutine c_sp2_alg2_genseq(h, rho, threshold, bndfil, minit, maxit, conv, idemtol, &
         pp, icount, vv, verbose) bind(C, name="prg_sp2_alg2_genseq")
      import :: c_ptr, c_int, c_double, c_char
      type(c_ptr), value :: h, rho
      real(c_double), value :: threshold, bndfil, idemtol
      integer(c_int), value :: minit, maxit, verbose
      character(kind=c_char), dimension(*) :: conv
      integer(c_int) :: pp(*), icount
      real(c_double) :: vv(*)
    end subroutine c_sp2_alg2_genseq

    subroutine c_sp2_alg1_genseq(h, rho, threshold, bndfil, minit, maxit, conv, idemtol, &
         pp, icount, vv) bind(C, name="prg_sp2_alg1_genseq")
      import :: c_ptr, c_int, c_double, c_char
      type(c_ptr), value :: h, rho
      real(c_double), value :: threshold, bndfil, idemtol
      integer(c_int), value :: minit, maxit
      character(kind=c_char), dimension(*) :: conv
      integer(c_int) :: pp(*), icount
      real(c_double) :: vv(*)
    end subroutine c_sp2_alg1_genseq

    subroutine c_sp2_alg2_seq(h, rho, threshold, pp, icount, vv, verbose) &
         bind(C, name="prg_sp2_alg2_seq")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: h, rho
      real(c_double), value :: threshold
      integer(c_int) :: pp(*), icount
      real(c_double) :: vv(*)
      integer(c_int), value :: verbose
    end subroutine c_sp2_alg2_seq

    subroutine c_sp2_alg1_seq(h, rho, threshold, pp, icount, vv) bind(C, name="prg_sp2_alg1_seq")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: h, rho
      real(c_double), value :: threshold
      integer(c_int) :: pp(*), icount
      real(c_double) :: vv(*)
    end subroutine c_sp2_alg1_seq

    subroutine c_sp2_alg2_seq_inplace(rho, threshold, ppsize, pp, icount, vv, mineval, maxeval) &
         bind(C, name="prg_prg_sp2_alg2_seq_inplace")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: rho
      real(c_double), value :: threshold, mineval, maxeval
      integer(c_int), value :: ppsize
      integer(c_int) :: pp(*), icount
      real(c_double) :: vv(*)
    end subroutine c_sp2_alg2_seq_inplace

    subroutine c_sp2_alg1_seq_inplace(rho, threshold, ppsize, pp, icount, vv, mineval, maxeval) &
         bind(C, name="prg_prg_sp2_alg1_seq_inplace")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: rho
      real(c_double), value :: threshold, mineval, maxeval
      integer(c_int), value :: ppsize
      integer(c_int) :: pp(*), icount
      real(c_double) :: vv(*)
    end subroutine c_sp2_alg1_seq_inplace

    subroutine c_sp2_submatrix(ham, rho, threshold, pp, icount, vv, mineval, maxeval, core_size) &
         bind(C, name="prg_sp2_submatrix")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ham, rho
      real(c_double), value :: threshold, mineval, maxeval
      integer(c_int) :: pp(*), icount
      real(c_double) :: vv(*)
      integer(c_int), value :: core_size
    end subroutine c_sp2_submatrix

    subroutine c_sp2_submatrix_inplace(rho, threshold, pp, icount, vv, mineval, maxeval, &
         core_size) bind(C, name="prg_sp2_submatrix_inplace")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: rho
      real(c_double), value :: threshold, mineval, maxeval
      integer(c_int) :: pp(*), icount
      real(c_double) :: vv(*)
      integer(c_int), value :: core_size
    end subroutine c_sp2_submatrix_inplace

    integer(c_int) function c_last_status() bind(C, name="sp2b_prg_last_status")
      import :: c_int
    end function c_last_status

    type(c_ptr) function c_last_error() bind(C, name="sp2b_last_error")
      import :: c_ptr
    end function c_last_error
  end interface

  integer(c_int), parameter :: SP2B_NOT_CONVERGED = 4

contains

  !> Stops the program when the last call failed, as the reference does on
  !! non-convergence; prints the library's message for any other failure.
  subroutine check(who)
    character(len=*), intent(in) :: who
    integer(c_int) :: st
    character(kind=c_char), pointer :: msg(:)
    integer :: k
    st = c_last_status()
    if (st == 0) return
    if (st == SP2B_NOT_CONVERGED) then
      write(*,*) "SP2 purification is not converging: STOP!"
      stop
    end if
    call c_f_pointer(c_last_error(), msg, [1024])
    k = 0
    do while (k < 1024)
      if (msg(k + 1) == c_null_char) exit
      k = k + 1
    end do
    write(*,*) who, ": libsp2b status ", st, ": ", msg(1:k)
    stop
  end subroutine check

  integer(c_int) function verb(verbose)
    integer, optional, intent(in) :: verbose
    verb = 0
    if (present(verbose)) verb = int(verbose, c_int)
  end function verb

  subroutine prg_sp2_basic(h_bml, rho_bml, threshold, bndfil, minsp2iter, maxsp2iter, &
       sp2conv, idemtol, verbose)
    type(bml_matrix_t), intent(in) :: h_bml
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold, bndfil, idemtol
    integer, intent(in) :: minsp2iter, maxsp2iter, verbose
    character(len=*), intent(in) :: sp2conv
    call c_sp2_basic(h_bml%ptr, rho_bml%ptr, threshold, bndfil, int(minsp2iter, c_int), &
         int(maxsp2iter, c_int), trim(sp2conv)//c_null_char, idemtol, int(verbose, c_int))
    call check("prg_sp2_basic")
  end subroutine prg_sp2_basic

  subroutine prg_sp2_basic_tcore(h_bml, rho_bml, rhofull_bml, threshold, bndfil, minsp2iter, &
       maxsp2iter, sp2conv, idemtol, verbose)
    type(bml_matrix_t), intent(in) :: h_bml
    type(bml_matrix_t), intent(inout) :: rho_bml, rhofull_bml
    real(dp), intent(in) :: threshold, bndfil, idemtol
    integer, intent(in) :: minsp2iter, maxsp2iter, verbose
    character(len=*), intent(in) :: sp2conv
    call prg_sp2_basic(h_bml, rho_bml, threshold, bndfil, minsp2iter, maxsp2iter, sp2conv, &
         idemtol, verbose)
    call bml_copy(rho_bml, rhofull_bml)
  end subroutine prg_sp2_basic_tcore

  subroutine prg_sp2_alg2(h_bml, rho_bml, threshold, bndfil, minsp2iter, maxsp2iter, sp2conv, &
       idemtol, verbose)
    type(bml_matrix_t), intent(in) :: h_bml
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold, bndfil, idemtol
    integer, intent(in) :: minsp2iter, maxsp2iter
    character(len=*), intent(in) :: sp2conv
    integer, optional, intent(in) :: verbose
    call c_sp2_alg2(h_bml%ptr, rho_bml%ptr, threshold, bndfil, int(minsp2iter, c_int), &
         int(maxsp2iter, c_int), trim(sp2conv)//c_null_char, idemtol, verb(verbose))
    call check("prg_sp2_alg2")
  end subroutine prg_sp2_alg2

  subroutine prg_sp2_alg2_genseq(h_bml, rho_bml, threshold, bndfil, minsp2iter, maxsp2iter, &
       sp2conv, idemtol, pp, icount, vv, verbose)
    type(bml_matrix_t), intent(in) :: h_bml
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold, bndfil, idemtol
    integer, intent(in) :: minsp2iter, maxsp2iter
    character(len=*), intent(in) :: sp2conv
    integer, intent(inout) :: icount
    integer, intent(inout) :: pp(:)
    real(dp), intent(inout) :: vv(:)
    integer, optional, intent(in) :: verbose
    integer(c_int) :: ppc(size(pp)), ic
    ppc = int(pp, c_int)
    ic = int(icount, c_int)
    call c_sp2_alg2_genseq(h_bml%ptr, rho_bml%ptr, threshold, bndfil, int(minsp2iter, c_int), &
         int(maxsp2iter, c_int), trim(sp2conv)//c_null_char, idemtol, ppc, ic, vv, verb(verbose))
    pp = int(ppc)
    icount = int(ic)
    call check("prg_sp2_alg2_genseq")
  end subroutine prg_sp2_alg2_genseq

  subroutine prg_sp2_alg2_seq(h_bml, rho_bml, threshold, pp, icount, vv, verbose)
    type(bml_matrix_t), intent(in) :: h_bml
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold
    integer, intent(inout) :: icount
    integer, intent(inout) :: pp(:)
    real(dp), intent(inout) :: vv(:)
    integer, optional, intent(in) :: verbose
    integer(c_int) :: ppc(size(pp)), ic
    ppc = int(pp, c_int)
    ic = int(icount, c_int)
    call c_sp2_alg2_seq(h_bml%ptr, rho_bml%ptr, threshold, ppc, ic, vv, verb(verbose))
    call check("prg_sp2_alg2_seq")
  end subroutine prg_sp2_alg2_seq

  !> mineval / maxeval optional as in the reference; when absent the Gershgorin bounds of
  !! rho_bml are used, as bml_normalize does without them.
  subroutine prg_prg_sp2_alg2_seq_inplace(rho_bml, threshold, pp, icount, vv, mineval, &
       maxeval, verbose)
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold
    integer, intent(inout) :: icount
    integer, intent(inout) :: pp(:)
    real(dp), intent(inout) :: vv(:)
    real(dp), optional, intent(in) :: mineval, maxeval
    integer, optional, intent(in) :: verbose
    integer(c_int) :: ppc(size(pp)), ic
    real(dp) :: gbnd(2)
    if (present(mineval) .and. present(maxeval)) then
      gbnd = [mineval, maxeval]
    else
      call bml_gershgorin(rho_bml, gbnd)
    end if
    ppc = int(pp, c_int)
    ic = int(icount, c_int)
    call c_sp2_alg2_seq_inplace(rho_bml%ptr, threshold, int(size(pp), c_int), ppc, ic, vv, &
         gbnd(1), gbnd(2))
    call check("prg_prg_sp2_alg2_seq_inplace")
  end subroutine prg_prg_sp2_alg2_seq_inplace

  subroutine prg_sp2_alg1(h_bml, rho_bml, threshold, bndfil, minsp2iter, maxsp2iter, sp2conv, &
       idemtol, verbose)
    type(bml_matrix_t), intent(in) :: h_bml
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold, bndfil, idemtol
    integer, intent(in) :: minsp2iter, maxsp2iter
    character(len=*), intent(in) :: sp2conv
    integer, optional, intent(in) :: verbose
    call c_sp2_alg1(h_bml%ptr, rho_bml%ptr, threshold, bndfil, int(minsp2iter, c_int), &
         int(maxsp2iter, c_int), trim(sp2conv)//c_null_char, idemtol, verb(verbose))
    call check("prg_sp2_alg1")
  end subroutine prg_sp2_alg1

  subroutine prg_sp2_alg1_genseq(h_bml, rho_bml, threshold, bndfil, minsp2iter, maxsp2iter, &
       sp2conv, idemtol, pp, icount, vv)
    type(bml_matrix_t), intent(in) :: h_bml
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold, bndfil, idemtol
    integer, intent(in) :: minsp2iter, maxsp2iter
    character(len=*), intent(in) :: sp2conv
    integer, intent(inout) :: icount
    integer, intent(inout) :: pp(:)
    real(dp), intent(inout) :: vv(:)
    integer(c_int) :: ppc(size(pp)), ic
    ppc = int(pp, c_int)
    ic = int(icount, c_int)
    call c_sp2_alg1_genseq(h_bml%ptr, rho_bml%ptr, threshold, bndfil, int(minsp2iter, c_int), &
         int(maxsp2iter, c_int), trim(sp2conv)//c_null_char, idemtol, ppc, ic, vv)
    pp = int(ppc)
    icount = int(ic)
    call check("prg_sp2_alg1_genseq")
  end subroutine prg_sp2_alg1_genseq

  subroutine prg_sp2_alg1_seq(h_bml, rho_bml, threshold, pp, icount, vv)
    type(bml_matrix_t), intent(in) :: h_bml
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold
    integer, intent(inout) :: icount
    integer, intent(inout) :: pp(:)
    real(dp), intent(inout) :: vv(:)
    integer(c_int) :: ppc(size(pp)), ic
    ppc = int(pp, c_int)
    ic = int(icount, c_int)
    call c_sp2_alg1_seq(h_bml%ptr, rho_bml%ptr, threshold, ppc, ic, vv)
    call check("prg_sp2_alg1_seq")
  end subroutine prg_sp2_alg1_seq

  subroutine prg_prg_sp2_alg1_seq_inplace(rho_bml, threshold, pp, icount, vv, mineval, maxeval)
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold
    integer, intent(inout) :: icount
    integer, intent(inout) :: pp(:)
    real(dp), intent(inout) :: vv(:)
    real(dp), intent(in) :: mineval, maxeval
    integer(c_int) :: ppc(size(pp)), ic
    ppc = int(pp, c_int)
    ic = int(icount, c_int)
    call c_sp2_alg1_seq_inplace(rho_bml%ptr, threshold, int(size(pp), c_int), ppc, ic, vv, &
         mineval, maxeval)
    call check("prg_prg_sp2_alg1_seq_inplace")
  end subroutine prg_prg_sp2_alg1_seq_inplace

  subroutine prg_sp2_submatrix(ham_bml, rho_bml, threshold, pp, icount, vv, mineval, maxeval, &
       core_size)
    type(bml_matrix_t), intent(in) :: ham_bml
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold, mineval, maxeval
    integer, intent(in) :: icount, core_size
    integer, intent(in) :: pp(:)
    real(dp), intent(inout) :: vv(:)
    integer(c_int) :: ppc(size(pp)), ic
    ppc = int(pp, c_int)
    ic = int(icount, c_int)
    call c_sp2_submatrix(ham_bml%ptr, rho_bml%ptr, threshold, ppc, ic, vv, mineval, maxeval, &
         int(core_size, c_int))
    call check("prg_sp2_submatrix")
  end subroutine prg_sp2_submatrix

  subroutine prg_sp2_submatrix_inplace(rho_bml, threshold, pp, icount, vv, mineval, maxeval, &
       core_size)
    type(bml_matrix_t), intent(inout) :: rho_bml
    real(dp), intent(in) :: threshold, mineval, maxeval
    integer, intent(inout) :: icount
    integer, intent(inout) :: pp(:)
    integer, intent(in) :: core_size
    real(dp), intent(inout) :: vv(:)
    integer(c_int) :: ppc(size(pp)), ic
    ppc = int(pp, c_int)
    ic = int(icount, c_int)
    call c_sp2_submatrix_inplace(rho_bml%ptr, threshold, ppc, ic, vv, mineval, maxeval, &
         int(core_size, c_int))
    call check("prg_sp2_submatrix_inplace")
  end subroutine prg_sp2_submatrix_inplace

end module prg_sp2_mod
