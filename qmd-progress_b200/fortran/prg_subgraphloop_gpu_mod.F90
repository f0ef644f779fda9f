!> GPU form of prg_subgraphSP2Loop (src/prg_subgraphloop_mod.F90:36-126) over libsp2b.
!!
!! NOT COMPILED IN THIS REPOSITORY: the build image has no Fortran compiler (gfortran is
!! absent), so this file is source for a PROGRESS maintainer, checked only by reading.
!! It builds next to prg_subgraphloop_mod (it uses prg_graph_mod's types and routines)
!! and links with -lsp2b.
!!
!! prg_subgraphSP2Loop_gpu takes the arguments of prg_subgraphSP2Loop.  It keeps the
!! reference's index step (bml_matrix2submatrix_index with the double jump, :55-69) and
!! its fnorm and collection steps (prg_fnormGraph, prg_collectMatrixFromParts), and
!! replaces the serial part loop (extract, prg_sp2_submatrix_inplace, reassemble,
!! :86-116) with one batched call, sp2b_subgraph_sp2_loop, over this rank's parts.  H
!! reaches the library as CSR, scanned from the dense export of h_bml; the core rows of
!! every local part come back in a dense N x N array (zero elsewhere) that is imported
!! into rho_bml with the call's threshold, as bml_submatrix2matrix thresholds them.  The
!! library returns vv after the square root of prg_fnormGraph; the squares are handed to
!! prg_fnormGraph, which sums them over ranks and takes the root again.
module prg_subgraphloop_gpu_mod

  use iso_c_binding
  use bml
  use prg_graph_mod

  implicit none

  private

  integer, parameter :: dp = kind(1.0d0)

  public :: prg_subgraphSP2Loop_gpu

  interface
    integer(c_int) function sp2b_subgraph_sp2_loop(n, h_row_ptr, h_col, h_val, nparts, &
         halo_ptr, halo_idx, llsize, pp, maxiter, mineval, maxeval, rho_core, rho_dense, vv, &
         opts) bind(C, name="sp2b_subgraph_sp2_loop")
      import :: c_int, c_long_long, c_double, c_ptr
      integer(c_int), value :: n, nparts, maxiter
      integer(c_long_long) :: h_row_ptr(*), halo_ptr(*)
      integer(c_int) :: h_col(*), halo_idx(*), llsize(*), pp(*)
      real(c_double) :: h_val(*), vv(*)
      real(c_double), value :: mineval, maxeval
      type(c_ptr), value :: rho_core, rho_dense, opts
    end function sp2b_subgraph_sp2_loop
  end interface

contains

  subroutine prg_subgraphSP2Loop_gpu(h_bml, g_bml, rho_bml, gp, threshold)
    type(bml_matrix_t), intent(in) :: h_bml, g_bml
    type(bml_matrix_t), intent(inout) :: rho_bml
    type(graph_partitioning_t), intent(inout) :: gp
    real(dp), intent(in) :: threshold

    integer :: i, j, k, n, p0, p1, np, nnz
    integer, allocatable :: vsize(:)
    real(dp), allocatable, target :: h(:,:), rho(:,:)
    real(c_double), allocatable :: val(:), vv(:)
    integer(c_long_long), allocatable :: rp(:), hptr(:)
    integer(c_int), allocatable :: col(:), hidx(:), lls(:), ppc(:)
    integer(c_int) :: st

    n = bml_get_N(h_bml)
    allocate(vsize(2))

    ! core+halo node lists of every part, as the reference builds them
    do i = 1, gp%totalParts
      call bml_matrix2submatrix_index(g_bml, gp%sgraph(i)%nodeInPart, gp%nnodesInPart(i), &
           gp%sgraph(i)%core_halo_index, vsize, .true., h_bml)
      gp%sgraph(i)%lsize = vsize(1)
      gp%sgraph(i)%llsize = vsize(2)
    end do
    deallocate(vsize)

    ! H as CSR (0-based columns), row i of the CSR is row i of H
    allocate(h(n, n))
    call bml_export_to_dense(h_bml, h)
    nnz = count(h /= 0.0_dp)
    allocate(rp(n + 1), col(max(nnz, 1)), val(max(nnz, 1)))
    rp(1) = 0
    k = 0
    do i = 1, n
      do j = 1, n
        if (h(i, j) /= 0.0_dp) then
          k = k + 1
          col(k) = int(j - 1, c_int)
          val(k) = h(i, j)
        end if
      end do
      rp(i + 1) = int(k, c_long_long)
    end do
    deallocate(h)

    ! this rank's parts: node lists concatenated (0-based), core counts
    p0 = gp%localPartMin(gp%myRank + 1)
    p1 = gp%localPartMax(gp%myRank + 1)
    np = p1 - p0 + 1
    allocate(hptr(np + 1), lls(np))
    hptr(1) = 0
    do i = p0, p1
      hptr(i - p0 + 2) = hptr(i - p0 + 1) + int(gp%sgraph(i)%lsize, c_long_long)
      lls(i - p0 + 1) = int(gp%sgraph(i)%llsize, c_int)
    end do
    allocate(hidx(max(int(hptr(np + 1)), 1)))
    do i = p0, p1
      do j = 1, gp%sgraph(i)%lsize
        hidx(hptr(i - p0 + 1) + j) = int(gp%sgraph(i)%core_halo_index(j), c_int)
      end do
    end do

    allocate(ppc(max(gp%maxIter, 1)), vv(max(gp%maxIter, 1)), rho(n, n))
    ppc(1:gp%maxIter) = int(gp%pp(1:gp%maxIter), c_int)
    st = sp2b_subgraph_sp2_loop(int(n, c_int), rp, col, val, int(np, c_int), hptr, hidx, lls, &
         ppc, int(gp%maxIter, c_int), gp%mineval, gp%maxeval, c_null_ptr, c_loc(rho), vv, &
         c_null_ptr)
    if (st /= 0) then
      write(*,*) "prg_subgraphSP2Loop_gpu: libsp2b status ", st
      stop
    end if

    ! core rows into rho_bml (bml_submatrix2matrix thresholds with the same value)
    call bml_import_from_dense(bml_get_type(rho_bml), rho, rho_bml, threshold, &
         bml_get_M(rho_bml))

    ! sums of squares per iteration, summed over ranks and rooted by prg_fnormGraph
    gp%vv(1:gp%maxIter) = vv(1:gp%maxIter)**2
    call prg_fnormGraph(gp)
    call prg_collectMatrixFromParts(gp, rho_bml)

    deallocate(rp, col, val, hptr, lls, hidx, ppc, vv, rho)
  end subroutine prg_subgraphSP2Loop_gpu

end module prg_subgraphloop_gpu_mod
