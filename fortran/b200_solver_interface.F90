!
! b200_solver_interface.F90 -- Fortran side of the hprmat-b200 C ABI (include/hprmat_b200.h).
!
! HPRMAT reaches the B200 library as solver type 7 through this module: iso_c_binding
! interfaces to the library's extern "C" entry points, interoperable mirrors of its option and
! statistics structs, and two module procedures for the reference's call sites:
!
!   solve_rmatrix_b200  -- the solve inside solve_rmatrix / rmatrix (C X = blockdiag(q2) and
!                          R = normfac q2^T X), with the argument list of the reference's
!                          solve_rmatrix_dense (src/rmat_solvers.F90:98-148); the `case (7)` of
!                          the two dispatches (src/rmatrix_hp.F90:299-322, src/rmat_solvers.F90:
!                          69-88, fortran/solver_type7.patch) calls it with ch(:,:,is);
!   rmatrix_b200        -- the whole rmatrix (src/rmatrix_hp.F90:175-368, local and non-local
!                          potentials, ns >= 1 intervals, wave functions) on the GPU: C(E) is
!                          assembled on the device, so no N x N host matrix exists.
!
! Both use one library context on device 0, created on first use (the reference initialises
! its GPU backend the same way, src/cusolver_interface.cu:193-220) and released by
! b200_finalize.  A nonzero library status is an error: there is no CPU fallback.  Status 99
! (refinement stopped above its tolerance) still returns the results, as the reference's
! info = 99 does.
!
! Kinds: complex arrays are complex(c_double_complex) (the memory of complex*16), passed where
! the C prototype has double*; scalars the C side takes by value carry the VALUE attribute.
! tests/test_fortran_interface.py checks every bind(C) interface here against the C header
! (names, argument order, by-value versus by-reference, kinds) and the struct mirrors' fields.
!
module b200_solver_interface
  use iso_c_binding
  implicit none
  private

  public :: b200_opts, b200_stats, b200_scan_block
  public :: solve_rmatrix_b200, rmatrix_b200, b200_finalize, b200_set_opts, b200_last_error
  public :: gpu_b200_solve_mixed, gpu_b200_solve_double, gpu_b200_finalize
  public :: hprmat_b200_default_opts, hprmat_b200_create, hprmat_b200_destroy, hprmat_b200_set_opts
  public :: hprmat_b200_set_stream, hprmat_b200_rmat_ini, hprmat_b200_rmatrix, hprmat_b200_rmatrix_device
  public :: hprmat_b200_rmatrix_wf, hprmat_b200_rmatrix_full, hprmat_b200_solve_linear
  public :: hprmat_b200_solve_linear_device, hprmat_b200_solve_rmatrix, hprmat_b200_boundary
  public :: hprmat_b200_rmatrix_adjoint, hprmat_b200_rmatrix_scan, hprmat_b200_rmatrix_scan_shifted
  public :: hprmat_b200_solve_linear_noalloc
  public :: hprmat_b200_status_string, hprmat_b200_last_error, hprmat_b200_version
  public :: B200_OK, B200_NOT_CONVERGED, B200_PREC_FP64, B200_PREC_MIXED, B200_ABI_VERSION

  integer(c_int), parameter :: B200_OK = 0, B200_NOT_CONVERGED = 99
  integer(c_int), parameter :: B200_PREC_FP64 = 0, B200_PREC_MIXED = 1
  integer(c_int), parameter :: B200_ABI_VERSION = 101

  ! hprmat_b200_opts (48 bytes)
  type, bind(C) :: b200_opts
    integer(c_int) :: precision = B200_PREC_MIXED
    integer(c_int) :: max_refine = 3
    real(c_double) :: tol = 1.0d-12
    real(c_double) :: surface_tol = 1.0d-11
    integer(c_int) :: panel_nb = 0
    integer(c_int) :: reuse_factors = 0
    integer(c_int) :: estimate_condition = 0
    integer(c_int) :: growth_error = 0
    integer(c_int) :: reserved(1) = 0
  end type

  ! hprmat_b200_stats
  type, bind(C) :: b200_stats
    integer(c_int) :: status, info, refine_steps, inner_iterations, nb, n, nrhs
    real(c_double) :: rel_residual, surface_change, residual_floor
    real(c_double) :: floor_history(9), residual_history(9)
    real(c_double) :: ms_assemble, ms_factor, ms_solve, ms_refine, ms_umatrix, ms_total
    integer(c_int) :: factorizations, fp64_fallback
    real(c_double) :: pivot_growth, cond_estimate, ms_condest
  end type

  ! hprmat_b200_scan_block (pointer members as c_ptr: c_loc of the caller's arrays)
  type, bind(C) :: b200_scan_block
    integer(c_int) :: nch
    type(c_ptr) :: lval
    type(c_ptr) :: cpot
    integer(c_int) :: ncp1
    integer(c_int) :: nenergies
    type(c_ptr) :: qk
    type(c_ptr) :: eta
    type(c_ptr) :: cu
    type(c_ptr) :: nopen
    type(c_ptr) :: status
  end type

  interface
    ! ---- drop-in twins of the reference's GPU C ABI (src/gpu_solver_interface.F90:61-99)
    integer(c_int) function gpu_b200_solve_mixed(A, B, n, nrhs, max_refine, tol, info) &
        bind(C, name="gpu_b200_solve_mixed_")
      import :: c_int, c_double, c_double_complex
      complex(c_double_complex), intent(in) :: A(*)
      complex(c_double_complex), intent(inout) :: B(*)
      integer(c_int), intent(in) :: n, nrhs, max_refine
      real(c_double), intent(in) :: tol
      integer(c_int), intent(out) :: info
    end function

    integer(c_int) function gpu_b200_solve_double(A, B, n, nrhs, info) bind(C, name="gpu_b200_solve_double_")
      import :: c_int, c_double_complex
      complex(c_double_complex), intent(in) :: A(*)
      complex(c_double_complex), intent(inout) :: B(*)
      integer(c_int), intent(in) :: n, nrhs
      integer(c_int), intent(out) :: info
    end function

    integer(c_int) function gpu_b200_finalize() bind(C, name="gpu_b200_finalize_")
      import :: c_int
    end function

    ! ---- contexts and options
    subroutine hprmat_b200_default_opts(opts) bind(C, name="hprmat_b200_default_opts")
      import :: b200_opts
      type(b200_opts), intent(out) :: opts
    end subroutine

    integer(c_int) function hprmat_b200_create(device, opts, ctx) bind(C, name="hprmat_b200_create")
      import :: c_int, c_ptr, b200_opts
      integer(c_int), value :: device
      type(b200_opts), intent(in) :: opts
      type(c_ptr), intent(out) :: ctx
    end function

    integer(c_int) function hprmat_b200_destroy(ctx) bind(C, name="hprmat_b200_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    integer(c_int) function hprmat_b200_set_opts(ctx, opts) bind(C, name="hprmat_b200_set_opts")
      import :: c_int, c_ptr, b200_opts
      type(c_ptr), value :: ctx
      type(b200_opts), intent(in) :: opts
    end function

    integer(c_int) function hprmat_b200_set_stream(ctx, stream) bind(C, name="hprmat_b200_set_stream")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream
    end function

    ! ---- the R-matrix path
    integer(c_int) function hprmat_b200_rmat_ini(ctx, nr, ns, rmax, zrma) bind(C, name="hprmat_b200_rmat_ini")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: nr, ns
      real(c_double), value :: rmax
      real(c_double), intent(out) :: zrma(*)
    end function

    integer(c_int) function hprmat_b200_rmatrix(ctx, nch, lval, qk, eta, rmax, nr, ns, cpot, ncp1, ndim, cu, &
        nopen, stats) bind(C, name="hprmat_b200_rmatrix")
      import :: c_int, c_ptr, c_double, c_double_complex, b200_stats
      type(c_ptr), value :: ctx
      integer(c_int), value :: nch
      integer(c_int), intent(in) :: lval(*)
      real(c_double), intent(in) :: qk(*), eta(*)
      real(c_double), value :: rmax
      integer(c_int), value :: nr, ns
      complex(c_double_complex), intent(in) :: cpot(*)
      integer(c_int), value :: ncp1, ndim
      complex(c_double_complex), intent(out) :: cu(*)
      integer(c_int), intent(out) :: nopen
      type(b200_stats), intent(out) :: stats
    end function

    integer(c_int) function hprmat_b200_rmatrix_device(ctx, nch, lval, qk, eta, rmax, nr, ns, d_cpot, ncp1, &
        ndim, d_cu, nopen, stats) bind(C, name="hprmat_b200_rmatrix_device")
      import :: c_int, c_ptr, c_double, b200_stats
      type(c_ptr), value :: ctx
      integer(c_int), value :: nch
      integer(c_int), intent(in) :: lval(*)
      real(c_double), intent(in) :: qk(*), eta(*)
      real(c_double), value :: rmax
      integer(c_int), value :: nr, ns
      type(c_ptr), value :: d_cpot
      integer(c_int), value :: ncp1, ndim
      type(c_ptr), value :: d_cu
      integer(c_int), intent(out) :: nopen
      type(b200_stats), intent(out) :: stats
    end function

    integer(c_int) function hprmat_b200_rmatrix_wf(ctx, nch, lval, qk, eta, rmax, nr, ns, cpot, ncp1, ndim, &
        cu, nopen, nc, nvc, cf, nwf1, nwf2, stats) bind(C, name="hprmat_b200_rmatrix_wf")
      import :: c_int, c_ptr, c_double, c_double_complex, b200_stats
      type(c_ptr), value :: ctx
      integer(c_int), value :: nch
      integer(c_int), intent(in) :: lval(*)
      real(c_double), intent(in) :: qk(*), eta(*)
      real(c_double), value :: rmax
      integer(c_int), value :: nr, ns
      complex(c_double_complex), intent(in) :: cpot(*)
      integer(c_int), value :: ncp1, ndim
      complex(c_double_complex), intent(out) :: cu(*)
      integer(c_int), intent(out) :: nopen
      integer(c_int), value :: nc
      integer(c_int), intent(in) :: nvc(*)
      complex(c_double_complex), intent(out) :: cf(*)
      integer(c_int), value :: nwf1, nwf2
      type(b200_stats), intent(out) :: stats
    end function

    integer(c_int) function hprmat_b200_rmatrix_full(ctx, nch, lval, qk, eta, rmax, nr, ns, cpot, ncp1, ndim, &
        cu, nopen, twf, cf, nwf1, nwf2, nc, nvc, ncp2, cpnl, stats) bind(C, name="hprmat_b200_rmatrix_full")
      import :: c_int, c_ptr, c_double, c_double_complex, b200_stats
      type(c_ptr), value :: ctx
      integer(c_int), value :: nch
      integer(c_int), intent(in) :: lval(*)
      real(c_double), intent(in) :: qk(*), eta(*)
      real(c_double), value :: rmax
      integer(c_int), value :: nr, ns
      complex(c_double_complex), intent(in) :: cpot(*)
      integer(c_int), value :: ncp1, ndim
      complex(c_double_complex), intent(out) :: cu(*)
      integer(c_int), intent(out) :: nopen
      integer(c_int), value :: twf
      complex(c_double_complex), intent(out) :: cf(*)
      integer(c_int), value :: nwf1, nwf2, nc
      integer(c_int), intent(in) :: nvc(*)
      integer(c_int), value :: ncp2
      complex(c_double_complex), intent(in) :: cpnl(*)
      type(b200_stats), intent(out) :: stats
    end function

    integer(c_int) function hprmat_b200_rmatrix_adjoint(ctx, nch, lval, qk, eta, rmax, nr, ns, cpot, ncp1, ndim, &
        gu, cu, nopen, grad, stats) bind(C, name="hprmat_b200_rmatrix_adjoint")
      import :: c_int, c_ptr, c_double, c_double_complex, b200_stats
      type(c_ptr), value :: ctx
      integer(c_int), value :: nch
      integer(c_int), intent(in) :: lval(*)
      real(c_double), intent(in) :: qk(*), eta(*)
      real(c_double), value :: rmax
      integer(c_int), value :: nr, ns
      complex(c_double_complex), intent(in) :: cpot(*)
      integer(c_int), value :: ncp1, ndim
      complex(c_double_complex), intent(in) :: gu(*)
      complex(c_double_complex), intent(out) :: cu(*)
      integer(c_int), intent(out) :: nopen
      complex(c_double_complex), intent(out) :: grad(*)
      type(b200_stats), intent(out) :: stats
    end function

    integer(c_int) function hprmat_b200_rmatrix_scan(ctx, nblocks, blocks, rmax, nr, nworkers, seconds) &
        bind(C, name="hprmat_b200_rmatrix_scan")
      import :: c_int, c_ptr, c_double, b200_scan_block
      type(c_ptr), value :: ctx
      integer(c_int), value :: nblocks
      type(b200_scan_block), intent(in) :: blocks(*)
      real(c_double), value :: rmax
      integer(c_int), value :: nr, nworkers
      real(c_double), intent(out) :: seconds
    end function

    integer(c_int) function hprmat_b200_rmatrix_scan_shifted(ctx, nblocks, blocks, rmax, nr, seconds) &
        bind(C, name="hprmat_b200_rmatrix_scan_shifted")
      import :: c_int, c_ptr, c_double, b200_scan_block
      type(c_ptr), value :: ctx
      integer(c_int), value :: nblocks
      type(b200_scan_block), intent(in) :: blocks(*)
      real(c_double), value :: rmax
      integer(c_int), value :: nr
      real(c_double), intent(out) :: seconds
    end function

    integer(c_int) function hprmat_b200_boundary(nch, lval, qk, eta, rmax, co, cop, xc1, xc2, nopen) &
        bind(C, name="hprmat_b200_boundary")
      import :: c_int, c_double, c_double_complex
      integer(c_int), value :: nch
      integer(c_int), intent(in) :: lval(*)
      real(c_double), intent(in) :: qk(*), eta(*)
      real(c_double), value :: rmax
      complex(c_double_complex), intent(out) :: co(*), cop(*)
      real(c_double), intent(out) :: xc1(*), xc2(*)
      integer(c_int), intent(out) :: nopen
    end function

    ! ---- dense solves
    integer(c_int) function hprmat_b200_solve_linear(ctx, A, B, n, nrhs, stats) &
        bind(C, name="hprmat_b200_solve_linear")
      import :: c_int, c_ptr, c_double_complex, b200_stats
      type(c_ptr), value :: ctx
      complex(c_double_complex), intent(in) :: A(*)
      complex(c_double_complex), intent(inout) :: B(*)
      integer(c_int), value :: n, nrhs
      type(b200_stats), intent(out) :: stats
    end function

    integer(c_int) function hprmat_b200_solve_linear_device(ctx, d_A, d_B, n, nrhs, stats) &
        bind(C, name="hprmat_b200_solve_linear_device")
      import :: c_int, c_ptr, b200_stats
      type(c_ptr), value :: ctx, d_A, d_B
      integer(c_int), value :: n, nrhs
      type(b200_stats), intent(out) :: stats
    end function

    integer(c_int) function hprmat_b200_solve_rmatrix(ctx, cmat, bvec, nch, nlag, normfac, rmat, stats) &
        bind(C, name="hprmat_b200_solve_rmatrix")
      import :: c_int, c_ptr, c_double, c_double_complex, b200_stats
      type(c_ptr), value :: ctx
      complex(c_double_complex), intent(in) :: cmat(*), bvec(*)
      integer(c_int), value :: nch, nlag
      real(c_double), value :: normfac
      complex(c_double_complex), intent(out) :: rmat(*)
      type(b200_stats), intent(out) :: stats
    end function

    integer(c_int) function hprmat_b200_solve_linear_noalloc(d_A, d_B, n, nrhs, stream, info) &
        bind(C, name="hprmat_b200_solve_linear_noalloc")
      import :: c_int, c_ptr
      type(c_ptr), value :: d_A, d_B
      integer(c_int), value :: n, nrhs
      type(c_ptr), value :: stream
      integer(c_int), intent(out) :: info
    end function

    ! ---- messages and version
    type(c_ptr) function hprmat_b200_status_string(status) bind(C, name="hprmat_b200_status_string")
      import :: c_int, c_ptr
      integer(c_int), value :: status
    end function

    type(c_ptr) function hprmat_b200_last_error() bind(C, name="hprmat_b200_last_error")
      import :: c_ptr
    end function

    integer(c_int) function hprmat_b200_version() bind(C, name="hprmat_b200_version")
      import :: c_int
    end function
  end interface

  ! the module's context (device 0), created on first use
  type(c_ptr), save :: g_ctx = c_null_ptr
  type(b200_opts), save :: g_opts
  integer, save :: g_nr = -1, g_ns = -1
  real(c_double), save :: g_rmax = -1.0d0

contains

  ! The library's last error message as a Fortran string.
  function b200_last_error() result(msg)
    character(len=:), allocatable :: msg
    character(kind=c_char), pointer :: p(:)
    integer :: n
    type(c_ptr) :: cp
    cp = hprmat_b200_last_error()
    msg = ''
    if (.not. c_associated(cp)) return
    call c_f_pointer(cp, p, [4096])
    n = 0
    do while (n < 4096)
      if (p(n + 1) == c_null_char) exit
      n = n + 1
    end do
    allocate(character(len=n) :: msg)
    msg = transfer(p(1:n), msg)
  end function

  ! Context of the module on device 0 (the library checks its ABI against this module's
  ! B200_ABI_VERSION on first use).
  subroutine ensure_ctx(ierr)
    integer, intent(out) :: ierr
    ierr = 0
    if (c_associated(g_ctx)) return
    if (hprmat_b200_version() /= B200_ABI_VERSION) then
      write(*, '(a)') 'b200_solver_interface: library ABI differs from this module; rebuild'
      ierr = -1
      return
    end if
    ierr = hprmat_b200_create(0_c_int, g_opts, g_ctx)
    if (ierr /= 0) write(*, '(2a)') 'b200_solver_interface: create failed: ', b200_last_error()
  end subroutine

  ! Options of the module's context (defaults: mixed precision, 3 refinement steps, tol 1e-12).
  subroutine b200_set_opts(opts, ierr)
    type(b200_opts), intent(in) :: opts
    integer, intent(out) :: ierr
    g_opts = opts
    ierr = 0
    if (c_associated(g_ctx)) ierr = hprmat_b200_set_opts(g_ctx, g_opts)
  end subroutine

  ! Releases the module's context (and with it every device buffer it holds).
  subroutine b200_finalize()
    integer(c_int) :: s
    if (c_associated(g_ctx)) s = hprmat_b200_destroy(g_ctx)
    g_ctx = c_null_ptr
    g_nr = -1
    g_ns = -1
    g_rmax = -1.0d0
  end subroutine

  ! Solver type 7 of solve_rmatrix / rmatrix: solves cmat X = blockdiag(B_vector) on the GPU and
  ! returns Rmat(i, j) = normfac sum_r B_vector(r) X((i-1)*nlag + r, j), the argument list and
  ! result of solve_rmatrix_dense (src/rmat_solvers.F90:98-148).  cmat is read only.  On a
  ! library error Rmat is zeroed and the message printed, as solve_rmatrix_dense does on a
  ! nonzero ZGESV info.
  subroutine solve_rmatrix_b200(cmat, B_vector, nch, nlag, normfac, Rmat)
    integer, intent(in) :: nch, nlag
    real(c_double), intent(in) :: normfac
    complex(c_double_complex), intent(in) :: cmat(nch*nlag, nch*nlag), B_vector(nlag)
    complex(c_double_complex), intent(out) :: Rmat(nch, nch)
    type(b200_stats) :: st
    integer :: ierr
    integer(c_int) :: s
    call ensure_ctx(ierr)
    if (ierr /= 0) then
      Rmat = (0.0d0, 0.0d0)
      return
    end if
    s = hprmat_b200_solve_rmatrix(g_ctx, cmat, B_vector, int(nch, c_int), int(nlag, c_int), normfac, Rmat, st)
    if (s /= B200_OK .and. s /= B200_NOT_CONVERGED) then
      write(*, '(a,i0,2a)') 'solve_rmatrix_b200: status ', s, ': ', b200_last_error()
      Rmat = (0.0d0, 0.0d0)
    end if
  end subroutine

  ! The whole rmatrix call (src/rmatrix_hp.F90:175-186, same arguments; isolver is not needed:
  ! this is solver type 7) with C(E) assembled on the device.  The mesh (rmat_ini) is set up
  ! on the device whenever nr, ns or rmax change.  twf = .true. adds the wave functions in cf;
  ! ncp2 > 0 the non-local potential cpnl.
  subroutine rmatrix_b200(nch, lval, qk, eta, rmax, nr, ns, cpot, cu, ncp1, ndim, nopen, twf, cf, nwf1, nwf2, &
                          nc, nvc, ncp2, cpnl)
    integer, intent(in) :: nch, nr, ns, ncp1, ndim, nwf1, nwf2, nc, ncp2
    integer, intent(in) :: lval(nch), nvc(*)
    real(c_double), intent(in) :: qk(nch), eta(nch), rmax
    complex(c_double_complex), intent(in) :: cpot(ncp1, ndim, ndim), cpnl(*)
    complex(c_double_complex), intent(out) :: cu(ndim, ndim), cf(nwf1, nwf2, *)
    integer, intent(out) :: nopen
    logical, intent(in) :: twf
    type(b200_stats) :: st
    integer(c_int) :: s, nop, itwf
    integer(c_int), allocatable :: lv(:), vc(:)
    real(c_double), allocatable :: zr(:)
    integer :: ierr
    call ensure_ctx(ierr)
    if (ierr /= 0) then
      cu = (0.0d0, 0.0d0)
      nopen = 0
      return
    end if
    if (nr /= g_nr .or. ns /= g_ns .or. rmax /= g_rmax) then
      allocate(zr(nr * ns))
      s = hprmat_b200_rmat_ini(g_ctx, int(nr, c_int), int(ns, c_int), rmax, zr)
      if (s /= B200_OK) write(*, '(2a)') 'rmatrix_b200: rmat_ini failed: ', b200_last_error()
      g_nr = nr
      g_ns = ns
      g_rmax = rmax
    end if
    lv = int(lval, c_int)
    vc = int(nvc(1:max(nc, 1)), c_int)
    itwf = 0
    if (twf) itwf = 1
    s = hprmat_b200_rmatrix_full(g_ctx, int(nch, c_int), lv, qk, eta, rmax, int(nr, c_int), int(ns, c_int), cpot, &
                                 int(ncp1, c_int), int(ndim, c_int), cu, nop, itwf, cf, int(nwf1, c_int), &
                                 int(nwf2, c_int), int(nc, c_int), vc, int(ncp2, c_int), cpnl, st)
    nopen = nop
    if (s /= B200_OK .and. s /= B200_NOT_CONVERGED) &
      write(*, '(a,i0,2a)') 'rmatrix_b200: status ', s, ': ', b200_last_error()
  end subroutine

end module b200_solver_interface
