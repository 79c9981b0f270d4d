! ISO_C_BINDING interface module for libzolo_b200 (include/zolo_b200.h).
!
! Explicit interfaces for the reference-named host-array entry points of the
! polar-decomposition path (1x1 process grid: DESC(9) descriptors with
! DTYPE_ = 1, RSRC_ = CSRC_ = 0, IA = JA = IQ = JQ = 1), the handle and option
! calls, and the device-array entry points.  Scalars travel by value and arrays
! by reference, CHARACTER arguments as one c_char each.  Argument meanings and
! INFO codes are those of the reference routines cited per interface.
!
! Unchanged drivers do not need this module: the gfortran-mangled symbols
! (pzolopd1_, pzolopd2_, pqdwhfacs_, zolopd_, zoloeig_) take the reference's
! implicit-interface calls as they are.
!
! Build:  gfortran -c zolo_b200.f90   (links with -lzolo_b200)
module zolo_b200
  use, intrinsic :: iso_c_binding, only: c_int, c_double, c_char, c_ptr, c_int64_t
  implicit none
  private
  public :: zolo_pzolopd1, zolo_pzolopd2, zolo_pqdwhfacs, zolo_zolopd, zolo_zoloeig
  public :: zolo_default_handle, zolo_create, zolo_destroy, zolo_set_option, zolo_release_workspace
  public :: zolo_polar_dev, zolo_pzolopd1_dev, zolo_qdwh_dev
  public :: ZOLO_OPT_SHARED_QR, ZOLO_OPT_NS_FINISH, ZOLO_OPT_CHOL_INVERSE, ZOLO_OPT_BETA_FROB, &
            ZOLO_OPT_TERM_PLAN, ZOLO_OPT_MIXED, ZOLO_OPT_MIXED_SLICES, ZOLO_OPT_OWN_BOUNDS, &
            ZOLO_OPT_NORM2_BOUND, ZOLO_OPT_BATCH_GRAPH

  ! zolo_set_option options (values as in include/zolo_b200.h)
  integer(c_int), parameter :: ZOLO_OPT_SHARED_QR = 1
  integer(c_int), parameter :: ZOLO_OPT_NS_FINISH = 2
  integer(c_int), parameter :: ZOLO_OPT_CHOL_INVERSE = 3
  integer(c_int), parameter :: ZOLO_OPT_BETA_FROB = 4
  integer(c_int), parameter :: ZOLO_OPT_TERM_PLAN = 5
  integer(c_int), parameter :: ZOLO_OPT_MIXED = 6
  integer(c_int), parameter :: ZOLO_OPT_MIXED_SLICES = 7
  integer(c_int), parameter :: ZOLO_OPT_OWN_BOUNDS = 8
  integer(c_int), parameter :: ZOLO_OPT_NORM2_BOUND = 10
  integer(c_int), parameter :: ZOLO_OPT_BATCH_GRAPH = 11

  interface
    ! PZOLOPD1 (pzolopd1.f90:2): Zolo-PD of As/(ALPHA*BETA) with RK <= 8 terms; Q = polar factor.
    subroutine zolo_pzolopd1(sym, rk, m, n, alpha, beta, as, ia, ja, desca, q, iq, jq, descq, info, polar) &
        bind(C, name="zolo_pzolopd1")
      import :: c_char, c_int, c_double
      character(kind=c_char), value :: sym
      integer(c_int), value :: rk, m, n
      real(c_double), value :: alpha, beta
      real(c_double), intent(in) :: as(*)
      integer(c_int), value :: ia, ja
      integer(c_int), intent(in) :: desca(9)
      real(c_double), intent(inout) :: q(*)
      integer(c_int), value :: iq, jq
      integer(c_int), intent(in) :: descq(9)
      integer(c_int), intent(out) :: info
      character(kind=c_char), value :: polar
    end subroutine zolo_pzolopd1

    ! PZOLOPD2 (pzolopd2.f90:2): the PZOLOPD1 contract.
    subroutine zolo_pzolopd2(sym, rk, m, n, alpha, beta, as, ia, ja, desca, q, iq, jq, descq, info, polar) &
        bind(C, name="zolo_pzolopd2")
      import :: c_char, c_int, c_double
      character(kind=c_char), value :: sym
      integer(c_int), value :: rk, m, n
      real(c_double), value :: alpha, beta
      real(c_double), intent(in) :: as(*)
      integer(c_int), value :: ia, ja
      integer(c_int), intent(in) :: desca(9)
      real(c_double), intent(inout) :: q(*)
      integer(c_int), value :: iq, jq
      integer(c_int), intent(in) :: descq(9)
      integer(c_int), intent(out) :: info
      character(kind=c_char), value :: polar
    end subroutine zolo_pzolopd2

    ! PQDWHFACS (pqdwhfacs.f90:2-3): QDWH-PD of A - SIGMA*I; WORK2 = H when POLAR = 'T';
    ! LWORK = -1 or LWORK2 = -1 returns the workspace sizes in WORK(1:2).
    subroutine zolo_pqdwhfacs(sym, m, n, sigma, a, ia, ja, desca, q, iq, jq, descq, work, lwork, descw, &
        tau, work2, lwork2, info, polar) bind(C, name="zolo_pqdwhfacs")
      import :: c_char, c_int, c_double
      character(kind=c_char), value :: sym
      integer(c_int), value :: m, n
      real(c_double), value :: sigma
      real(c_double), intent(in) :: a(*)
      integer(c_int), value :: ia, ja
      integer(c_int), intent(in) :: desca(9)
      real(c_double), intent(inout) :: q(*)
      integer(c_int), value :: iq, jq
      integer(c_int), intent(in) :: descq(9)
      real(c_double), intent(inout) :: work(*)
      integer(c_int), value :: lwork
      integer(c_int), intent(in) :: descw(9)
      real(c_double), intent(inout) :: tau(*), work2(*)
      integer(c_int), value :: lwork2
      integer(c_int), intent(out) :: info
      character(kind=c_char), value :: polar
    end subroutine zolo_pqdwhfacs

    ! ZOLOPD (zolopd.f90:2-3): the older QDWH entry (no SYM argument).
    subroutine zolo_zolopd(m, n, sigma, a, ia, ja, desca, q, iq, jq, descq, work, lwork, descw, &
        tau, work2, lwork2, info, polar) bind(C, name="zolo_zolopd")
      import :: c_char, c_int, c_double
      integer(c_int), value :: m, n
      real(c_double), value :: sigma
      real(c_double), intent(in) :: a(*)
      integer(c_int), value :: ia, ja
      integer(c_int), intent(in) :: desca(9)
      real(c_double), intent(inout) :: q(*)
      integer(c_int), value :: iq, jq
      integer(c_int), intent(in) :: descq(9)
      real(c_double), intent(inout) :: work(*)
      integer(c_int), value :: lwork
      integer(c_int), intent(in) :: descw(9)
      real(c_double), intent(inout) :: tau(*), work2(*)
      integer(c_int), value :: lwork2
      integer(c_int), intent(out) :: info
      character(kind=c_char), value :: polar
    end subroutine zolo_zolopd

    ! ZoloEig (ZoloEig.f90:2): one spectral split of the symmetric As from its polar factor Q.
    subroutine zolo_zoloeig(n, nblk, q, as, contxt, mpi_newcomm, work, lwork, work2, lwork2, tau, info) &
        bind(C, name="zolo_zoloeig")
      import :: c_int, c_double
      integer(c_int), value :: n, nblk
      real(c_double), intent(inout) :: q(*), as(*)
      integer(c_int), value :: contxt, mpi_newcomm
      real(c_double), intent(inout) :: work(*)
      integer(c_int), value :: lwork
      real(c_double), intent(inout) :: work2(*)
      integer(c_int), value :: lwork2
      real(c_double), intent(inout) :: tau(*)
      integer(c_int), intent(out) :: info
    end subroutine zolo_zoloeig

    ! Handles and options (no reference counterpart).
    integer(c_int) function zolo_default_handle(handle) bind(C, name="zolo_default_handle")
      import :: c_int, c_ptr
      type(c_ptr), intent(out) :: handle
    end function zolo_default_handle

    integer(c_int) function zolo_create(device, handle) bind(C, name="zolo_create")
      import :: c_int, c_ptr
      integer(c_int), value :: device
      type(c_ptr), intent(out) :: handle
    end function zolo_create

    integer(c_int) function zolo_destroy(handle) bind(C, name="zolo_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: handle
    end function zolo_destroy

    integer(c_int) function zolo_set_option(handle, option, val) bind(C, name="zolo_set_option")
      import :: c_int, c_ptr
      type(c_ptr), value :: handle
      integer(c_int), value :: option, val
    end function zolo_set_option

    integer(c_int) function zolo_release_workspace(handle) bind(C, name="zolo_release_workspace")
      import :: c_int, c_ptr
      type(c_ptr), value :: handle
    end function zolo_release_workspace

    ! Device arrays (pointers from cudaMalloc or a CUDA Fortran device array's c_devloc).
    integer(c_int) function zolo_polar_dev(handle, rk, m, n, da, lda, dq, ldq, dh, ldh) &
        bind(C, name="zolo_polar_dev")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: handle
      integer(c_int), value :: rk, m, n
      type(c_ptr), value :: da
      integer(c_int64_t), value :: lda
      type(c_ptr), value :: dq
      integer(c_int64_t), value :: ldq
      type(c_ptr), value :: dh
      integer(c_int64_t), value :: ldh
    end function zolo_polar_dev

    integer(c_int) function zolo_pzolopd1_dev(handle, sym, rk, m, n, alpha, beta, da, lda, dq, ldq, dh, ldh) &
        bind(C, name="zolo_pzolopd1_dev")
      import :: c_int, c_ptr, c_int64_t, c_char, c_double
      type(c_ptr), value :: handle
      character(kind=c_char), value :: sym
      integer(c_int), value :: rk, m, n
      real(c_double), value :: alpha, beta
      type(c_ptr), value :: da
      integer(c_int64_t), value :: lda
      type(c_ptr), value :: dq
      integer(c_int64_t), value :: ldq
      type(c_ptr), value :: dh
      integer(c_int64_t), value :: ldh
    end function zolo_pzolopd1_dev

    integer(c_int) function zolo_qdwh_dev(handle, sym, m, n, sigma, da, lda, dq, ldq, dh, ldh, bounds_mode, &
        maxit, left_solve) bind(C, name="zolo_qdwh_dev")
      import :: c_int, c_ptr, c_int64_t, c_char, c_double
      type(c_ptr), value :: handle
      character(kind=c_char), value :: sym
      integer(c_int), value :: m, n
      real(c_double), value :: sigma
      type(c_ptr), value :: da
      integer(c_int64_t), value :: lda
      type(c_ptr), value :: dq
      integer(c_int64_t), value :: ldq
      type(c_ptr), value :: dh
      integer(c_int64_t), value :: ldh
      integer(c_int), value :: bounds_mode, maxit, left_solve
    end function zolo_qdwh_dev
  end interface
end module zolo_b200
