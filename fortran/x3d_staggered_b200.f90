! Drop-in for the reference's module x3d_staggered (src/x3d_staggered.f90):
! the same module name and the same twelve public routines with the same
! argument lists, each one call of the B200 library's routine of that name.
! Build this file instead of src/x3d_staggered.f90; navier.f90 and the other
! callers stay unchanged.  The operator argument is not consulted: the
! library's built-in instance of the routine's operator is used (the
! reference binds exactly one instance to each routine,
! src/x3d_operator_1d.f90:90-130), and the sizes pass through in the
! routine's own order (nx, nxm, ... as in the reference).  Fields are passed
! by address as in x3d_b200_derive.f90 (device addresses under OpenACC).
!
! Preprocessed Fortran, as the reference's own sources.  Not compiled in
! this repository's image: it has no Fortran compiler.

module x3d_staggered

  use iso_c_binding
  use decomp_2d_constants, only : mytype
  use x3d_operator_1d, only : x3doperator1d
  use x3d_b200_bind

  implicit none

  private
  public :: derxvp, interxvp, derxpv, interxpv
  public :: interyvp, deryvp, interypv, derypv
  public :: derzvp, interzvp, derzpv, interzpv

contains

  ! ---- x (src/x3d_staggered.f90:23-404) -------------------------------------

  subroutine derxvp(tx, ux, x3dop, nx, nxm, ny, nz)
    integer, intent(in) :: nx, nxm, ny, nz
    real(mytype), intent(out), dimension(nxm,ny,nz) :: tx
    real(mytype), intent(in), dimension(nx,ny,nz) :: ux
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_DERXVP, tx, ux, nx, nxm, ny, nz)
  end subroutine derxvp

  subroutine interxvp(tx, ux, x3dop, nx, nxm, ny, nz)
    integer, intent(in) :: nx, nxm, ny, nz
    real(mytype), intent(out), dimension(nxm,ny,nz) :: tx
    real(mytype), intent(in), dimension(nx,ny,nz) :: ux
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_INTXVP, tx, ux, nx, nxm, ny, nz)
  end subroutine interxvp

  subroutine derxpv(tx, ux, x3dop, nxm, nx, ny, nz)
    integer, intent(in) :: nx, nxm, ny, nz
    real(mytype), intent(out), dimension(nx,ny,nz) :: tx
    real(mytype), intent(in), dimension(nxm,ny,nz) :: ux
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_DERXPV, tx, ux, nxm, nx, ny, nz)
  end subroutine derxpv

  subroutine interxpv(tx, ux, x3dop, nxm, nx, ny, nz)
    integer, intent(in) :: nx, nxm, ny, nz
    real(mytype), intent(out), dimension(nx,ny,nz) :: tx
    real(mytype), intent(in), dimension(nxm,ny,nz) :: ux
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_INTXPV, tx, ux, nxm, nx, ny, nz)
  end subroutine interxpv

  ! ---- y (:408-883); deryvp and derypv take the stretching metric ------------

  subroutine interyvp(ty, uy, x3dop, nx, ny, nym, nz)
    integer, intent(in) :: nx, ny, nym, nz
    real(mytype), intent(out), dimension(nx,nym,nz) :: ty
    real(mytype), intent(in), dimension(nx,ny,nz) :: uy
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_INTYVP, ty, uy, nx, ny, nym, nz)
  end subroutine interyvp

  subroutine deryvp(ty, uy, x3dop, ppyi, nx, ny, nym, nz)
    integer, intent(in) :: nx, ny, nym, nz
    real(mytype), intent(out), dimension(nx,nym,nz) :: ty
    real(mytype), intent(in), dimension(nx,ny,nz) :: uy
    real(mytype), intent(in), dimension(nym) :: ppyi
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_DERYVP, ty, uy, nx, ny, nym, nz, ppyi, nym)
  end subroutine deryvp

  subroutine interypv(ty, uy, x3dop, nx, nym, ny, nz)
    integer, intent(in) :: nx, ny, nym, nz
    real(mytype), intent(out), dimension(nx,ny,nz) :: ty
    real(mytype), intent(in), dimension(nx,nym,nz) :: uy
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_INTYPV, ty, uy, nx, nym, ny, nz)
  end subroutine interypv

  subroutine derypv(ty, uy, x3dop, ppy, nx, nym, ny, nz)
    integer, intent(in) :: nx, ny, nym, nz
    real(mytype), intent(out), dimension(nx,ny,nz) :: ty
    real(mytype), intent(in), dimension(nx,nym,nz) :: uy
    real(mytype), intent(in), dimension(ny) :: ppy
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_DERYPV, ty, uy, nx, nym, ny, nz, ppy, ny)
  end subroutine derypv

  ! ---- z (:887-1383) ---------------------------------------------------------

  subroutine derzvp(tz, uz, x3dop, nx, ny, nz, nzm)
    integer, intent(in) :: nx, ny, nz, nzm
    real(mytype), intent(out), dimension(nx,ny,nzm) :: tz
    real(mytype), intent(in), dimension(nx,ny,nz) :: uz
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_DERZVP, tz, uz, nx, ny, nz, nzm)
  end subroutine derzvp

  subroutine interzvp(tz, uz, x3dop, nx, ny, nz, nzm)
    integer, intent(in) :: nx, ny, nz, nzm
    real(mytype), intent(out), dimension(nx,ny,nzm) :: tz
    real(mytype), intent(in), dimension(nx,ny,nz) :: uz
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_INTZVP, tz, uz, nx, ny, nz, nzm)
  end subroutine interzvp

  subroutine derzpv(tz, uz, x3dop, nx, ny, nzm, nz)
    integer, intent(in) :: nx, ny, nz, nzm
    real(mytype), intent(out), dimension(nx,ny,nz) :: tz
    real(mytype), intent(in), dimension(nx,ny,nzm) :: uz
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_DERZPV, tz, uz, nx, ny, nzm, nz)
  end subroutine derzpv

  subroutine interzpv(tz, uz, x3dop, nx, ny, nzm, nz)
    integer, intent(in) :: nx, ny, nz, nzm
    real(mytype), intent(out), dimension(nx,ny,nz) :: tz
    real(mytype), intent(in), dimension(nx,ny,nzm) :: uz
    type(x3doperator1d), intent(in) :: x3dop
    call stag(X3D_OP_INTZPV, tz, uz, nx, ny, nzm, nz)
  end subroutine interzpv

  ! ---- the one helper: sizes s1 .. s4 in the routine's own order -------------

  subroutine stag(which, t, u, s1, s2, s3, s4, pp, npp)
    use param, only : istret
    integer(c_int), intent(in) :: which
    real(mytype), intent(out), dimension(*), target :: t
    real(mytype), intent(in), dimension(*), target :: u
    integer, intent(in) :: s1, s2, s3, s4
    real(mytype), intent(in), dimension(*), optional :: pp
    integer, intent(in), optional :: npp
    real(c_double), allocatable, target :: metric(:)
    type(c_ptr) :: op, pm, tp, up
    integer(c_int) :: rc
    call x3d_check(x3d_op_builtin(x3d_ctx, which, op), "x3d_op_builtin")
    pm = c_null_ptr
    if (present(pp) .and. istret /= 0) then
       allocate(metric(npp))
       metric = real(pp(1:npp), c_double)  ! a host copy in FP64: the library reads either
       pm = c_loc(metric)
    end if
    !$acc host_data use_device(t, u)
    tp = c_loc(t(1))
    up = c_loc(u(1))
    !$acc end host_data
    select case (which)
    case (X3D_OP_DERXVP)
       rc = x3d_derxvp(x3d_ctx, tp, up, op, s1, s2, s3, s4)
    case (X3D_OP_INTXVP)
       rc = x3d_interxvp(x3d_ctx, tp, up, op, s1, s2, s3, s4)
    case (X3D_OP_DERXPV)
       rc = x3d_derxpv(x3d_ctx, tp, up, op, s1, s2, s3, s4)
    case (X3D_OP_INTXPV)
       rc = x3d_interxpv(x3d_ctx, tp, up, op, s1, s2, s3, s4)
    case (X3D_OP_INTYVP)
       rc = x3d_interyvp(x3d_ctx, tp, up, op, s1, s2, s3, s4)
    case (X3D_OP_DERYVP)
       rc = x3d_deryvp(x3d_ctx, tp, up, op, pm, s1, s2, s3, s4)
    case (X3D_OP_INTYPV)
       rc = x3d_interypv(x3d_ctx, tp, up, op, s1, s2, s3, s4)
    case (X3D_OP_DERYPV)
       rc = x3d_derypv(x3d_ctx, tp, up, op, pm, s1, s2, s3, s4)
    case (X3D_OP_DERZVP)
       rc = x3d_derzvp(x3d_ctx, tp, up, op, s1, s2, s3, s4)
    case (X3D_OP_INTZVP)
       rc = x3d_interzvp(x3d_ctx, tp, up, op, s1, s2, s3, s4)
    case (X3D_OP_DERZPV)
       rc = x3d_derzpv(x3d_ctx, tp, up, op, s1, s2, s3, s4)
    case default
       rc = x3d_interzpv(x3d_ctx, tp, up, op, s1, s2, s3, s4)
    end select
    call x3d_check(rc, "staggered routine")
    if (allocated(metric)) deallocate(metric)
  end subroutine stag

end module x3d_staggered
