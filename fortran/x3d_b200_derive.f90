! The B200 library at the reference host's own plug-in points:
!   - the derivative pointers derx, dery, derz (src/x3d_derive.f90:54-59,
!     bound to derx_00 ... in x3d_derive_init, :66-93), re-pointed to
!     derx_b200, dery_b200, derz_b200 with the same abstract interfaces
!     (DERIVATIVE_X/Y/Z, :19-52);
!   - the second-derivative pointers derxx, deryy, derzz, which the reference
!     declares and never binds (:54-59, empty block :91-92);
!   - the Poisson pointer (src/poisson.f90:57-65, bound to poisson_000 at
!     :104-105), re-pointed to poisson_b200.
! The staggered routines are module procedures, not pointers: their drop-in
! is x3d_staggered_b200.f90, a module of the same name built instead of
! src/x3d_staggered.f90.
!
! Fields stay where the host keeps them.  In the reference's OpenACC build
! they are device-resident inside !$acc data regions
! (src/xcompact3d.f90:43-72), so each call passes their device addresses
! (!$acc host_data use_device); in a host build without OpenACC the library
! stages host arrays itself (or keeps mirrors, x3d_buf_register).
!
! c_loc needs the TARGET attribute, which is a characteristic of a dummy
! argument: the public routines keep the reference's interfaces exactly (so
! the procedure-pointer assignments are legal) and pass their arrays on to
! private helpers whose dummies are targets.
!
! Preprocessed Fortran, as the reference's own sources.  Not compiled in
! this repository's image: it has no Fortran compiler.

module x3d_b200_derive
  use iso_c_binding
  use decomp_2d_constants, only : mytype
  use x3d_operator_1d, only : x3doperator1d
  use x3d_b200_bind
  implicit none
  private

  public :: x3d_b200_setup, x3d_b200_teardown, x3d_b200_repoint
  public :: derx_b200, dery_b200, derz_b200, derxx_b200, deryy_b200, derzz_b200
  public :: poisson_b200

contains

  ! Creates the library context for the host's box (the global grid: lines
  ! are never split), its boundary conditions and its precision, on device
  ! `device` (the one the host's OpenACC runtime uses).  Call after
  ! init_xcompact3d has read the parameters (src/x3d_tools.f90:163-185).
  subroutine x3d_b200_setup(device)
    use variables, only : nx, ny, nz
    use param, only : xlx, yly, zlz, nclx1, nclxn, ncly1, nclyn, nclz1, nclzn
    integer, intent(in) :: device
    integer(c_int), target :: ncl(6)
    integer(c_int) :: prec
    if (kind(0.0_mytype) == c_double) then
       prec = X3D_F64
    else
       prec = X3D_F32
    end if
    ncl = (/ nclx1, nclxn, ncly1, nclyn, nclz1, nclzn /)
    call x3d_check(x3d_ctx_create_bc(x3d_ctx, int(nx, c_int), int(ny, c_int), int(nz, c_int), &
         real(xlx, c_double), real(yly, c_double), real(zlz, c_double), prec, int(device, c_int), ncl), &
         "x3d_ctx_create_bc")
  end subroutine x3d_b200_setup

  subroutine x3d_b200_teardown()
    if (c_associated(x3d_ctx)) call x3d_check(x3d_ctx_destroy(x3d_ctx), "x3d_ctx_destroy")
    x3d_ctx = c_null_ptr
  end subroutine x3d_b200_teardown

  ! Binds the pointers to the library: after x3d_derive_init and
  ! decomp_2d_poisson_init, in place of their bindings.
  subroutine x3d_b200_repoint()
    use x3d_derive, only : derx, dery, derz, derxx, deryy, derzz
    use decomp_2d_poisson, only : poisson
    derx => derx_b200
    dery => dery_b200
    derz => derz_b200
    derxx => derxx_b200
    deryy => deryy_b200
    derzz => derzz_b200
    poisson => poisson_b200
  end subroutine x3d_b200_repoint

  ! ---- the reference's interfaces -------------------------------------------

  ! DERIVATIVE_X: derx_00 / derx_ij.  The library's built-in operators are
  ! the reference's instances; x3d_op_derx has npaire 0 and x3d_op_derxp
  ! npaire 1 (src/x3d_operator_1d.f90:78-79), X3D_OP_DERX + npaire.
  subroutine derx_b200(t, u, x3dop, nx, ny, nz)
    integer, intent(in) :: nx, ny, nz
    real(mytype), intent(out), dimension(nx,ny,nz) :: t
    real(mytype), intent(in), dimension(nx,ny,nz) :: u
    type(x3doperator1d), intent(in) :: x3dop
    call first_deriv(X3D_DIR_X, X3D_OP_DERX + x3dop%npaire, t, u, nx, ny, nz)
  end subroutine derx_b200

  ! DERIVATIVE_Y: dery_00 / dery_ij with the stretching metric pp (used when
  ! istret /= 0, src/x3d_derive.f90:331-337).
  subroutine dery_b200(t, u, x3dop, pp, nx, ny, nz)
    integer, intent(in) :: nx, ny, nz
    real(mytype), intent(out), dimension(nx,ny,nz) :: t
    real(mytype), intent(in), dimension(nx,ny,nz) :: u
    real(mytype), intent(in), dimension(ny) :: pp
    type(x3doperator1d), intent(in) :: x3dop
    call first_deriv(X3D_DIR_Y, X3D_OP_DERY + x3dop%npaire, t, u, nx, ny, nz, pp)
  end subroutine dery_b200

  ! DERIVATIVE_Z: derz_00 / derz_ij.
  subroutine derz_b200(t, u, x3dop, nx, ny, nz)
    integer, intent(in) :: nx, ny, nz
    real(mytype), intent(out), dimension(nx,ny,nz) :: t
    real(mytype), intent(in), dimension(nx,ny,nz) :: u
    type(x3doperator1d), intent(in) :: x3dop
    call first_deriv(X3D_DIR_Z, X3D_OP_DERZ + x3dop%npaire, t, u, nx, ny, nz)
  end subroutine derz_b200

  ! DERIVATIVE_X / YY / Z for the second derivatives (periodic): the operator
  ! argument is not consulted, the library's 6th-order compact second
  ! derivative is used.
  subroutine derxx_b200(t, u, x3dop, nx, ny, nz)
    integer, intent(in) :: nx, ny, nz
    real(mytype), intent(out), dimension(nx,ny,nz) :: t
    real(mytype), intent(in), dimension(nx,ny,nz) :: u
    type(x3doperator1d), intent(in) :: x3dop
    call second_deriv(X3D_DIR_X, t, u, nx, ny, nz)
  end subroutine derxx_b200

  subroutine deryy_b200(t, u, x3dop, nx, ny, nz)
    integer, intent(in) :: nx, ny, nz
    real(mytype), intent(out), dimension(nx,ny,nz) :: t
    real(mytype), intent(in), dimension(nx,ny,nz) :: u
    type(x3doperator1d), intent(in) :: x3dop
    call second_deriv(X3D_DIR_Y, t, u, nx, ny, nz)
  end subroutine deryy_b200

  subroutine derzz_b200(t, u, x3dop, nx, ny, nz)
    integer, intent(in) :: nx, ny, nz
    real(mytype), intent(out), dimension(nx,ny,nz) :: t
    real(mytype), intent(in), dimension(nx,ny,nz) :: u
    type(x3doperator1d), intent(in) :: x3dop
    call second_deriv(X3D_DIR_Z, t, u, nx, ny, nz)
  end subroutine derzz_b200

  ! poisson_xxx (src/poisson.f90:57-62): the right-hand side in, the
  ! pressure out, in place.  The library's solve is FP64 (the north-star
  ! precision split), so a single-precision host passes through an FP64 copy.
  subroutine poisson_b200(rhs)
    real(mytype), dimension(:,:,:), intent(inout) :: rhs
#ifdef DOUBLE_PREC
    call poisson_dev(rhs, size(rhs))
#else
    real(c_double), allocatable, dimension(:,:,:) :: r64
    allocate(r64(size(rhs, 1), size(rhs, 2), size(rhs, 3)))
    !$acc data create(r64)
    !$acc kernels default(present)
    r64 = real(rhs, c_double)
    !$acc end kernels
    call poisson_dev(r64, size(r64))
    !$acc kernels default(present)
    rhs = real(r64, mytype)
    !$acc end kernels
    !$acc end data
    deallocate(r64)
#endif
  end subroutine poisson_b200

  ! ---- helpers with target dummies ------------------------------------------

  subroutine first_deriv(dir, which, t, u, nx, ny, nz, pp)
    use param, only : istret
    integer(c_int), intent(in) :: dir, which
    integer, intent(in) :: nx, ny, nz
    real(mytype), intent(out), dimension(nx,ny,nz), target :: t
    real(mytype), intent(in), dimension(nx,ny,nz), target :: u
    real(mytype), intent(in), dimension(ny), optional :: pp
    real(c_double), target :: metric(ny)
    type(c_ptr) :: op, pm
    integer(c_int) :: rc
    call x3d_check(x3d_op_builtin(x3d_ctx, which, op), "x3d_op_builtin")
    pm = c_null_ptr
    if (present(pp) .and. istret /= 0) then
       metric = real(pp, c_double)  ! a host copy in FP64: the library reads either
       pm = c_loc(metric)
    end if
    !$acc host_data use_device(t, u)
    select case (dir)
    case (X3D_DIR_X)
       rc = x3d_derx(x3d_ctx, c_loc(t), c_loc(u), op, nx, ny, nz)
    case (X3D_DIR_Y)
       rc = x3d_dery(x3d_ctx, c_loc(t), c_loc(u), op, pm, nx, ny, nz)
    case default
       rc = x3d_derz(x3d_ctx, c_loc(t), c_loc(u), op, nx, ny, nz)
    end select
    !$acc end host_data
    call x3d_check(rc, "first derivative")
  end subroutine first_deriv

  subroutine second_deriv(dir, t, u, nx, ny, nz)
    integer(c_int), intent(in) :: dir
    integer, intent(in) :: nx, ny, nz
    real(mytype), intent(out), dimension(nx,ny,nz), target :: t
    real(mytype), intent(in), dimension(nx,ny,nz), target :: u
    type(c_ptr) :: op
    integer(c_int) :: rc
    call x3d_check(x3d_op_builtin(x3d_ctx, X3D_OP_DERXX + dir, op), "x3d_op_builtin")
    !$acc host_data use_device(t, u)
    select case (dir)
    case (X3D_DIR_X)
       rc = x3d_derxx(x3d_ctx, c_loc(t), c_loc(u), op, nx, ny, nz)
    case (X3D_DIR_Y)
       rc = x3d_deryy(x3d_ctx, c_loc(t), c_loc(u), op, nx, ny, nz)
    case default
       rc = x3d_derzz(x3d_ctx, c_loc(t), c_loc(u), op, nx, ny, nz)
    end select
    !$acc end host_data
    call x3d_check(rc, "second derivative")
  end subroutine second_deriv

  subroutine poisson_dev(rhs, n)
    integer, intent(in) :: n
    real(c_double), dimension(n), target :: rhs
    integer(c_int) :: rc
    !$acc host_data use_device(rhs)
    rc = x3d_poisson(x3d_ctx, c_loc(rhs))
    !$acc end host_data
    call x3d_check(rc, "poisson")
  end subroutine poisson_dev

end module x3d_b200_derive
