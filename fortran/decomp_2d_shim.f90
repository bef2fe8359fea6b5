! One-rank (1 x 1) stand-in for the four 2decomp&FFT modules the reference
! host uses, for a build whose hot path runs on the B200 library:
!   decomp_2d_constants  mytype, real_type (src/mom.f90:9, src/navier.f90:102)
!   decomp_2d_mpi        nrank, nproc, decomp_2d_abort, decomp_2d_warning
!                        (src/x3d_tools.f90:62, src/mom.f90:10)
!   decomp_2d            decomp_info, the pencil sizes and starts, ph1..phG,
!                        decomp_2d_init/finalize, decomp_info_init/finalize,
!                        init_coarser_mesh_stat*, alloc_x/y/z, transpose_*
!                        (src/x3d_tools.f90:83-87,168-186,215-243,
!                        src/var.f90:43-46, src/navier.f90:105-111,171-190)
!   decomp_2d_fft        decomp_2d_fft_init/3d/finalize (src/poisson.f90:11-13)
! With one rank every pencil is the whole box with x fastest (xsize = ysize
! = zsize), so a transpose is a copy of the same array, and the distributed
! FFT is not needed: the B200 build points poisson at poisson_b200
! (x3d_b200_derive.f90), which solves on the device.  A process grid other
! than 1 x 1 stops in decomp_2d_init: for several ranks keep 2decomp&FFT and
! call the library per pencil (x3d_poisson_zpencil, lines never split).
!
! Preprocessed Fortran (__FILE__, __LINE__, DOUBLE_PREC), as the reference's
! own sources.  Not compiled in this repository's image: it has no Fortran
! compiler.

module decomp_2d_constants
  use mpi, only : MPI_DOUBLE_PRECISION, MPI_REAL, MPI_DOUBLE_COMPLEX, MPI_COMPLEX
  implicit none
#ifdef DOUBLE_PREC
  integer, parameter :: mytype = kind(0.0d0)
  integer, parameter :: real_type = MPI_DOUBLE_PRECISION
  integer, parameter :: complex_type = MPI_DOUBLE_COMPLEX
#else
  integer, parameter :: mytype = kind(0.0)
  integer, parameter :: real_type = MPI_REAL
  integer, parameter :: complex_type = MPI_COMPLEX
#endif
  ! which pencil holds physical space for the 3-D FFT (2decomp's values)
  integer, parameter :: PHYSICAL_IN_X = 1, PHYSICAL_IN_Z = 3
end module decomp_2d_constants


module decomp_2d_mpi
  use mpi
  implicit none
  ! set by the host (src/x3d_tools.f90:71-74)
  integer, save :: nrank = 0, nproc = 1

  interface decomp_2d_abort
     module procedure abort_at, abort_code
  end interface decomp_2d_abort
  interface decomp_2d_warning
     module procedure warning_at, warning_code
  end interface decomp_2d_warning

contains

  subroutine abort_at(file, line, errorcode, msg)
    character(len=*), intent(in) :: file, msg
    integer, intent(in) :: line, errorcode
    integer :: ierr
    write(*, '(a, ":", i0, ": error ", i0, ": ", a)') file, line, errorcode, msg
    call MPI_ABORT(MPI_COMM_WORLD, errorcode, ierr)
    stop 1
  end subroutine abort_at

  subroutine abort_code(errorcode, msg)
    integer, intent(in) :: errorcode
    character(len=*), intent(in) :: msg
    call abort_at("decomp_2d", 0, errorcode, msg)
  end subroutine abort_code

  subroutine warning_at(file, line, errorcode, msg)
    character(len=*), intent(in) :: file, msg
    integer, intent(in) :: line, errorcode
    write(*, '(a, ":", i0, ": warning ", i0, ": ", a)') file, line, errorcode, msg
  end subroutine warning_at

  subroutine warning_code(errorcode, msg)
    integer, intent(in) :: errorcode
    character(len=*), intent(in) :: msg
    call warning_at("decomp_2d", 0, errorcode, msg)
  end subroutine warning_code

end module decomp_2d_mpi


module decomp_2d
  use decomp_2d_constants, only : mytype
  use decomp_2d_mpi
  implicit none
  private

  ! start, end and size of the X, Y and Z pencils of one decomposition
  type, public :: decomp_info
     integer, dimension(3) :: xst, xen, xsz
     integer, dimension(3) :: yst, yen, ysz
     integer, dimension(3) :: zst, zen, zsz
  end type decomp_info

  integer, save, public :: nx_global = 0, ny_global = 0, nz_global = 0
  integer, save, dimension(3), public :: xstart, xend, xsize
  integer, save, dimension(3), public :: ystart, yend, ysize
  integer, save, dimension(3), public :: zstart, zend, zsize
  type(decomp_info), save, target, public :: decomp_main
  ! the host's own decompositions (src/x3d_tools.f90:173-186)
  type(decomp_info), save, target, public :: ph1, ph2, ph3, phG

  public :: decomp_2d_init, decomp_2d_finalize, decomp_info_init, decomp_info_finalize
  public :: init_coarser_mesh_statS, init_coarser_mesh_statV, init_coarser_mesh_statP
  public :: alloc_x, alloc_y, alloc_z
  public :: transpose_x_to_y, transpose_y_to_z, transpose_z_to_y, transpose_y_to_x

  interface alloc_x
     module procedure alloc_x_real, alloc_x_cplx
  end interface alloc_x
  interface alloc_y
     module procedure alloc_y_real, alloc_y_cplx
  end interface alloc_y
  interface alloc_z
     module procedure alloc_z_real, alloc_z_cplx
  end interface alloc_z
  ! at 1 x 1 the four transposes are one copy
  interface transpose_x_to_y
     module procedure copy_real, copy_cplx
  end interface transpose_x_to_y
  interface transpose_y_to_z
     module procedure copy_real, copy_cplx
  end interface transpose_y_to_z
  interface transpose_z_to_y
     module procedure copy_real, copy_cplx
  end interface transpose_z_to_y
  interface transpose_y_to_x
     module procedure copy_real, copy_cplx
  end interface transpose_y_to_x

contains

  subroutine decomp_2d_init(nx, ny, nz, p_row, p_col)
    integer, intent(in) :: nx, ny, nz, p_row, p_col
    if (p_row * p_col > 1 .or. nproc > 1) &
         call decomp_2d_abort(__FILE__, __LINE__, p_row * p_col, &
         "the 1 x 1 decomp_2d shim runs one rank; use 2decomp&FFT for a process grid")
    nx_global = nx
    ny_global = ny
    nz_global = nz
    call decomp_info_init(nx, ny, nz, decomp_main)
    xstart = decomp_main%xst
    xend = decomp_main%xen
    xsize = decomp_main%xsz
    ystart = decomp_main%yst
    yend = decomp_main%yen
    ysize = decomp_main%ysz
    zstart = decomp_main%zst
    zend = decomp_main%zen
    zsize = decomp_main%zsz
  end subroutine decomp_2d_init

  subroutine decomp_2d_finalize()
  end subroutine decomp_2d_finalize

  ! Every pencil of an nx x ny x nz decomposition on one rank: the whole box.
  subroutine decomp_info_init(nx, ny, nz, decomp)
    integer, intent(in) :: nx, ny, nz
    type(decomp_info), intent(inout) :: decomp
    decomp%xst = 1
    decomp%yst = 1
    decomp%zst = 1
    decomp%xsz = (/ nx, ny, nz /)
    decomp%ysz = decomp%xsz
    decomp%zsz = decomp%xsz
    decomp%xen = decomp%xsz
    decomp%yen = decomp%xsz
    decomp%zen = decomp%xsz
  end subroutine decomp_info_init

  subroutine decomp_info_finalize(decomp)
    type(decomp_info), intent(inout) :: decomp
    decomp%xsz = 0
    decomp%ysz = 0
    decomp%zsz = 0
  end subroutine decomp_info_finalize

  ! Coarser meshes for statistics, visualisation and probes are not on the
  ! hot path; nothing to set up on one rank.
  subroutine init_coarser_mesh_statS(i_skip, j_skip, k_skip, from1)
    integer, intent(in) :: i_skip, j_skip, k_skip
    logical, intent(in) :: from1
  end subroutine init_coarser_mesh_statS

  subroutine init_coarser_mesh_statV(i_skip, j_skip, k_skip, from1)
    integer, intent(in) :: i_skip, j_skip, k_skip
    logical, intent(in) :: from1
  end subroutine init_coarser_mesh_statV

  subroutine init_coarser_mesh_statP(i_skip, j_skip, k_skip, from1)
    integer, intent(in) :: i_skip, j_skip, k_skip
    logical, intent(in) :: from1
  end subroutine init_coarser_mesh_statP

  ! The decomposition a call names, else the main one.  Local and global
  ! indices coincide on one rank, so opt_global changes nothing.
  function pick(opt_decomp) result(d)
    type(decomp_info), intent(in), optional :: opt_decomp
    type(decomp_info) :: d
    if (present(opt_decomp)) then
       d = opt_decomp
    else
       d = decomp_main
    end if
  end function pick

  subroutine alloc_x_real(var, opt_decomp, opt_global)
    real(mytype), allocatable, dimension(:,:,:) :: var
    type(decomp_info), intent(in), optional :: opt_decomp
    logical, intent(in), optional :: opt_global
    type(decomp_info) :: d
    d = pick(opt_decomp)
    allocate(var(d%xst(1):d%xen(1), d%xst(2):d%xen(2), d%xst(3):d%xen(3)))
  end subroutine alloc_x_real

  subroutine alloc_x_cplx(var, opt_decomp, opt_global)
    complex(mytype), allocatable, dimension(:,:,:) :: var
    type(decomp_info), intent(in), optional :: opt_decomp
    logical, intent(in), optional :: opt_global
    type(decomp_info) :: d
    d = pick(opt_decomp)
    allocate(var(d%xst(1):d%xen(1), d%xst(2):d%xen(2), d%xst(3):d%xen(3)))
  end subroutine alloc_x_cplx

  subroutine alloc_y_real(var, opt_decomp, opt_global)
    real(mytype), allocatable, dimension(:,:,:) :: var
    type(decomp_info), intent(in), optional :: opt_decomp
    logical, intent(in), optional :: opt_global
    type(decomp_info) :: d
    d = pick(opt_decomp)
    allocate(var(d%yst(1):d%yen(1), d%yst(2):d%yen(2), d%yst(3):d%yen(3)))
  end subroutine alloc_y_real

  subroutine alloc_y_cplx(var, opt_decomp, opt_global)
    complex(mytype), allocatable, dimension(:,:,:) :: var
    type(decomp_info), intent(in), optional :: opt_decomp
    logical, intent(in), optional :: opt_global
    type(decomp_info) :: d
    d = pick(opt_decomp)
    allocate(var(d%yst(1):d%yen(1), d%yst(2):d%yen(2), d%yst(3):d%yen(3)))
  end subroutine alloc_y_cplx

  subroutine alloc_z_real(var, opt_decomp, opt_global)
    real(mytype), allocatable, dimension(:,:,:) :: var
    type(decomp_info), intent(in), optional :: opt_decomp
    logical, intent(in), optional :: opt_global
    type(decomp_info) :: d
    d = pick(opt_decomp)
    allocate(var(d%zst(1):d%zen(1), d%zst(2):d%zen(2), d%zst(3):d%zen(3)))
  end subroutine alloc_z_real

  subroutine alloc_z_cplx(var, opt_decomp, opt_global)
    complex(mytype), allocatable, dimension(:,:,:) :: var
    type(decomp_info), intent(in), optional :: opt_decomp
    logical, intent(in), optional :: opt_global
    type(decomp_info) :: d
    d = pick(opt_decomp)
    allocate(var(d%zst(1):d%zen(1), d%zst(2):d%zen(2), d%zst(3):d%zen(3)))
  end subroutine alloc_z_cplx

  ! A transpose on one rank: the pencils share one layout, so the data
  ! moves unchanged (on the device when the arrays are present there, as in
  ! the reference's OpenACC build).
  subroutine copy_real(src, dst, opt_decomp)
    real(mytype), dimension(:,:,:), intent(in) :: src
    real(mytype), dimension(:,:,:), intent(out) :: dst
    type(decomp_info), intent(in), optional :: opt_decomp
    !$acc kernels default(present)
    dst = src
    !$acc end kernels
  end subroutine copy_real

  subroutine copy_cplx(src, dst, opt_decomp)
    complex(mytype), dimension(:,:,:), intent(in) :: src
    complex(mytype), dimension(:,:,:), intent(out) :: dst
    type(decomp_info), intent(in), optional :: opt_decomp
    !$acc kernels default(present)
    dst = src
    !$acc end kernels
  end subroutine copy_cplx

end module decomp_2d


module decomp_2d_fft
  use decomp_2d_constants, only : mytype, PHYSICAL_IN_X, PHYSICAL_IN_Z
  use decomp_2d_mpi, only : decomp_2d_abort
  implicit none
  private
  public :: decomp_2d_fft_init, decomp_2d_fft_3d, decomp_2d_fft_finalize

  interface decomp_2d_fft_3d
     module procedure fft_r2c, fft_c2r
  end interface decomp_2d_fft_3d

contains

  subroutine decomp_2d_fft_init(pencil)
    integer, intent(in), optional :: pencil
  end subroutine decomp_2d_fft_init

  subroutine decomp_2d_fft_finalize()
  end subroutine decomp_2d_fft_finalize

  ! poisson_000 is the only caller (src/poisson.f90:325,412); the B200 build
  ! replaces it with poisson_b200, so reaching these is a set-up error.
  subroutine fft_r2c(in_r, out_c)
    real(mytype), dimension(:,:,:), intent(in) :: in_r
    complex(mytype), dimension(:,:,:), intent(out) :: out_c
    call decomp_2d_abort(__FILE__, __LINE__, -1, &
         "no 3-D FFT in the 1 x 1 shim: point poisson at poisson_b200 (x3d_b200_repoint)")
  end subroutine fft_r2c

  subroutine fft_c2r(in_c, out_r)
    complex(mytype), dimension(:,:,:), intent(inout) :: in_c
    real(mytype), dimension(:,:,:), intent(out) :: out_r
    call decomp_2d_abort(__FILE__, __LINE__, -1, &
         "no 3-D FFT in the 1 x 1 shim: point poisson at poisson_b200 (x3d_b200_repoint)")
  end subroutine fft_c2r

end module decomp_2d_fft
