! ISO_C_BINDING module of the B200 hot-path library (include/x3d_b200.h).
! Written by fortran/gen_bind.py from the header; do not edit by hand.
! Not compiled in this repository's image (it has no Fortran compiler).
module x3d_b200_bind
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: X3D_OK = 0
  integer(c_int), parameter :: X3D_EINVAL = -1
  integer(c_int), parameter :: X3D_EUNSUPPORTED = -2
  integer(c_int), parameter :: X3D_ECUDA = -3
  integer(c_int), parameter :: X3D_ENOMEM = -4
  integer(c_int), parameter :: X3D_ETIMEOUT = -5
  integer(c_int), parameter :: X3D_F64 = 0
  integer(c_int), parameter :: X3D_F32 = 1
  integer(c_int), parameter :: X3D_DIR_X = 0
  integer(c_int), parameter :: X3D_DIR_Y = 1
  integer(c_int), parameter :: X3D_DIR_Z = 2
  integer(c_int), parameter :: X3D_KIND_DER = 0
  integer(c_int), parameter :: X3D_KIND_DER2 = 1
  integer(c_int), parameter :: X3D_KIND_DERVP = 2
  integer(c_int), parameter :: X3D_KIND_DERPV = 3
  integer(c_int), parameter :: X3D_KIND_INTVP = 4
  integer(c_int), parameter :: X3D_KIND_INTPV = 5
  integer(c_int), parameter :: X3D_OP_DERX = 0
  integer(c_int), parameter :: X3D_OP_DERXP = 1
  integer(c_int), parameter :: X3D_OP_DERY = 2
  integer(c_int), parameter :: X3D_OP_DERYP = 3
  integer(c_int), parameter :: X3D_OP_DERZ = 4
  integer(c_int), parameter :: X3D_OP_DERZP = 5
  integer(c_int), parameter :: X3D_OP_DERXVP = 6
  integer(c_int), parameter :: X3D_OP_DERYVP = 7
  integer(c_int), parameter :: X3D_OP_DERZVP = 8
  integer(c_int), parameter :: X3D_OP_DERXPV = 9
  integer(c_int), parameter :: X3D_OP_DERYPV = 10
  integer(c_int), parameter :: X3D_OP_DERZPV = 11
  integer(c_int), parameter :: X3D_OP_INTXVP = 12
  integer(c_int), parameter :: X3D_OP_INTYVP = 13
  integer(c_int), parameter :: X3D_OP_INTZVP = 14
  integer(c_int), parameter :: X3D_OP_INTXPV = 15
  integer(c_int), parameter :: X3D_OP_INTYPV = 16
  integer(c_int), parameter :: X3D_OP_INTZPV = 17
  integer(c_int), parameter :: X3D_OP_DERXX = 18
  integer(c_int), parameter :: X3D_OP_DERYY = 19
  integer(c_int), parameter :: X3D_OP_DERZZ = 20
  integer(c_int), parameter :: X3D_OP_COUNT = 21
  integer(c_int), parameter :: X3D_NOALLOC_MAX_POINTS = 262144

  ! the structs the entry points take by address (pass c_loc of an array of them)
  type, bind(C) :: x3d_work
     type(c_ptr) :: op
     type(c_ptr) :: src
     type(c_ptr) :: dst
  end type x3d_work
  type, bind(C) :: x3d_box
     integer(c_int) :: nx
     integer(c_int) :: ny
     integer(c_int) :: nz
     real(c_double) :: xlx
     real(c_double) :: yly
     real(c_double) :: zlz
  end type x3d_box
  type, bind(C) :: x3d_block
     integer(c_long_long) :: src_offset
     integer(c_long_long) :: dst_offset
     integer(c_int) :: nx
     integer(c_int) :: ny
     integer(c_int) :: nz
     integer(c_long_long) :: src_ystride
     integer(c_long_long) :: src_zstride
     integer(c_long_long) :: dst_ystride
     integer(c_long_long) :: dst_zstride
  end type x3d_block

  ! the context the re-pointed routines use (x3d_b200_derive.f90)
  type(c_ptr), save :: x3d_ctx = c_null_ptr

  interface
     integer(c_int) function x3d_ctx_create(ctx, nx, ny, nz, xlx, yly, zlz, prec, &
          device) bind(C, name="x3d_ctx_create")
       import :: c_ptr, c_int, c_double
       type(c_ptr) :: ctx
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
       real(c_double), value :: xlx
       real(c_double), value :: yly
       real(c_double), value :: zlz
       integer(c_int), value :: prec
       integer(c_int), value :: device
     end function
     integer(c_int) function x3d_ctx_create_bc(ctx, nx, ny, nz, xlx, yly, zlz, prec, device, &
          ncl) bind(C, name="x3d_ctx_create_bc")
       import :: c_ptr, c_int, c_double
       type(c_ptr) :: ctx
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
       real(c_double), value :: xlx
       real(c_double), value :: yly
       real(c_double), value :: zlz
       integer(c_int), value :: prec
       integer(c_int), value :: device
       integer(c_int) :: ncl(*)
     end function
     integer(c_int) function x3d_ctx_destroy(ctx) bind(C, name="x3d_ctx_destroy")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
     end function
     integer(c_int) function x3d_ctx_set_stream(ctx, stream) bind(C, name="x3d_ctx_set_stream")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: stream
     end function
     integer(c_int) function x3d_ctx_get_stream(ctx, stream) bind(C, name="x3d_ctx_get_stream")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr) :: stream
     end function
     integer(c_int) function x3d_ctx_sync(ctx) bind(C, name="x3d_ctx_sync")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
     end function
     integer(c_int) function x3d_ctx_selftest_timeout(ctx, limit_s) bind(C, &
          name="x3d_ctx_selftest_timeout")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: ctx
       real(c_double), value :: limit_s
     end function
     integer(c_int) function x3d_roofline_probe(ctx, pattern, w, ctas_per_sm, src, outs, nx, &
          ny, nz) bind(C, name="x3d_roofline_probe")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int), value :: pattern
       integer(c_int), value :: w
       integer(c_int), value :: ctas_per_sm
       type(c_ptr), value :: src
       type(c_ptr) :: outs(*)
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     type(c_ptr) function x3d_ctx_last_error(ctx) bind(C, name="x3d_ctx_last_error")
       import :: c_ptr
       type(c_ptr), value :: ctx
     end function
     integer(c_int) function x3d_ctx_launch_count(ctx, cnt) bind(C, name="x3d_ctx_launch_count")
       import :: c_ptr, c_int, c_long_long
       type(c_ptr), value :: ctx
       integer(c_long_long) :: cnt
     end function
     integer(c_int) function x3d_ctx_last_kernel(ctx, cfg) bind(C, name="x3d_ctx_last_kernel")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int) :: cfg
     end function
     integer(c_int) function x3d_ctx_geometry(ctx, dims, lengths, spacing, prec) bind(C, &
          name="x3d_ctx_geometry")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int) :: dims(*)
       type(c_ptr), value :: lengths
       type(c_ptr), value :: spacing
       integer(c_int) :: prec
     end function
     integer(c_int) function x3d_op_builtin(ctx, which, op) bind(C, name="x3d_op_builtin")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int), value :: which
       type(c_ptr) :: op
     end function
     integer(c_int) function x3d_op_create(ctx, op_kind, dir, n, npaire, alfa, f, s, w, &
          periodic, rhs, op) bind(C, name="x3d_op_create")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: op_kind
       integer(c_int), value :: dir
       integer(c_int), value :: n
       integer(c_int), value :: npaire
       real(c_double), value :: alfa
       type(c_ptr), value :: f
       type(c_ptr), value :: s
       type(c_ptr), value :: w
       type(c_ptr), value :: periodic
       type(c_ptr), value :: rhs
       type(c_ptr) :: op
     end function
     integer(c_int) function x3d_op_destroy(ctx, op) bind(C, name="x3d_op_destroy")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: op
     end function
     integer(c_int) function x3d_op_info(op, meta, scal, f, s, w, periodic) bind(C, &
          name="x3d_op_info")
       import :: c_ptr, c_int
       type(c_ptr), value :: op
       integer(c_int) :: meta(*)
       type(c_ptr), value :: scal
       type(c_ptr), value :: f
       type(c_ptr), value :: s
       type(c_ptr), value :: w
       type(c_ptr), value :: periodic
     end function
     integer(c_int) function x3d_derx(ctx, tx, ux, op, nx, ny, nz) bind(C, name="x3d_derx")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tx
       type(c_ptr), value :: ux
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_dery(ctx, ty, uy, op, ppy, nx, ny, nz) bind(C, name="x3d_dery")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: ty
       type(c_ptr), value :: uy
       type(c_ptr), value :: op
       type(c_ptr), value :: ppy
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_derz(ctx, tz, uz, op, nx, ny, nz) bind(C, name="x3d_derz")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tz
       type(c_ptr), value :: uz
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_derxx(ctx, tx, ux, op, nx, ny, nz) bind(C, name="x3d_derxx")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tx
       type(c_ptr), value :: ux
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_deryy(ctx, ty, uy, op, nx, ny, nz) bind(C, name="x3d_deryy")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: ty
       type(c_ptr), value :: uy
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_derzz(ctx, tz, uz, op, nx, ny, nz) bind(C, name="x3d_derzz")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tz
       type(c_ptr), value :: uz
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_derxvp(ctx, tx, ux, op, nx, nxm, ny, nz) bind(C, &
          name="x3d_derxvp")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tx
       type(c_ptr), value :: ux
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: nxm
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_interxvp(ctx, tx, ux, op, nx, nxm, ny, nz) bind(C, &
          name="x3d_interxvp")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tx
       type(c_ptr), value :: ux
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: nxm
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_derxpv(ctx, tx, ux, op, nxm, nx, ny, nz) bind(C, &
          name="x3d_derxpv")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tx
       type(c_ptr), value :: ux
       type(c_ptr), value :: op
       integer(c_int), value :: nxm
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_interxpv(ctx, tx, ux, op, nxm, nx, ny, nz) bind(C, &
          name="x3d_interxpv")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tx
       type(c_ptr), value :: ux
       type(c_ptr), value :: op
       integer(c_int), value :: nxm
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_interyvp(ctx, ty, uy, op, nx, ny, nym, nz) bind(C, &
          name="x3d_interyvp")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: ty
       type(c_ptr), value :: uy
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nym
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_deryvp(ctx, ty, uy, op, ppyi, nx, ny, nym, nz) bind(C, &
          name="x3d_deryvp")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: ty
       type(c_ptr), value :: uy
       type(c_ptr), value :: op
       type(c_ptr), value :: ppyi
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nym
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_interypv(ctx, ty, uy, op, nx, nym, ny, nz) bind(C, &
          name="x3d_interypv")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: ty
       type(c_ptr), value :: uy
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: nym
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_derypv(ctx, ty, uy, op, ppy, nx, nym, ny, nz) bind(C, &
          name="x3d_derypv")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: ty
       type(c_ptr), value :: uy
       type(c_ptr), value :: op
       type(c_ptr), value :: ppy
       integer(c_int), value :: nx
       integer(c_int), value :: nym
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_derzvp(ctx, tz, uz, op, nx, ny, nz, nzm) bind(C, &
          name="x3d_derzvp")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tz
       type(c_ptr), value :: uz
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
       integer(c_int), value :: nzm
     end function
     integer(c_int) function x3d_interzvp(ctx, tz, uz, op, nx, ny, nz, nzm) bind(C, &
          name="x3d_interzvp")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tz
       type(c_ptr), value :: uz
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
       integer(c_int), value :: nzm
     end function
     integer(c_int) function x3d_derzpv(ctx, tz, uz, op, nx, ny, nzm, nz) bind(C, &
          name="x3d_derzpv")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tz
       type(c_ptr), value :: uz
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nzm
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_interzpv(ctx, tz, uz, op, nx, ny, nzm, nz) bind(C, &
          name="x3d_interzpv")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tz
       type(c_ptr), value :: uz
       type(c_ptr), value :: op
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nzm
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_apply_batch(ctx, items, cnt) bind(C, name="x3d_apply_batch")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: items
       integer(c_int), value :: cnt
     end function
     integer(c_int) function x3d_apply(ctx, op, src, dst) bind(C, name="x3d_apply")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: op
       type(c_ptr), value :: src
       type(c_ptr), value :: dst
     end function
     integer(c_int) function x3d_autotune(ctx, max_group) bind(C, name="x3d_autotune")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int), value :: max_group
     end function
     integer(c_int) function x3d_ctx_set_kernel(ctx, cfg) bind(C, name="x3d_ctx_set_kernel")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int), value :: cfg
     end function
     integer(c_int) function x3d_autotune_choice(ctx, dir, group, cfg) bind(C, &
          name="x3d_autotune_choice")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int), value :: dir
       integer(c_int), value :: group
       integer(c_int) :: cfg
     end function
     integer(c_int) function x3d_autotune_stage_choice(ctx, stage, cfg) bind(C, &
          name="x3d_autotune_stage_choice")
       import :: c_ptr, c_int, c_char
       type(c_ptr), value :: ctx
       character(kind=c_char) :: stage(*)
       integer(c_int) :: cfg
     end function
     integer(c_int) function x3d_ctx_set_stage_choice(ctx, stage, val) bind(C, &
          name="x3d_ctx_set_stage_choice")
       import :: c_ptr, c_int, c_char
       type(c_ptr), value :: ctx
       character(kind=c_char) :: stage(*)
       integer(c_int), value :: val
     end function
     integer(c_int) function x3d_batch_create(batch, boxes, nboxes, prec, device) bind(C, &
          name="x3d_batch_create")
       import :: c_ptr, c_int
       type(c_ptr) :: batch
       type(c_ptr), value :: boxes
       integer(c_int), value :: nboxes
       integer(c_int), value :: prec
       integer(c_int), value :: device
     end function
     integer(c_int) function x3d_batch_destroy(batch) bind(C, name="x3d_batch_destroy")
       import :: c_ptr, c_int
       type(c_ptr), value :: batch
     end function
     integer(c_int) function x3d_batch_set_stream(batch, stream) bind(C, &
          name="x3d_batch_set_stream")
       import :: c_ptr, c_int
       type(c_ptr), value :: batch
       type(c_ptr), value :: stream
     end function
     type(c_ptr) function x3d_batch_last_error(batch) bind(C, name="x3d_batch_last_error")
       import :: c_ptr
       type(c_ptr), value :: batch
     end function
     integer(c_int) function x3d_batch_bind_sweep(batch, nfields, fields, outs, nops) bind(C, &
          name="x3d_batch_bind_sweep")
       import :: c_ptr, c_int
       type(c_ptr), value :: batch
       integer(c_int), value :: nfields
       type(c_ptr) :: fields(*)
       type(c_ptr) :: outs(*)
       integer(c_int), value :: nops
     end function
     integer(c_int) function x3d_batch_run(batch) bind(C, name="x3d_batch_run")
       import :: c_ptr, c_int
       type(c_ptr), value :: batch
     end function
     integer(c_int) function x3d_batch_capture(batch) bind(C, name="x3d_batch_capture")
       import :: c_ptr, c_int
       type(c_ptr), value :: batch
     end function
     integer(c_int) function x3d_batch_replay(batch) bind(C, name="x3d_batch_replay")
       import :: c_ptr, c_int
       type(c_ptr), value :: batch
     end function
     integer(c_int) function x3d_batch_sync(batch) bind(C, name="x3d_batch_sync")
       import :: c_ptr, c_int
       type(c_ptr), value :: batch
     end function
     integer(c_int) function x3d_batch_info(batch, points, tiles, jobs, fallback_jobs) bind(C, &
          name="x3d_batch_info")
       import :: c_ptr, c_int, c_long_long
       type(c_ptr), value :: batch
       integer(c_long_long) :: points
       integer(c_long_long) :: tiles
       integer(c_int) :: jobs
       integer(c_int) :: fallback_jobs
     end function
     integer(c_int) function x3d_batch_autotune(batch) bind(C, name="x3d_batch_autotune")
       import :: c_ptr, c_int
       type(c_ptr), value :: batch
     end function
     integer(c_int) function x3d_batch_choice(batch, box, dir, chunk, lines) bind(C, &
          name="x3d_batch_choice")
       import :: c_ptr, c_int
       type(c_ptr), value :: batch
       integer(c_int), value :: box
       integer(c_int), value :: dir
       integer(c_int) :: chunk
       integer(c_int) :: lines
     end function
     integer(c_int) function x3d_xthomas(ctx, tt, ff, fs, fw, perio, alfa, nx, ny, nz) bind(C, &
          name="x3d_xthomas")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tt
       type(c_ptr), value :: ff
       type(c_ptr), value :: fs
       type(c_ptr), value :: fw
       type(c_ptr), value :: perio
       real(c_double), value :: alfa
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_ythomas(ctx, tt, ff, fs, fw, perio, alfa, nx, ny, nz) bind(C, &
          name="x3d_ythomas")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tt
       type(c_ptr), value :: ff
       type(c_ptr), value :: fs
       type(c_ptr), value :: fw
       type(c_ptr), value :: perio
       real(c_double), value :: alfa
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_zthomas(ctx, tt, ff, fs, fw, perio, alfa, nx, ny, nz) bind(C, &
          name="x3d_zthomas")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: ctx
       type(c_ptr), value :: tt
       type(c_ptr), value :: ff
       type(c_ptr), value :: fs
       type(c_ptr), value :: fw
       type(c_ptr), value :: perio
       real(c_double), value :: alfa
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_transpose_x_to_y(ctx, src, dst, is_complex) bind(C, &
          name="x3d_transpose_x_to_y")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: src
       type(c_ptr), value :: dst
       integer(c_int), value :: is_complex
     end function
     integer(c_int) function x3d_transpose_y_to_z(ctx, src, dst, is_complex) bind(C, &
          name="x3d_transpose_y_to_z")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: src
       type(c_ptr), value :: dst
       integer(c_int), value :: is_complex
     end function
     integer(c_int) function x3d_transpose_z_to_y(ctx, src, dst, is_complex) bind(C, &
          name="x3d_transpose_z_to_y")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: src
       type(c_ptr), value :: dst
       integer(c_int), value :: is_complex
     end function
     integer(c_int) function x3d_transpose_y_to_x(ctx, src, dst, is_complex) bind(C, &
          name="x3d_transpose_y_to_x")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: src
       type(c_ptr), value :: dst
       integer(c_int), value :: is_complex
     end function
     integer(c_int) function x3d_copy_blocks(ctx, dst, src, elem_bytes, blocks, cnt) bind(C, &
          name="x3d_copy_blocks")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: dst
       type(c_ptr), value :: src
       integer(c_int), value :: elem_bytes
       type(c_ptr), value :: blocks
       integer(c_int), value :: cnt
     end function
     integer(c_int) function x3d_poisson(ctx, rhs) bind(C, name="x3d_poisson")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: rhs
     end function
     integer(c_int) function x3d_poisson_zlines(ctx, spec, ny_loc, j0) bind(C, &
          name="x3d_poisson_zlines")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: spec
       integer(c_int), value :: ny_loc
       integer(c_int), value :: j0
     end function
     integer(c_int) function x3d_poisson_zpencil(ctx, spec, nxh_loc, i0, ny_loc, j0) bind(C, &
          name="x3d_poisson_zpencil")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: spec
       integer(c_int), value :: nxh_loc
       integer(c_int), value :: i0
       integer(c_int), value :: ny_loc
       integer(c_int), value :: j0
     end function
     integer(c_int) function x3d_divergence(ctx, pp3, ux1, uy1, uz1, nlock) bind(C, &
          name="x3d_divergence")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: pp3
       type(c_ptr), value :: ux1
       type(c_ptr), value :: uy1
       type(c_ptr), value :: uz1
       integer(c_int), value :: nlock
     end function
     integer(c_int) function x3d_divergence_noalloc(ctx, pp3, ux1, uy1, uz1) bind(C, &
          name="x3d_divergence_noalloc")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: pp3
       type(c_ptr), value :: ux1
       type(c_ptr), value :: uy1
       type(c_ptr), value :: uz1
     end function
     integer(c_int) function x3d_gradp(ctx, px1, py1, pz1, pp3) bind(C, name="x3d_gradp")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: px1
       type(c_ptr), value :: py1
       type(c_ptr), value :: pz1
       type(c_ptr), value :: pp3
     end function
     integer(c_int) function x3d_cor_vel(ctx, ux, uy, uz, px, py, pz) bind(C, &
          name="x3d_cor_vel")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: ux
       type(c_ptr), value :: uy
       type(c_ptr), value :: uz
       type(c_ptr), value :: px
       type(c_ptr), value :: py
       type(c_ptr), value :: pz
     end function
     integer(c_int) function x3d_solve_poisson(ctx, pp3, px1, py1, pz1, ux1, uy1, uz1) bind(C, &
          name="x3d_solve_poisson")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: pp3
       type(c_ptr), value :: px1
       type(c_ptr), value :: py1
       type(c_ptr), value :: pz1
       type(c_ptr), value :: ux1
       type(c_ptr), value :: uy1
       type(c_ptr), value :: uz1
     end function
     integer(c_int) function x3d_div_stats(ctx, pp3, dst) bind(C, name="x3d_div_stats")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: pp3
       type(c_ptr), value :: dst
     end function
     integer(c_int) function x3d_momentum_rhs_eq(ctx, dux1, duy1, duz1, ux1, uy1, uz1) bind(C, &
          name="x3d_momentum_rhs_eq")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: dux1
       type(c_ptr), value :: duy1
       type(c_ptr), value :: duz1
       type(c_ptr), value :: ux1
       type(c_ptr), value :: uy1
       type(c_ptr), value :: uz1
     end function
     integer(c_int) function x3d_int_time(ctx, ux1, uy1, uz1, dux1, duy1, duz1, gdt) bind(C, &
          name="x3d_int_time")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: ctx
       type(c_ptr), value :: ux1
       type(c_ptr), value :: uy1
       type(c_ptr), value :: uz1
       type(c_ptr), value :: dux1
       type(c_ptr), value :: duy1
       type(c_ptr), value :: duz1
       real(c_double), value :: gdt
     end function
     integer(c_int) function x3d_euler_step(ctx, ux1, uy1, uz1, dux1, duy1, duz1, pp3, px1, &
          py1, pz1, dt) bind(C, name="x3d_euler_step")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: ctx
       type(c_ptr), value :: ux1
       type(c_ptr), value :: uy1
       type(c_ptr), value :: uz1
       type(c_ptr), value :: dux1
       type(c_ptr), value :: duy1
       type(c_ptr), value :: duz1
       type(c_ptr), value :: pp3
       type(c_ptr), value :: px1
       type(c_ptr), value :: py1
       type(c_ptr), value :: pz1
       real(c_double), value :: dt
     end function
     integer(c_int) function x3d_step_capture(ctx, ux1, uy1, uz1, dux1, duy1, duz1, pp3, px1, &
          py1, pz1, dt) bind(C, name="x3d_step_capture")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: ctx
       type(c_ptr), value :: ux1
       type(c_ptr), value :: uy1
       type(c_ptr), value :: uz1
       type(c_ptr), value :: dux1
       type(c_ptr), value :: duy1
       type(c_ptr), value :: duz1
       type(c_ptr), value :: pp3
       type(c_ptr), value :: px1
       type(c_ptr), value :: py1
       type(c_ptr), value :: pz1
       real(c_double), value :: dt
     end function
     integer(c_int) function x3d_step_launch(ctx) bind(C, name="x3d_step_launch")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
     end function
     integer(c_int) function x3d_transeq_part(ctx, dir, du, u, add, unew, dt, nx, ny, &
          nz) bind(C, name="x3d_transeq_part")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: dir
       type(c_ptr) :: du(*)
       type(c_ptr) :: u(*)
       type(c_ptr) :: add(*)
       type(c_ptr) :: unew(*)
       real(c_double), value :: dt
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_divergence_part(ctx, dir, dst, src, nx, ny, nz) bind(C, &
          name="x3d_divergence_part")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int), value :: dir
       type(c_ptr) :: dst(*)
       type(c_ptr) :: src(*)
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_gradp_part(ctx, dir, dst, src, ucor, nx, ny, nz) bind(C, &
          name="x3d_gradp_part")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int), value :: dir
       type(c_ptr) :: dst(*)
       type(c_ptr) :: src(*)
       type(c_ptr) :: ucor(*)
       integer(c_int), value :: nx
       integer(c_int), value :: ny
       integer(c_int), value :: nz
     end function
     integer(c_int) function x3d_buf_register(ctx, host, nbytes, dev) bind(C, &
          name="x3d_buf_register")
       import :: c_ptr, c_int, c_size_t
       type(c_ptr), value :: ctx
       type(c_ptr), value :: host
       integer(c_size_t), value :: nbytes
       type(c_ptr) :: dev
     end function
     integer(c_int) function x3d_buf_unregister(ctx, host) bind(C, name="x3d_buf_unregister")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: host
     end function
     integer(c_int) function x3d_sync_to_device(ctx, host) bind(C, name="x3d_sync_to_device")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: host
     end function
     integer(c_int) function x3d_sync_to_host(ctx, host) bind(C, name="x3d_sync_to_host")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: host
     end function
     integer(c_int) function x3d_vel(ctx, u, v, w) bind(C, name="x3d_vel")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       type(c_ptr), value :: u
       type(c_ptr), value :: v
       type(c_ptr), value :: w
     end function
     integer(c_int) function x3d_test_rms(ctx, which, du, rms) bind(C, name="x3d_test_rms")
       import :: c_ptr, c_int
       type(c_ptr), value :: ctx
       integer(c_int), value :: which
       type(c_ptr), value :: du
       type(c_ptr), value :: rms
     end function
  end interface

contains

  ! A non-zero status from the library becomes the reference's abort.
  subroutine x3d_check(rc, where)
    use decomp_2d_mpi, only : decomp_2d_abort
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: where
    if (rc /= 0) call decomp_2d_abort(__FILE__, __LINE__, int(rc), where)
  end subroutine x3d_check

end module x3d_b200_bind
