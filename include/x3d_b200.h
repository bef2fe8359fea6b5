/*
 * x3d_b200.h -- C ABI of the B200 (sm_100a) implementation of x3div's
 * Euler-timestep hot path: compact finite-difference derivatives, staggered
 * derivatives and interpolations (each an explicit stencil followed by a
 * batched periodic Thomas line solve), pencil transposes, the spectral
 * Poisson projection and the stage compositions that call them.
 *
 * Every entry point mirrors one reference routine (cited beside it as
 * path:line inside the xcompact3d/x3div source tree) with the same argument
 * order and meaning, prefixed by a context handle, so that the reference's
 * Fortran driver can bind to it through ISO_C_BINDING.
 *
 * Conventions
 *  - Fields are (nx, ny, nz) arrays with x fastest (Fortran order), exactly
 *    the layout of every 2decomp pencil.  At the supported 1x1 decomposition
 *    the X, Y and Z pencils of a field share this layout.
 *  - Field pointers are device pointers whose element type is the context
 *    precision: double for X3D_F64, float for X3D_F32.  Pressure arguments
 *    (pp3) are always double.  A pointer to ordinary or pinned host memory
 *    is also accepted: the call then stages it through device memory and
 *    returns only after the results are back in host memory.  The staging
 *    buffers stay with the context for later calls (freed by
 *    x3d_ctx_destroy).
 *  - Calls on device pointers are asynchronous on the context's stream, as
 *    CUDA launches are; x3d_ctx_sync() waits and reports device-side errors.
 *  - Every function returns an int status: X3D_OK (0) or a negative code.
 *    The reference aborts through decomp_2d_abort instead; a Fortran shim
 *    maps a non-zero status to that call.
 *  - Boundaries are periodic unless the context is made with
 *    x3d_ctx_create_bc; then the operators of a non-periodic direction
 *    exist, nxm = nx - 1 in its staggered signatures, x3d_poisson solves
 *    with Neumann conditions on the pressure there (a case the reference's
 *    Poisson solver stops on, src/poisson.f90:104-108), and the Euler-step
 *    compositions refuse it.
 *    Periodic directions have nxm == nx, nym == ny, nzm == nz.
 *  - Line lengths must be >= 8 (the 8-point interpolation stencils).
 */
#ifndef X3D_B200_H
#define X3D_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define X3D_OK 0
#define X3D_EINVAL -1       /* bad argument: null handle, shape, kind, direction */
#define X3D_EUNSUPPORTED -2 /* non-periodic boundary condition, line shorter than 8 */
#define X3D_ECUDA -3        /* CUDA runtime, driver or cuFFT error */
#define X3D_ENOMEM -4       /* device allocation failed */
#define X3D_ETIMEOUT -5     /* a bounded device-side wait gave up (error flag set) */

/* field precision of a context */
#define X3D_F64 0 /* FP64 fields and sweeps */
#define X3D_F32 1 /* FP32 fields and sweeps; FP64 coefficients, Sherman-Morrison scalar and Poisson */

/* directions */
#define X3D_DIR_X 0
#define X3D_DIR_Y 1
#define X3D_DIR_Z 2

/* operator kinds (x3doperator1d families, src/x3d_operator_1d.f90:32-47) */
#define X3D_KIND_DER 0   /* 6th-order compact first derivative, derx_00 */
#define X3D_KIND_DER2 1  /* 6th-order compact second derivative (declared, never built, in the reference) */
#define X3D_KIND_DERVP 2 /* staggered derivative, velocity -> pressure grid */
#define X3D_KIND_DERPV 3 /* staggered derivative, pressure -> velocity grid */
#define X3D_KIND_INTVP 4 /* 6th-order interpolation, velocity -> pressure grid */
#define X3D_KIND_INTPV 5 /* 6th-order interpolation, pressure -> velocity grid */

/* named operator instances of x3d_operator_1d_init (src/x3d_operator_1d.f90:135-189),
 * plus the three second-derivative operators the reference declares at
 * src/x3d_derive.f90:54-59 but never builds */
#define X3D_OP_DERX 0
#define X3D_OP_DERXP 1
#define X3D_OP_DERY 2
#define X3D_OP_DERYP 3
#define X3D_OP_DERZ 4
#define X3D_OP_DERZP 5
#define X3D_OP_DERXVP 6
#define X3D_OP_DERYVP 7
#define X3D_OP_DERZVP 8
#define X3D_OP_DERXPV 9
#define X3D_OP_DERYPV 10
#define X3D_OP_DERZPV 11
#define X3D_OP_INTXVP 12
#define X3D_OP_INTYVP 13
#define X3D_OP_INTZVP 14
#define X3D_OP_INTXPV 15
#define X3D_OP_INTYPV 16
#define X3D_OP_INTZPV 17
#define X3D_OP_DERXX 18
#define X3D_OP_DERYY 19
#define X3D_OP_DERZZ 20
#define X3D_OP_COUNT 21

typedef struct x3d_ctx_s *x3d_ctx;
typedef struct x3d_op_s *x3d_op;

/* ---- context ---------------------------------------------------------- */

/* Replaces init_xcompact3d's set-up path (src/x3d_tools.f90:163-185):
 * parameter() geometry (dx = xlx/nx ...), x3d_operator_{x,y,z}_data_init,
 * x3d_operator_1d_init, x3d_derive_init and decomp_2d_poisson_init, for a
 * fully periodic nx*ny*nz box of size xlx*yly*zlz at a 1x1 decomposition.
 * device: CUDA ordinal.  precision: X3D_F64 or X3D_F32. */
int x3d_ctx_create(x3d_ctx *ctx, int nx, int ny, int nz, double xlx, double yly, double zlz,
                   int precision, int device);
/* x3d_ctx_create with the boundary conditions of src/parameters.f90:
 * ncl[6] = {nclx1, nclxn, ncly1, nclyn, nclz1, nclzn}, each 0 (periodic,
 * both ends of a direction), 1 (free slip) or 2 (Dirichlet); NULL means all
 * periodic.  Along a non-periodic direction nxm = nx - 1 (dx = xlx/(nx-1)):
 *  - derx (npaire 0) and derxp (npaire 1) use der?_ij (src/x3d_derive.f90:
 *    156-215, 343-435, 562-665) with the closures and factors of
 *    first_deriv_exp_/first_deriv_imp_ (src/x3d_operator_1d.f90:325-488);
 *  - the staggered operators take the factors of interpol_imp_
 *    (:549-706) with the parities x3d_operator_1d_init binds (:152-189:
 *    dervp 1, derpv 0, intvp 1, intpv 1) and run the nclx = .false.
 *    branches of src/x3d_staggered.f90 from an nx-point to an nxm-point
 *    line or back.  Where the reference has no branch for an operator's
 *    parity (deryvp npaire 1, :595; der?pv npaire 0, :262, :843, :1199) it
 *    computes nothing, and the call returns X3D_EUNSUPPORTED;
 *  - the second derivatives do not exist, and the Euler-step compositions
 *    return X3D_EUNSUPPORTED;
 *  - x3d_poisson takes the pressure grid (nxm = nx - 1 points) and solves
 *    with the bc = 1 (Neumann) conditions that decomp_2d_poisson_init
 *    assigns there (src/poisson.f90:85-99) and the reference then stops on
 *    (:104-108); the pencil entry points x3d_poisson_zlines/zpencil stay
 *    periodic. */
int x3d_ctx_create_bc(x3d_ctx *ctx, int nx, int ny, int nz, double xlx, double yly, double zlz,
                      int precision, int device, const int *ncl);
/* finalise_xcompact3d's device-side part (src/x3d_tools.f90:212-248). */
int x3d_ctx_destroy(x3d_ctx ctx);
/* Run the context's work on a caller-owned stream (a cudaStream_t; NULL is
 * the legacy default stream).  A new context uses its own non-blocking
 * stream, which x3d_ctx_get_stream returns. */
int x3d_ctx_set_stream(x3d_ctx ctx, void *stream);
int x3d_ctx_get_stream(x3d_ctx ctx, void **stream);
/* Wait for the context's stream; returns X3D_ETIMEOUT if a kernel recorded a
 * bounded-wait failure since the last call, else a CUDA error or X3D_OK. */
int x3d_ctx_sync(x3d_ctx ctx);
/* Checks the failure path of the bounded device waits: launches one kernel
 * whose wait nothing can complete (an mbarrier with no arrival and no copy
 * in flight) and which gives up after limit_s (0 < limit_s <= 1) seconds,
 * recording the failure; the next x3d_ctx_sync returns X3D_ETIMEOUT and
 * clears it, and the context stays usable.  No reference counterpart. */
int x3d_ctx_selftest_timeout(x3d_ctx ctx, double limit_s);
/* Measurement aid for the roofline of the sweep launches (no reference
 * counterpart): moves one FP32 (nx, ny, nz) device field to six FP32 device
 * fields (outs[6]) with no arithmetic, in a flat order (pattern 0: 16-byte
 * vectors, consecutive threads on consecutive vectors) or in the y stage
 * kernels' order (pattern 1: tiles of w in {8, 16, 32, 64, 128} x-adjacent
 * columns of the ny rows of a z plane, each thread on consecutive rows;
 * pattern 2: the same tiles over blocks of 128 rows; pattern 3: pattern 1
 * with each store of the CTA on consecutive rows; pattern 4: pattern 1 with
 * consecutive tiles on different z planes; pattern 5: pattern 1 with the
 * tiles claimed in order from a counter, as the persistent stage kernels
 * take them (w in {8, 16, 32}); pattern 6: pattern 5 in the z stage
 * kernels' order (tiles of w columns of one y row over all nz planes);
 * nx % w == 0, ny a multiple of the rows a
 * thread moves (32, or 16 for w = 128) and of the block), so that timing it
 * gives the
 * bandwidth that traffic mix and access order can reach.  ctas_per_sm sets
 * the grid (0: 2 per SM). */
int x3d_roofline_probe(x3d_ctx ctx, int pattern, int w, int ctas_per_sm, const void *in, void *const *outs,
                       int nx, int ny, int nz);
/* Text of the last error recorded on this context (never NULL). */
const char *x3d_ctx_last_error(x3d_ctx ctx);
/* Number of this library's kernels launched on the context so far (library
 * kernels such as cuFFT's are not counted). */
int x3d_ctx_launch_count(x3d_ctx ctx, unsigned long long *count);
/* Configuration (as in x3d_ctx_set_kernel) of the last periodic line-solve
 * or fused-stage launch on the context, -1 before the first: shows which
 * kernel a call ran after fall-backs.  No reference counterpart. */
int x3d_ctx_last_kernel(x3d_ctx ctx, int *cfg);
/* Geometry query: dims[3], lengths[3], spacing[3] (any may be NULL). */
int x3d_ctx_geometry(x3d_ctx ctx, int *dims, double *lengths, double *spacing, int *precision);

/* ---- operators: type x3doperator1d (src/x3d_operator_1d.f90:12-30) ---- */

/* One of the X3D_OP_* instances built by x3d_ctx_create. */
int x3d_op_builtin(x3d_ctx ctx, int which, x3d_op *op);
/* An operator from explicit x3doperator1d contents, as the reference host
 * would hand over after its own x3d_operator_1d_init: n, npaire, alfa, the
 * Thomas arrays f, s, w (see prepare, src/x3d_operator_1d.f90:301-323), the
 * Sherman-Morrison vector periodic, plus the explicit RHS scalars that the
 * reference keeps as module globals of x3d_operator_{x,y,z}_data (rhs[4] =
 * a, b, c, d, e.g. afix, bfix, 0, 0 for derx, aicix6..dicix6 for
 * interpolation).  periodic = NULL makes a non-periodic staggered operator
 * (kinds DERVP, DERPV, INTVP, INTPV; n is its output length, nm = nx - 1
 * for the vp kinds), applied by the staggered routines when nxm = nx - 1;
 * non-periodic first derivatives come from x3d_ctx_create_bc, which knows
 * their boundary closures.  Host pointers, FP64, copied. */
int x3d_op_create(x3d_ctx ctx, int kind, int dir, int n, int npaire, double alfa,
                  const double *f, const double *s, const double *w, const double *periodic,
                  const double *rhs, x3d_op *op);
int x3d_op_destroy(x3d_ctx ctx, x3d_op op);
/* Read back an operator's FP64 contents: any output may be NULL.
 * meta[0..3] = n, kind, dir, npaire; scal[0..4] = alfa, a, b, c, d;
 * f, s, w, periodic: length n. */
int x3d_op_info(x3d_op op, int *meta, double *scal, double *f, double *s, double *w,
                double *periodic);

/* ---- collocated derivatives: x3d_derive (src/x3d_derive.f90:18-59) ---- */

/* derx_00 (src/x3d_derive.f90:111-152): tx = d(ux)/dx */
int x3d_derx(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nx, int ny, int nz);
/* dery_00 (src/x3d_derive.f90:279-339).  ppy: the stretching metric (ny
 * values, host or device); NULL stands for istret = 0, the reference's
 * setting (src/parameters.f90:117), otherwise ty(i,j,k) *= ppy(j) after the
 * solve (:331-337).  deryvp takes ppyi and derypv ppy the same way
 * (src/x3d_staggered.f90:629-635, 875-881). */
int x3d_dery(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, const double *ppy, int nx, int ny,
             int nz);
/* derz_00 (src/x3d_derive.f90:503-558) */
int x3d_derz(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nz);
/* second derivatives: the DERIVATIVE_X / _YY / _Z pointers derxx, deryy,
 * derzz (src/x3d_derive.f90:54-59), left null by the reference */
int x3d_derxx(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nx, int ny, int nz);
int x3d_deryy(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, int nx, int ny, int nz);
int x3d_derzz(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nz);

/* ---- staggered operators: x3d_staggered (src/x3d_staggered.f90) -------- */

int x3d_derxvp(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nx, int nxm, int ny, int nz);   /* :23-106 */
int x3d_interxvp(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nx, int nxm, int ny, int nz); /* :110-217 */
int x3d_derxpv(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nxm, int nx, int ny, int nz);   /* :221-285 */
int x3d_interxpv(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nxm, int nx, int ny, int nz); /* :289-404 */
int x3d_interyvp(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, int nx, int ny, int nym, int nz); /* :408-541 */
int x3d_deryvp(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, const double *ppyi, int nx, int ny,
               int nym, int nz);                                                                     /* :545-637 */
int x3d_interypv(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, int nx, int nym, int ny, int nz); /* :641-786 */
int x3d_derypv(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, const double *ppy, int nx, int nym,
               int ny, int nz);                                                                      /* :790-883 */
int x3d_derzvp(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nz, int nzm);   /* :887-997 */
int x3d_interzvp(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nz, int nzm); /* :1001-1139 */
int x3d_derzpv(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nzm, int nz);   /* :1143-1229 */
int x3d_interzpv(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nzm, int nz); /* :1233-1383 */

/* ---- batched operator applications -------------------------------------- */

/* One operator application of a batch: out = op(in) along op's direction. */
typedef struct {
    x3d_op op;      /* built-in or user operator (its kind and direction decide the routine) */
    const void *in; /* (nx,ny,nz) input field of the context grid */
    void *out;      /* (nx,ny,nz) output field; must not alias any input of the batch */
} x3d_work;

/* Apply every item of a work-list, e.g. all the derivative and
 * interpolation sweeps of one RHS stage.  Items are independent.  With host
 * pointers each distinct input is uploaded once and every output is
 * downloaded once, and the call returns when the results are in host
 * memory.  No reference counterpart: it replaces a sequence of der* and
 * staggered calls (src/transeq.f90, src/navier.f90) by one call. */
int x3d_apply_batch(x3d_ctx ctx, const x3d_work *items, int count);
/* One application out = op(in) on the context grid, whatever the operator's
 * kind and direction: the work-list of one item.  No reference counterpart
 * as a single routine: it stands for whichever der* or staggered routine
 * the operator's kind and direction name. */
int x3d_apply(x3d_ctx ctx, x3d_op op, const void *in, void *out);

/* Times every kernel configuration (lines per CTA, chunk length, or one
 * thread per line) for each direction and for groups of 1, 2, 3 and 6
 * operators sharing an input (up to max_group), on the context grid, and
 * keeps the fastest for later calls; then does the same for each fused
 * stage of the Euler step (transeq + int_time, divergence, gradp + cor_vel,
 * per direction).  Synchronous; uses context scratch fields (up to 14 of
 * nx*ny*nz doubles); not callable during stream capture.  Without it a
 * fixed default configuration is used.  No reference counterpart. */
int x3d_autotune(x3d_ctx ctx, int max_group);
/* Force kernel configuration cfg (0..5 chunked, one CTA per tile;
 * 6..11 the same shapes as persistent double-buffered kernels; 12..15 y/z
 * kernels that carry two x-adjacent lines per thread in packed FP32
 * registers (FP32 contexts, even nx); 16 one thread per line; 17 the y/z
 * kernel of configuration 6 built for three CTAs per SM, for operators that
 * each write their own output, on lines of at most 16 chunks; 18, 19 and 20
 * the same for configurations 9, 3 and 0, x lines too) for every
 * later call and forget tuned choices; -1 restores the default.  A
 * configuration that cannot handle a call (alignment, shared memory) still
 * falls back to one that can.  No reference counterpart. */
int x3d_ctx_set_kernel(x3d_ctx ctx, int cfg);
/* The configuration chosen for (direction, group size): *cfg = -1 when not
 * tuned, 0..15 and 17..20 chunked variants, 16 one thread per line. */
int x3d_autotune_choice(x3d_ctx ctx, int dir, int group, int *cfg);
/* The configuration chosen for a fused stage of the Euler step (*cfg = -1
 * when not tuned): stage is one of transeq_x, transeq_y, transeq_z, div_x,
 * div_y, div_z, gradp_z, gradp_y, gradp_x, gradp_x_cor.  A stage may run as
 * several launches: "<stage>.split" = 1 for a momentum stage as two launches
 * ("<stage>.b", then "<stage>.a"), "<stage>.parts" = k > 1 for a stage as k
 * launches over disjoint staged inputs ("<stage>.1" .. "<stage>.k"); each
 * launch has its own configuration under its own name. */
int x3d_autotune_stage_choice(x3d_ctx ctx, const char *stage, int *cfg);
/* Sets one of those choices (a saved tuning, or a form to test); value -1
 * removes it.  Configurations are 0..15 and 17..20; "<stage>.split" 0 or 1;
 * "<stage>.parts" a launch count, used only where the stage splits into
 * exactly that many parts; "poisson_x" 0 or 1 (x3d_poisson).  Extension. */
int x3d_ctx_set_stage_choice(x3d_ctx ctx, const char *stage, int value);

/* ---- batches of independent boxes ----------------------------------------- */

/* A periodic box of a batch (no reference counterpart: the reference runs one
 * box per job; a batch sweeps many uneven boxes in one launch). */
typedef struct {
    int nx, ny, nz;
    double xlx, yly, zlz;
} x3d_box;
typedef struct x3d_batch_s *x3d_batch;

int x3d_batch_create(x3d_batch *batch, const x3d_box *boxes, int nboxes, int precision, int device);
int x3d_batch_destroy(x3d_batch batch);
/* NULL is the legacy default stream; a new batch uses its own stream. */
int x3d_batch_set_stream(x3d_batch batch, void *stream);
const char *x3d_batch_last_error(x3d_batch batch);
/* Binds the derivative sweep: for box i and field f < nfields, input
 * fields[i*nfields + f] (device, the box's grid) and, for direction d and
 * operator family k < nops (X3D_KIND order: der, der2, dervp, derpv, intvp,
 * intpv), output outs[((i*nfields + f)*3 + d)*6 + k].  Plans the persistent
 * work-list (tiles, tensor maps) once; outputs must not alias inputs. */
int x3d_batch_bind_sweep(x3d_batch batch, int nfields, void *const *fields, void *const *outs, int nops);
/* One persistent launch over every tile of every bound job (boxes the
 * persistent kernel cannot take run as grouped launches after it). */
int x3d_batch_run(x3d_batch batch);
/* Captures x3d_batch_run into a CUDA graph (on the batch's own stream, after
 * waiting for the current one); x3d_batch_replay launches the graph on the
 * stream set with x3d_batch_set_stream. */
int x3d_batch_capture(x3d_batch batch);
int x3d_batch_replay(x3d_batch batch);
int x3d_batch_sync(x3d_batch batch);
/* points = operator-application points per run; tiles, jobs in the
 * persistent launch; fallback_jobs run as grouped launches. */
int x3d_batch_info(x3d_batch batch, long long *points, long long *tiles, int *jobs, int *fallback_jobs);
/* Tunes the bound sweep per box shape: for each distinct shape and
 * direction, times the persistent kernel on that shape's jobs with the long
 * and the short chunk length, each with as many lines per tile as its
 * threads allow and with half as many (x jobs also with their outputs
 * staged in shared memory and sent as row copies), keeps the fastest, then
 * times the whole work-list with those choices, with them but no staging,
 * with only the long-chunk choices' tile widths, and with the defaults, and
 * keeps the fastest of the four (a shape timed alone can mislead: in the
 * whole launch the largest tile sizes every CTA).  Overwrites the bound
 * outputs; synchronous; not during stream capture.  No reference
 * counterpart. */
int x3d_batch_autotune(x3d_batch batch);
/* The chunk length and lines per tile the jobs of box `box` along `dir`
 * run with (*lines = 0 for jobs that run outside the persistent launch).
 * No reference counterpart. */
int x3d_batch_choice(x3d_batch batch, int box, int dir, int *chunk, int *lines);

/* ---- batched Thomas line solves: module thomas (src/thomas.f90:15-28) --- */

/* In-place solve of every line of tt.  With perio != NULL this is
 * ?thomas_0 (periodic, Sherman-Morrison with alfa, :34-58/87-111/139-163);
 * with perio == NULL it is ?thomas_12 (:61-84/114-136/166-188) and alfa is
 * ignored.  ff, fs, fw, perio: FP64 arrays of the line length (host or
 * device memory). */
int x3d_xthomas(x3d_ctx ctx, void *tt, const double *ff, const double *fs, const double *fw,
                const double *perio, double alfa, int nx, int ny, int nz);
int x3d_ythomas(x3d_ctx ctx, void *tt, const double *ff, const double *fs, const double *fw,
                const double *perio, double alfa, int nx, int ny, int nz);
int x3d_zthomas(x3d_ctx ctx, void *tt, const double *ff, const double *fs, const double *fw,
                const double *perio, double alfa, int nx, int ny, int nz);

/* ---- pencil transposes: x3d_transpose (src/x3d_transpose.f90:21-47) ----- */

/* At a 1x1 decomposition the source and destination pencils have the same
 * shape and layout, so each transpose is a device copy (nothing when
 * in == out).  is_complex selects the complex variants (twice the bytes). */
int x3d_transpose_x_to_y(x3d_ctx ctx, const void *in, void *out, int is_complex);
int x3d_transpose_y_to_z(x3d_ctx ctx, const void *in, void *out, int is_complex);
int x3d_transpose_z_to_y(x3d_ctx ctx, const void *in, void *out, int is_complex);
int x3d_transpose_y_to_x(x3d_ctx ctx, const void *in, void *out, int is_complex);

/* Over a p_row x p_col process grid each transpose is an exchange of blocks
 * among the ranks of one row or column of the grid (2decomp's
 * transpose_x_to_y etc., which pack the blocks of the rank's pencil into a
 * send buffer, exchange them with MPI_ALLTOALLV and unpack what arrives).
 * The exchange is the host's collective (NCCL through torch.distributed in
 * x3div_b200.pencils); x3d_copy_blocks is the packing and the unpacking: it
 * copies `count` boxes of elements of elem_bytes (4, 8 or 16) bytes from
 * src to dst, box i from element src_offset with the given y and z strides
 * to element dst_offset with its own strides, in one launch per 32 boxes on
 * the context's stream.  Device pointers; the boxes must not overlap in
 * dst.  No reference counterpart as a routine. */
typedef struct x3d_block {
    long long src_offset, dst_offset; /* first element of the box */
    int nx, ny, nz;                   /* extents of the box */
    long long src_ystride, src_zstride; /* elements between rows / planes of src */
    long long dst_ystride, dst_zstride; /* elements between rows / planes of dst */
} x3d_block;
int x3d_copy_blocks(x3d_ctx ctx, void *dst, const void *src, int elem_bytes, const x3d_block *blocks, int count);

/* ---- spectral Poisson: decomp_2d_poisson (src/poisson.f90:57-65) -------- */

/* poisson_000 (src/poisson.f90:276-419), in place on the FP64 pressure-grid
 * field rhs (nx*ny*nz doubles).  On a context with non-periodic directions
 * (x3d_ctx_create_bc) rhs has nxm = nx - 1 points along each of them and
 * the pressure gets homogeneous Neumann conditions there: the bc = 1 case
 * of decomp_2d_poisson_init (src/poisson.f90:85-99, :114-117) with the
 * cosine modes of waves()'s bc = 1 tables (:539-553, :573-588, :603-613),
 * which x3div itself stops on (:104-108).  It is solved as the periodic
 * problem on the box mirrored about both walls of every such direction
 * (2 nxm points over 2 xlx) and cut back: the mirrored field holds exactly
 * those cosine modes.  The first call makes the mirrored box's periodic
 * context and right-hand side (kept until x3d_ctx_destroy).  Where nz and
 * nx / 2 are both 2^p 3^q from 8 to 1024 (nx even), the periodic solve is
 * five launches: the library's x transforms (real lines to a spectrum with
 * y fastest), batched 1-D cuFFT transforms along y, the fused z transform
 * and mode division, and back; the stage choice "poisson_x" = 0
 * (x3d_ctx_set_stage_choice) takes cuFFT's 2-D (x, y) transforms instead. */
int x3d_poisson(x3d_ctx ctx, double *rhs);
/* The z part of poisson_000 for a box whose y rows are spread over ranks:
 * spec is this rank's block of the x-y transformed half spectrum (complex
 * FP64, nx/2+1 x modes, ny_loc y rows starting at global row j0, nz z
 * points, x fastest; unnormalised 2-D r2c transforms of the z planes, as
 * cuFFT or 2decomp produce them).  In place: the forward z transform, the
 * division of every mode by -K ntot (zero where K < 1e-16), the inverse z
 * transform; the unnormalised 2-D c2r transforms then give the solution.
 * Device pointer.  z lengths 2^p 3^q from 8 to 1024 take one fused
 * kernel; other lengths take batched 1-D cuFFT transforms along z and a
 * division kernel.  Builds no cuFFT plan or spectrum of the whole box. */
int x3d_poisson_zlines(x3d_ctx ctx, void *spec, int ny_loc, int j0);
/* The same on a Z pencil of a p_row x p_col decomposition (2decomp's
 * zstart/zend of the half spectrum): spec holds x modes i0 .. i0 + nxh_loc
 * - 1 of the nx/2+1 and y rows j0 .. j0 + ny_loc - 1, all nz z points,
 * ((nz, ny_loc, nxh_loc) with x fastest).  x3d_poisson_zlines is the case
 * i0 = 0, nxh_loc = nx/2+1. */
int x3d_poisson_zpencil(x3d_ctx ctx, void *spec, int nxh_loc, int i0, int ny_loc, int j0);

/* ---- projection stage: module navier (src/navier.f90) ------------------- */

/* divergence (:98-236): pp3 = div(u) on the pressure grid (FP64 output).
 * nlock is accepted for signature parity; the test-mode print is replaced
 * by x3d_div_stats. */
int x3d_divergence(x3d_ctx ctx, double *pp3, const void *ux1, const void *uy1, const void *uz1,
                   int nlock);
/* Largest grid (points per field) x3d_divergence_noalloc can take. */
#define X3D_NOALLOC_MAX_POINTS 262144
/* x3d_divergence without any device allocation.  No counterpart in the
 * reference.  For hosts that cannot allocate device memory in their time
 * loop -- e.g. a Fortran host that maps its whole device working set up
 * front through OpenACC data regions and runs under a fixed memory budget,
 * or a solver sharing the GPU that must not take memory mid-step.  The five
 * intermediate fields live in one fixed array inside the library
 * (5 * X3D_NOALLOC_MAX_POINTS doubles = 10 MiB) instead of in context
 * scratch.  A GPU holds the array from the first call on it (that call loads
 * the library's module there under CUDA's lazy module loading, so make it
 * once before the time loop) until the process exits.
 * Inputs and output are caller-owned device pointers (host pointers are
 * refused, since staging them would allocate); the context must already
 * exist.  Grids above X3D_NOALLOC_MAX_POINTS points return X3D_EINVAL, grids
 * the fused stage kernels cannot take return X3D_EUNSUPPORTED.  The first
 * call on each device looks up the array's device address (again after a
 * device reset, which moves it); make that first call before any stream
 * capture.  All calls share the one array: calls that
 * overlap on the GPU (other streams or contexts at the same time) race on
 * it.  Every element of the array is written before it is read, so nothing
 * has to be cleared between calls. */
int x3d_divergence_noalloc(x3d_ctx ctx, double *pp3, const void *ux1, const void *uy1,
                           const void *uz1);
/* gradp (:249-359): px1, py1, pz1 = grad(pp3) on the velocity grid */
int x3d_gradp(x3d_ctx ctx, void *px1, void *py1, void *pz1, const double *pp3);
/* cor_vel (:64-91): u -= grad p */
int x3d_cor_vel(x3d_ctx ctx, void *ux, void *uy, void *uz, const void *px, const void *py,
                const void *pz);
/* solve_poisson (:21-56): divergence, poisson, gradp */
int x3d_solve_poisson(x3d_ctx ctx, double *pp3, void *px1, void *py1, void *pz1, const void *ux1,
                      const void *uy1, const void *uz1);
/* The DIV U max/mean figures printed by divergence in test mode
 * (src/navier.f90:213-231), computed on the device: out[0] = max|pp3|,
 * out[1] = mean|pp3|.  Synchronous. */
int x3d_div_stats(x3d_ctx ctx, const double *pp3, double *out);

/* ---- convective RHS and time integration -------------------------------- */

/* momentum_rhs_eq (src/transeq.f90:44-355): du_c = sum_d d(u_d u_c)/dx_d
 * + u_d du_c/dx_d, with the reference's operator pairs and sign. */
int x3d_momentum_rhs_eq(x3d_ctx ctx, void *dux1, void *duy1, void *duz1, const void *ux1,
                        const void *uy1, const void *uz1);
/* int_time, Euler branch (src/time_integrators.f90:20-106): u = gdt*du + u */
int x3d_int_time(x3d_ctx ctx, void *ux1, void *uy1, void *uz1, const void *dux1, const void *duy1,
                 const void *duz1, double gdt);
/* One timestep of the reference loop body (src/xcompact3d.f90:80-95):
 * calculate_transeq_rhs, int_time, solve_poisson, cor_vel.  dux..duz,
 * pp3 and px..pz are outputs (the reference's dux1/duy1/duz1, pp3, px1..pz1). */
int x3d_euler_step(x3d_ctx ctx, void *ux1, void *uy1, void *uz1, void *dux1, void *duy1,
                   void *duz1, double *pp3, void *px1, void *py1, void *pz1, double dt);
/* Records x3d_euler_step on these fields into a CUDA graph kept by the
 * context (nothing runs), after allocating what the step would allocate on
 * first use; x3d_step_launch replays it on the context's stream, one
 * timestep per launch.  The fields must be device pointers or registered
 * host arrays (x3d_buf_register), and the context must be on a created
 * stream (not the legacy or per-thread default).  The graph keeps the
 * kernel configurations chosen at capture time; a new capture replaces it.
 * x3d_ctx_launch_count counts the captured launches once.  No reference
 * counterpart: the reference calls the step's routines one by one. */
int x3d_step_capture(x3d_ctx ctx, void *ux1, void *uy1, void *uz1, void *dux1, void *duy1,
                     void *duz1, double *pp3, void *px1, void *py1, void *pz1, double dt);
int x3d_step_launch(x3d_ctx ctx);

/* ---- the step's parts on one pencil of a process grid --------------------- */

/* The reference computes each stage of the step pencil by pencil, with a
 * transpose between (src/transeq.f90:44-355, src/navier.f90:98-359).  These
 * are the fused stage kernels of x3d_momentum_rhs_eq, x3d_divergence and
 * x3d_gradp + x3d_cor_vel, one direction at a time, on a dir-pencil of
 * local extents (nx, ny, nz) whose lines along dir are whole (the context's
 * length along dir); the host transposes between them.  Field arrays are
 * device pointers of the context's precision unless stated.
 *
 * x3d_transeq_part: for c = 0, 1, 2
 *   du[c] = add[c] + d(u_dir u_c)/dx_dir + u_dir d(u_c)/dx_dir
 * (add may be NULL, or add[c] may alias du[c]); with unew != NULL also
 *   unew[c] = u[c] + dt du[c]   (int_time, Euler; unew[c] may alias u[c]).
 * x3d_divergence_part (navier.f90:166-202):
 *   dir 0: out = {pp1, pgy1, pgz1} = {derxvp ux, interxvp uy, interxvp uz}, in = {ux, uy, uz}
 *   dir 1: out = {duydypi2, upi2} = {deryvp pgy1 + interyvp pp1, interyvp pgz1}, in = {pp1, pgy1, pgz1}
 *   dir 2: out = {pp3} = {interzvp duydypi2 + derzvp upi2} (FP64), in = {duydypi2, upi2}
 * x3d_gradp_part (navier.f90:273-304; cor_vel :83-87):
 *   dir 2: out = {ppi3, pgz3} = {interzpv pp3, derzpv pp3}, in = {pp3} (FP64)
 *   dir 1: out = {ppi2, pgy2, pgzi2} = {interypv ppi3, derypv ppi3, interypv pgz3}, in = {ppi3, pgz3}
 *   dir 0: out = {px, py, pz} = {derxpv ppi2, interxpv pgy2, interxpv pgzi2}, in = {ppi2, pgy2, pgzi2};
 *          with ucor != NULL also ucor[c] -= out[c]
 * Periodic contexts.  X3D_EUNSUPPORTED when the fused kernels cannot take
 * the pencil (its lines, alignment or x extent); the host then composes the
 * part from the single-operator routines. */
int x3d_transeq_part(x3d_ctx ctx, int dir, void *const *du, const void *const *u, const void *const *add,
                     void *const *unew, double dt, int nx, int ny, int nz);
int x3d_divergence_part(x3d_ctx ctx, int dir, void *const *out, const void *const *in, int nx, int ny,
                        int nz);
int x3d_gradp_part(x3d_ctx ctx, int dir, void *const *out, const void *const *in, void *const *ucor, int nx,
                   int ny, int nz);

/* ---- device-resident host arrays ------------------------------------------ */

/* The reference keeps its fields on the device between calls with OpenACC
 * data regions (src/xcompact3d.f90:43-72).  x3d_buf_register gives a host
 * array of nbytes a device mirror (filled from the host once; *dev, if not
 * NULL, receives its address): every later call passed a pointer inside the
 * host array works on the mirror, with no copies and no host results, until
 * x3d_sync_to_host copies the mirror back (x3d_sync_to_device the other
 * way).  x3d_buf_unregister frees the mirror without copying.  Registered
 * arrays must not overlap.  Synchronous.  No reference counterpart. */
int x3d_buf_register(x3d_ctx ctx, void *host, size_t nbytes, void **dev);
int x3d_buf_unregister(x3d_ctx ctx, void *host);
int x3d_sync_to_device(x3d_ctx ctx, void *host);
int x3d_sync_to_host(x3d_ctx ctx, void *host);

/* ---- initial field and analytic checks: module mom (src/mom.f90) -------- */

/* vel (:26-57) on the device */
int x3d_vel(x3d_ctx ctx, void *u, void *v, void *w);
/* test_du / test_dv / test_dw (:59-243): RMS error of du/dx (which=0),
 * dv/dy (1) or dw/dz (2) against the analytic derivative of vel's field.
 * Synchronous; result in *rms. */
int x3d_test_rms(x3d_ctx ctx, int which, const void *du, double *rms);

#ifdef __cplusplus
}
#endif

#endif /* X3D_B200_H */
