// Internal declarations shared by the translation units of libx3d_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/x3d_b200.h"

namespace x3d {

enum Kind { DER = 0, DER2 = 1, DERVP = 2, DERPV = 3, INTVP = 4, INTPV = 5, IDENT = 6 };
enum Dir { DX = 0, DY = 1, DZ = 2 };

// Device view of one operator, in the sweep precision T.  Built once per
// operator from the FP64 precompute; the kernels read it from global memory
// through the read-only cache (every lane of a warp reads the same element).
template <typename T>
struct LineOp {
    const T *s;       // forward factors, s[0] = 0
    const T *w;       // inverse pivots
    const T *fw;      // f[i] * w[i]: backward step y_i = z_i w_i - fw_i y_{i+1}
    const T *p;       // Sherman-Morrison vector (periodic operators)
    const double *g;  // first row of M^-1, so y_0 = sum_i g_i r_i is known after the forward pass
    T a, b, c, d;     // explicit RHS scalars
    double alfa;      // Sherman-Morrison alpha
    double den;       // 1 + p_0 - alfa p_{n-1}
    int n;
    int periodic;
    int glen;         // g_i == 0 (in FP64) for i >= glen
    // Factorised circulant form, read by the chunked kernels.  A periodic
    // operator of the reference is the circulant (alfa, 1, alfa) matrix once
    // Sherman-Morrison has folded its corners back in, and that matrix is
    //   M = (1 + rho^2)^-1 (1 - rho E^-1)(1 - rho E),   alfa rho^2 + rho + alfa = 0,
    // with |rho| < 1 and (E y)_i = y_{i+1}.  So M y = r is two first-order
    // periodic recurrences:  v_i = (1 + rho^2) r_i + rho v_{i-1},
    // y_i = v_i + rho y_{i+1}.  circ = 0 for an operator whose factors are not
    // that matrix's (the chunked kernels then decline it).
    T ca, cb, cc, cd;      // RHS scalars times (1 + rho^2)
    T rho;
    T mfull[2], mlast[2];  // rho^L and rho^(last chunk's length), [0] for kChunkLong<T>, [1] kChunkShort<T>
    T wrap;                // 1 / (1 - rho^n), the sum over turns around the line
    // Chunks a carry scan visits: beyond depth the product of chunk
    // multipliers is below 1e-20 (FP64) or 1e-12 (FP32); depth == C means
    // the whole line, summed once and scaled by wrap.
    int depth[2];
    int circ;
    // Non-periodic first derivatives (periodic == 0): boundary conditions at
    // the two ends (1 free slip, 2 Dirichlet), the operator's parity and the
    // one-sided closure scalars af1, bf1, cf1, af2, afm, afn, bfn, cfn of
    // first_deriv_exp_ (src/x3d_operator_1d.f90:375-390).
    int ncl1, ncln, npaire;
    T cl[8];
};

template <typename T>
constexpr int kChunkLong = sizeof(T) == 4 ? 32 : 16;
template <typename T>
constexpr int kChunkShort = sizeof(T) == 4 ? 16 : 8;

// Host-side operator: FP64 contents of x3doperator1d plus the RHS scalars.
struct OpHost {
    int kind = 0, dir = 0, n = 0, npaire = 0, periodic = 1;
    int ncl1 = 0, ncln = 0;  // boundary conditions of a non-periodic operator
    double cl[8] = {};       // its closure scalars (LineOp::cl)
    double alfa = 0, a = 0, b = 0, c = 0, d = 0;
    std::vector<double> f, s, w, per, g;
    double den = 1.0;
    int glen = 0;
};

}  // namespace x3d

struct x3d_op_s {
    x3d::OpHost h;
    // device copies: one allocation holding float s,w,fw,p | double s,w,fw,p | double g
    void *dmem = nullptr;
    x3d::LineOp<float> opf{};
    x3d::LineOp<double> opd{};
    bool builtin = false;
};

struct x3d_ctx_s {
    int nx = 0, ny = 0, nz = 0;
    double xlx = 1, yly = 1, zlz = 1;
    double dx = 1, dy = 1, dz = 1;
    int precision = X3D_F64;
    int device = 0;
    // boundary conditions nclx1, nclxn, ncly1, nclyn, nclz1, nclzn (0 periodic,
    // 1 free slip, 2 Dirichlet); the Euler-step compositions need all periodic
    int ncl[6] = {0, 0, 0, 0, 0, 0};
    bool periodic_all = true;
    int num_sms = 148;
    size_t smem_optin = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int *d_err = nullptr;  // device error flag written by bounded waits
    std::string last_error;
    x3d_op_s *builtin[X3D_OP_COUNT] = {};
    // Poisson: cuFFT plans, spectrum and the 1-D modified-wavenumber tables.
    // With zfused the plans are 2-D (x, y) transforms batched over the z
    // planes, and one kernel does the z transforms and the mode division.
    cufftHandle plan_d2z = 0, plan_z2d = 0;
    bool plans_ready = false;
    bool zfused = false;
    bool zfuse_allowed = true;  // cleared to force the 3-D cuFFT path
    double *d_zft_tw = nullptr;  // e^{-2 pi i t / nz}, t < nz, then (tz, k2z) of each z mode (complex)
    // Own x transforms (nx / 2 a fused-transform length, with zfused): real
    // x lines to a spectrum stored (nz, nx/2 + 1, ny) with y fastest, 1-D
    // cuFFT transforms along the contiguous y lines, the fused z kernel on
    // that layout, and back.  d_xft_tw: e^{-2 pi i t / (nx/2)}, t < nx/2, then
    // e^{-2 pi i k / nx}, k <= nx/2 (complex).
    double *d_xft_tw = nullptr;
    cufftHandle plan_y = 0;
    bool plan_y_ready = false;
    // batched 1-D z transforms of one rank's block of the half spectrum, for
    // z lengths without a fused kernel (nxl x modes, nyl y rows)
    cufftHandle plan_zblk = 0;
    bool zblk_ready = false;
    int zblk_nxl = 0, zblk_nyl = 0;
    void *spectrum = nullptr;  // complex double, nz * ny * (nx/2+1)
    // non-periodic directions: the periodic context of the box mirrored about
    // its walls, and the mirrored right-hand side (created on first use)
    x3d_ctx_s *mirror = nullptr;
    double *mirror_rhs = nullptr;
    double *d_k2x = nullptr, *d_tx = nullptr, *d_k2y = nullptr, *d_ty = nullptr, *d_k2z = nullptr,
           *d_tz = nullptr;
    // scratch fields owned by the context (sized nx*ny*nz elements)
    std::vector<void *> scratch;
    size_t scratch_elem_bytes = 0;
    // device buffers for host-pointer arguments (pointer, bytes), reused by
    // later calls and freed with the context
    std::vector<std::pair<void *, size_t>> staging;
    double *d_red = nullptr;  // small reduction buffer
    // tile counter of the persistent stage kernels (zeroed before each launch
    // on the context stream; allocated with the context, so no call allocates it)
    unsigned long long *d_claim = nullptr;
    double *d_metric = nullptr;  // device copy of a y stretching metric (ny doubles)
    int metric_len = 0;
    // host arrays with device-resident mirrors (x3d_buf_register)
    struct Resident {
        void *host, *dev;
        size_t bytes;
    };
    std::vector<Resident> resident;
    // one Euler step recorded by x3d_step_capture
    cudaGraph_t step_graph = nullptr;
    cudaGraphExec_t step_exec = nullptr;
    // kernel choice per (direction, grid, precision, operator-group size):
    // filled by the autotuner, default_cfg otherwise
    std::map<std::string, int> tuned;
    // kernel choice per fused stage of the Euler step (transeq_x, div_y, ...),
    // filled by the autotuner; while stage_tuning is set, each stage run
    // times every configuration instead
    std::map<std::string, int> stage_tuned;
    std::map<std::string, float> stage_ms;  // the tuned configuration's time (ms)
    bool stage_tuning = false;
    int default_cfg = 0;
    unsigned long long launches = 0;  // kernels of this library launched on the context
    int last_cfg = -1;                // configuration of the last line-solve launch (x3d_ctx_last_kernel)
    size_t elem() const { return precision == X3D_F32 ? 4 : 8; }
    size_t npts() const { return (size_t)nx * ny * nz; }
    // points of the pressure grid: n - 1 along a non-periodic direction
    int pdim(int d) const
    {
        const int n = d == 0 ? nx : (d == 1 ? ny : nz);
        return ncl[2 * d] == 0 && ncl[2 * d + 1] == 0 ? n : n - 1;
    }
    size_t ppts() const { return (size_t)pdim(0) * pdim(1) * pdim(2); }
};

namespace x3d {

// ---- coefficient precompute (coeffs.cpp) -------------------------------
void rhs_scalars(int kind, double d, double *alfa, double *a, double *b, double *c, double *dd);
int build_periodic_op(int kind, int dir, int n, double d, OpHost &op);
// Non-periodic first derivative: ncl1, ncln in {1, 2}, npaire 0 or 1.
int build_nonperiodic_der(int dir, int n, double d, int ncl1, int ncln, int npaire, OpHost &op);
int build_nonperiodic_stag(int kind, int dir, int n, double d, int ncl1, int ncln, int npaire, OpHost &op);
int launch_np_stag(x3d_ctx_s *ctx, const x3d_op_s *op, int dir, const void *in, void *out, int n_in, int o1, int o2,
                   bool fp32);
void finish_op(OpHost &op);  // computes g, den, glen from f, s, w, per
int upload_op(x3d_op_s *op);
void free_op(x3d_op_s *op);

// ---- line solves (linesolve.cu) -----------------------------------------
// Applies op (kind given by op.kind unless kind_override >= 0) along dir to
// the (nx,ny,nz) field in -> out (may alias for kind IDENT).
int launch_linesolve(x3d_ctx_s *ctx, const x3d_op_s *op, int kind, int dir, const void *in,
                     void *out, int nx, int ny, int nz, bool fp32);
// Up to six operators along one direction applied to one input, one output each.
int launch_group(x3d_ctx_s *ctx, int dir, const void *in, const x3d_op_s *const *ops,
                 const int *kinds, void *const *outs, int nops, int nx, int ny, int nz, bool fp32);
int autotune_group(x3d_ctx_s *ctx, int dir, const void *in, const x3d_op_s *const *ops,
                   const int *kinds, void *const *outs, int nops, bool fp32, int reps, float *best_ms);

// ---- fused stages (stages.cpp); X3D_EUNSUPPORTED when no fused kernel fits --
int fused_transeq(x3d_ctx_s *ctx, void *const du[3], const void *const u[3], bool step, double dt,
                  void *const unew[3]);
int fused_divergence(x3d_ctx_s *ctx, double *pp3, const void *const u[3]);
int fused_divergence_scratch(x3d_ctx_s *ctx, double *pp3, const void *const u[3], void *const s[5]);
int fused_gradp(x3d_ctx_s *ctx, void *const px[3], const double *pp3, void *const ucor[3]);
// the same stages one direction at a time on a pencil of local extents
// (nx, ny, nz) whose lines along dir are whole (x3d_transeq_part etc.)
int part_transeq(x3d_ctx_s *ctx, int dir, void *const du[3], const void *const u[3], const void *const *add,
                 void *const *unew, double dt, int nx, int ny, int nz);
int part_divergence(x3d_ctx_s *ctx, int dir, void *const *out, const void *const *in, int nx, int ny, int nz);
int part_gradp(x3d_ctx_s *ctx, int dir, void *const *out, const void *const *in, void *const *ucor, int nx, int ny,
               int nz);
// block copies of the pencil transposes (pencil.cu)
int copy_blocks(x3d_ctx_s *ctx, void *dst, const void *src, int elem_bytes, const x3d_block *blocks, int count);

// ---- elementwise / reductions / transposes (fields.cu) ------------------
int launch_copy(x3d_ctx_s *ctx, void *dst, const void *src, size_t bytes);
int launch_axpy3(x3d_ctx_s *ctx, bool fp32, void *u, void *v, void *w, const void *du,
                 const void *dv, const void *dw, double alpha, size_t n);  // u = alpha*du + u
int launch_sub3(x3d_ctx_s *ctx, bool fp32, void *u, void *v, void *w, const void *a,
                const void *b, const void *c, size_t n);                   // u -= a
int launch_mul(x3d_ctx_s *ctx, bool fp32, void *out, const void *a, const void *b, size_t n);
int launch_scale_y(x3d_ctx_s *ctx, bool fp32, void *t, const double *ppy, int nx, int ny, int nz);
int launch_wait_selftest(x3d_ctx_s *ctx, uint64_t limit_ns);
int poisson_zpencil(x3d_ctx_s *ctx, void *spec, int nxl, int i0, int ny_loc, int j0);
int launch_roofline_probe(x3d_ctx_s *ctx, int pattern, int w, int ctas_per_sm, const float *in, float *const *outs,
                          int nx, int ny, int nz);

// An NVTX range over one stage of the hot path, named after the reference
// routine it replaces (the reference has these ranges commented out around
// every stage, e.g. src/xcompact3d.f90:79-96, src/transeq.f90:84-94).  It
// costs a call per stage and records nothing unless a profiler is attached.
struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};
int launch_fma_acc(x3d_ctx_s *ctx, bool fp32, void *out, const void *base, const void *a,
                   const void *b, size_t n);  // out = base + a*b
int launch_add(x3d_ctx_s *ctx, bool fp32, void *out, const void *a, const void *b, size_t n);
int launch_convert(x3d_ctx_s *ctx, void *dst, bool dst_fp32, const void *src, bool src_fp32,
                   size_t n);
int launch_vel(x3d_ctx_s *ctx, bool fp32, void *u, void *v, void *w);
int reduce_test_rms(x3d_ctx_s *ctx, bool fp32, int which, const void *du, double *rms);
int reduce_absmax_mean(x3d_ctx_s *ctx, const double *p, size_t n, double *out);

// ---- Poisson (poisson.cu) ------------------------------------------------
int poisson_setup(x3d_ctx_s *ctx);
int poisson_solve(x3d_ctx_s *ctx, double *rhs);
// the solve with homogeneous Neumann conditions along the non-periodic
// directions, rhs on the pressure grid (ppts points)
int poisson_solve_mirror(x3d_ctx_s *ctx, double *rhs);
void poisson_free(x3d_ctx_s *ctx);

// ---- helpers (capi.cpp) --------------------------------------------------
int set_error(x3d_ctx_s *ctx, int code, const std::string &msg);
int cuda_check(x3d_ctx_s *ctx, cudaError_t e, const char *what);
void *ctx_scratch(x3d_ctx_s *ctx, int idx);  // scratch field idx (elem = ctx precision, or 8 bytes)

}  // namespace x3d
