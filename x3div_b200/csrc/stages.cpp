// Fused stage compositions of the Euler step, built from StageProgram
// launches (linesolve_chunk.cu).  At the supported 1x1 decomposition every
// transpose of the reference is a same-layout copy and is elided.
//
//   momentum_rhs_eq (src/transeq.f90:44-355): one launch per direction, each
//     solving d(u_d u_c)/dx_d and d(u_c)/dx_d for the three components and
//     accumulating  du_c += d(u_d u_c)/dx_d + u_d du_c/dx_d;  with a time step
//     the z launch also applies int_time (src/time_integrators.f90:41-43),
//     u_c = dt du_c + u_c, in place.  Each direction may instead run as two
//     launches of two staged fields each, (u_d, u_o2) for component o2, then
//     (u_d, u_o1) for components d and o1, which fit more CTAs on an SM; the
//     autotuner times both forms and keeps the faster.
//   divergence (src/navier.f90:166-202): x launch derxvp/interxvp/interxvp,
//     y launch interyvp + deryvp and interyvp, z launch interzvp + derzvp into
//     the FP64 pressure field.
//   gradp + cor_vel (src/navier.f90:273-304, :83-87): z launch interzpv and
//     derzpv, y launch interypv/derypv/interypv, x launch derxpv/interxpv/
//     interxpv writing px, py, pz and, for cor_vel, u_c -= p_c in place.
#include <algorithm>
#include <cstring>

#include "linesolve_chunk.h"
#include "stage_split.h"
#include "x3d_internal.h"

namespace x3d {

template <typename T>
static const LineOp<T> &lop(const x3d_op_s *op);
template <>
const LineOp<float> &lop<float>(const x3d_op_s *op)
{
    return op->opf;
}
template <>
const LineOp<double> &lop<double>(const x3d_op_s *op)
{
    return op->opd;
}

template <typename T>
static StageOp<T> sop(const x3d_op_s *op, int src_a, int src_b = -1)
{
    StageOp<T> s;
    std::memset(&s, 0, sizeof(s));
    s.op = lop<T>(op);
    s.kind = op->h.kind;
    s.src_a = (short)src_a;
    s.src_b = (short)src_b;
    s.mul_tile = -1;
    s.sign = 1.0;
    return s;
}

template <typename T>
static void set_flush(StageOp<T> &s, void *out, const void *base = nullptr, bool f64 = false)
{
    s.flush = 1;
    s.out = out;
    s.base = base;
    s.out_f64 = f64 ? 1 : 0;
}

// Local extents of the field a stage runs on: the context's box, or a
// pencil of it whose lines along the stage's direction are whole.
struct Ext {
    int nx, ny, nz;
};

static Ext box_ext(const x3d_ctx_s *ctx) { return {ctx->nx, ctx->ny, ctx->nz}; }

// The name a stage's tuned configuration is kept under: the stage's own on
// the context's box, with the extents appended on a pencil.
static std::string stage_key(const x3d_ctx_s *ctx, const char *name, Ext e)
{
    if (e.nx == ctx->nx && e.ny == ctx->ny && e.nz == ctx->nz) return name;
    return std::string(name) + "@" + std::to_string(e.nx) + "x" + std::to_string(e.ny) + "x" + std::to_string(e.nz);
}

// Times every configuration of a stage (one probe launch, then the fastest
// of three timed ones) and keeps the fastest for the stage's name.  Only the autotuner
// runs stages this way, on scratch fields.
template <typename T>
static int tune_stage(x3d_ctx_s *ctx, const StageProgram<T> &prog, int dir, const char *name, Ext e)
{
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int best = -1, rc = X3D_OK;
    float bt = 0.f;
    for (int cfg = 0; cfg < kAllConfigs; ++cfg) {
        if (!is_stage_cfg(cfg)) continue;
        rc = launch_stage<T>(ctx, prog, dir, e.nx, e.ny, e.nz, cfg);
        if (rc == X3D_EUNSUPPORTED) continue;
        if (rc) break;
        // the fastest of three separately timed launches
        float ms = 0.f;
        for (int r = 0; r < 3 && !rc; ++r) {
            cudaEventRecord(a, ctx->stream);
            rc = launch_stage<T>(ctx, prog, dir, e.nx, e.ny, e.nz, cfg);
            cudaEventRecord(b, ctx->stream);
            cudaEventSynchronize(b);
            float m = 0.f;
            cudaEventElapsedTime(&m, a, b);
            ms = r == 0 ? m : std::min(ms, m);
        }
        if (rc) break;
        if (best < 0 || ms < bt) {
            best = cfg;
            bt = ms;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc && rc != X3D_EUNSUPPORTED) return rc;
    if (best < 0) return X3D_EUNSUPPORTED;
    ctx->stage_tuned[name] = best;
    ctx->stage_ms[name] = bt;
    return X3D_OK;
}

// Runs one program with its tuned (or the default) configuration, then, if
// that one cannot take the grid, the others in order.
template <typename T>
static int run_program(x3d_ctx_s *ctx, const StageProgram<T> &prog, int dir, const std::string &name, Ext e)
{
    if (ctx->stage_tuning) return tune_stage<T>(ctx, prog, dir, name.c_str(), e);
    const auto it = ctx->stage_tuned.find(name);
    const int first = it != ctx->stage_tuned.end() ? it->second
                                                   : (is_stage_cfg(ctx->default_cfg) ? ctx->default_cfg : 0);
    int rc = launch_stage<T>(ctx, prog, dir, e.nx, e.ny, e.nz, first);
    for (int cfg = 0; rc == X3D_EUNSUPPORTED && cfg < kAllConfigs; ++cfg)
        if (cfg != first && is_stage_cfg(cfg)) rc = launch_stage<T>(ctx, prog, dir, e.nx, e.ny, e.nz, cfg);
    return rc;
}

// Runs a stage: one launch, or, where the autotuner found it faster, one
// launch per part of split_by_inputs (stages "<name>.1", "<name>.2", ...).
// While tuning, times both forms and records the choice as "<name>.parts".
template <typename T>
static int run_stage(x3d_ctx_s *ctx, const StageProgram<T> &prog, int dir, const char *cname, Ext e)
{
    const TraceRange trace(cname);
    const std::string name = stage_key(ctx, cname, e);
    StageProgram<T> part[kMaxStageOps];
    const int nparts = split_by_inputs<T>(prog, part);
    const auto it = ctx->stage_tuned.find(name + ".parts");
    const bool split = nparts > 1 && !ctx->stage_tuning && it != ctx->stage_tuned.end() && it->second == nparts;
    int rc = X3D_OK;
    if (!split) {
        rc = run_program<T>(ctx, prog, dir, name, e);
        if (rc || !ctx->stage_tuning || nparts < 2) return rc;
    }
    float total = 0.f;
    for (int q = 0; q < nparts && !rc; ++q) {
        const std::string pn = name + "." + std::to_string(q + 1);
        rc = run_program<T>(ctx, part[q], dir, pn, e);
        if (!rc && ctx->stage_tuning) total += ctx->stage_ms[pn];
    }
    if (ctx->stage_tuning) {
        ctx->stage_tuned[name + ".parts"] = !rc && total < ctx->stage_ms[name] ? nparts : 1;
        return rc == X3D_EUNSUPPORTED ? X3D_OK : rc;
    }
    return rc;
}

static x3d_op_s *B(x3d_ctx_s *ctx, int which) { return ctx->builtin[which]; }

// The momentum terms along direction d for the components comps[0..ncomp):
// the fields they read are staged once each, in component order.
//   du_c = add_c + d(u_d u_c)/dx_d + u_d d(u_c)/dx_d   (add null: no addend)
//   unew_c = u_c + dt du_c                           (unew non-null)
template <typename T>
static StageProgram<T> transeq_program(x3d_ctx_s *ctx, int d, const int *comps, int ncomp, void *const du[3],
                                       const void *const u[3], const void *const *add, void *const *unew,
                                       double dt)
{
    const int der_op[3] = {X3D_OP_DERX, X3D_OP_DERY, X3D_OP_DERZ};
    StageProgram<T> p;
    std::memset(&p, 0, sizeof(p));
    bool used[3] = {false, false, false};
    used[d] = true;
    for (int i = 0; i < ncomp; ++i) used[comps[i]] = true;
    int tile[3] = {-1, -1, -1};
    for (int c = 0; c < 3; ++c)
        if (used[c]) {
            tile[c] = p.ntiles;
            p.in[p.ntiles++] = static_cast<const T *>(u[c]);
        }
    p.nops = 2 * ncomp;
    for (int i = 0; i < ncomp; ++i) {
        const int c = comps[i];
        // u_d * d(u_c)/dx_d  (e.g. ux1 * derx(ux1), transeq.f90:107,114)
        StageOp<T> a = sop<T>(B(ctx, der_op[d]), tile[c]);
        a.mul_tile = (short)tile[d];
        a.accumulate = 0;
        // + d(u_d u_c)/dx_d   (e.g. derx(ux1*ux1), transeq.f90:101,106)
        StageOp<T> b = sop<T>(B(ctx, der_op[d]), tile[d], tile[c]);
        b.accumulate = 1;
        set_flush(b, du[c], add ? add[c] : nullptr);
        if (unew) {
            b.out2 = unew[c];
            b.base2 = u[c];
            b.scale2 = dt;
        }
        p.ops[2 * i] = a;
        p.ops[2 * i + 1] = b;
    }
    return p;
}

// The momentum terms along d for all three components: one launch, or two
// where the autotuner found them faster -- component o2 (staging u_d, u_o2),
// then d and o1 (staging u_d, u_o1).  When u is updated in place (unew = u)
// the launch that writes u_d runs last, and neither launch reads what the
// other writes.
template <typename T>
static int transeq_dir(x3d_ctx_s *ctx, int d, void *const du[3], const void *const u[3], const void *const *add,
                       void *const *unew, double dt, Ext e)
{
    static const char *const names[3] = {"transeq_x", "transeq_y", "transeq_z"};
    static const int all[3] = {0, 1, 2};
    const std::string name = stage_key(ctx, names[d], e);
    const int o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
    const int first[2] = {d, o1};
    const auto split_it = ctx->stage_tuned.find(name + ".split");
    const bool split = !ctx->stage_tuning && split_it != ctx->stage_tuned.end() && split_it->second;
    int rc;
    if (!split || ctx->stage_tuning) {
        rc = run_stage<T>(ctx, transeq_program<T>(ctx, d, all, 3, du, u, add, unew, dt), d, names[d], e);
        if (rc) return rc;
    }
    if (split || ctx->stage_tuning) {
        const std::string nb = std::string(names[d]) + ".b", na = std::string(names[d]) + ".a";
        rc = run_stage<T>(ctx, transeq_program<T>(ctx, d, &o2, 1, du, u, add, unew, dt), d, nb.c_str(), e);
        if (!rc) rc = run_stage<T>(ctx, transeq_program<T>(ctx, d, first, 2, du, u, add, unew, dt), d, na.c_str(), e);
        if (rc && !(ctx->stage_tuning && rc == X3D_EUNSUPPORTED)) return rc;
        if (ctx->stage_tuning) {
            const float t3 = ctx->stage_ms[name];
            const bool faster = !rc && ctx->stage_ms[stage_key(ctx, na.c_str(), e)] +
                                               ctx->stage_ms[stage_key(ctx, nb.c_str(), e)] <
                                           t3;
            ctx->stage_tuned[name + ".split"] = faster ? 1 : 0;
        }
    }
    return X3D_OK;
}

// momentum_rhs_eq on the box: x, then y and z accumulating into du; with a
// time step the z launch also applies int_time in place.
template <typename T>
static int transeq_t(x3d_ctx_s *ctx, void *const du[3], const void *const u[3], bool step, double dt,
                     void *const unew[3])
{
    const void *const acc[3] = {du[0], du[1], du[2]};
    for (int d = 0; d < 3; ++d) {
        const int rc = transeq_dir<T>(ctx, d, du, u, d == 0 ? nullptr : acc, step && d == 2 ? unew : nullptr, dt,
                                      box_ext(ctx));
        if (rc) return rc;
    }
    return X3D_OK;
}

// divergence (src/navier.f90:166-202), the part along dir:
//   x: pp1 = derxvp(ux), pgy1 = interxvp(uy), pgz1 = interxvp(uz)
//   y: duydypi2 = deryvp(pgy1) + interyvp(pp1) ; upi2 = interyvp(pgz1)
//   z: pp3 = interzvp(duydypi2) + derzvp(upi2), written in FP64
template <typename T>
static int divergence_dir(x3d_ctx_s *ctx, int dir, void *const *out, const void *const *in, Ext e)
{
    StageProgram<T> p;
    std::memset(&p, 0, sizeof(p));
    if (dir == DX) {
        p.ntiles = 3;
        p.nops = 3;
        for (int c = 0; c < 3; ++c) p.in[c] = static_cast<const T *>(in[c]);
        p.ops[0] = sop<T>(B(ctx, X3D_OP_DERXVP), 0);
        p.ops[1] = sop<T>(B(ctx, X3D_OP_INTXVP), 1);
        p.ops[2] = sop<T>(B(ctx, X3D_OP_INTXVP), 2);
        for (int k = 0; k < 3; ++k) set_flush(p.ops[k], out[k]);
        return run_stage<T>(ctx, p, DX, "div_x", e);
    }
    if (dir == DY) {
        p.ntiles = 3;
        p.nops = 3;
        for (int c = 0; c < 3; ++c) p.in[c] = static_cast<const T *>(in[c]);
        p.ops[0] = sop<T>(B(ctx, X3D_OP_INTYVP), 0);
        p.ops[1] = sop<T>(B(ctx, X3D_OP_DERYVP), 1);
        p.ops[1].accumulate = 1;
        set_flush(p.ops[1], out[0]);
        p.ops[2] = sop<T>(B(ctx, X3D_OP_INTYVP), 2);
        set_flush(p.ops[2], out[1]);
        return run_stage<T>(ctx, p, DY, "div_y", e);
    }
    p.ntiles = 2;
    p.nops = 2;
    p.in[0] = static_cast<const T *>(in[0]);
    p.in[1] = static_cast<const T *>(in[1]);
    p.ops[0] = sop<T>(B(ctx, X3D_OP_INTZVP), 0);
    p.ops[1] = sop<T>(B(ctx, X3D_OP_DERZVP), 1);
    p.ops[1].accumulate = 1;
    set_flush(p.ops[1], out[0], nullptr, true);
    return run_stage<T>(ctx, p, DZ, "div_z", e);
}

template <typename T>
static int divergence_t(x3d_ctx_s *ctx, double *pp3, const void *const u[3], void *const s[5])
{
    const Ext e = box_ext(ctx);
    int rc = divergence_dir<T>(ctx, DX, s, u, e);
    void *const y_out[2] = {s[3], s[4]};
    const void *const y_in[3] = {s[0], s[1], s[2]};
    if (!rc) rc = divergence_dir<T>(ctx, DY, y_out, y_in, e);
    void *const z_out[1] = {pp3};
    const void *const z_in[2] = {s[3], s[4]};
    if (!rc) rc = divergence_dir<T>(ctx, DZ, z_out, z_in, e);
    return rc;
}

// gradp (src/navier.f90:273-304) and cor_vel (:83-87), the part along dir:
//   z: ppi3 = interzpv(pp3), pgz3 = derzpv(pp3), from the FP64 pressure
//   y: ppi2 = interypv(ppi3), pgy2 = derypv(ppi3), pgzi2 = interypv(pgz3)
//   x: px = derxpv(ppi2), py = interxpv(pgy2), pz = interxpv(pgzi2);
//      with ucor, u_c -= p_c in place
// An FP32 step stages the FP64 pressure itself in its z launch where the
// kernels take it (even x extent); otherwise it solves an FP32 copy made in
// `copy` (the context's scratch field 5 when null: sized for the box).
template <typename T>
static int gradp_dir(x3d_ctx_s *ctx, int dir, void *const *out, const void *const *in, void *const *ucor, Ext e,
                     void *copy)
{
    StageProgram<T> p;
    std::memset(&p, 0, sizeof(p));
    if (dir == DZ) {
        p.ntiles = 1;
        p.nops = 2;
        p.in[0] = static_cast<const T *>(in[0]);
        p.in_f64 = sizeof(T) == 4 ? 1 : 0;
        p.ops[0] = sop<T>(B(ctx, X3D_OP_INTZPV), 0);
        set_flush(p.ops[0], out[0]);
        p.ops[1] = sop<T>(B(ctx, X3D_OP_DERZPV), 0);
        set_flush(p.ops[1], out[1]);
        int rc = run_stage<T>(ctx, p, DZ, "gradp_z", e);
        if (rc == X3D_EUNSUPPORTED && p.in_f64) {
            if (!copy && !(copy = ctx_scratch(ctx, 5)))
                return set_error(ctx, X3D_ENOMEM, "scratch allocation failed");
            const size_t n = (size_t)e.nx * e.ny * e.nz;
            if ((rc = launch_convert(ctx, copy, true, in[0], false, n))) return rc;
            p.in[0] = static_cast<const T *>(copy);
            p.in_f64 = 0;
            rc = run_stage<T>(ctx, p, DZ, "gradp_z.copy", e);
        }
        return rc;
    }
    if (dir == DY) {
        p.ntiles = 2;
        p.nops = 3;
        p.in[0] = static_cast<const T *>(in[0]);
        p.in[1] = static_cast<const T *>(in[1]);
        p.ops[0] = sop<T>(B(ctx, X3D_OP_INTYPV), 0);
        p.ops[1] = sop<T>(B(ctx, X3D_OP_DERYPV), 0);
        p.ops[2] = sop<T>(B(ctx, X3D_OP_INTYPV), 1);
        for (int k = 0; k < 3; ++k) set_flush(p.ops[k], out[k]);
        return run_stage<T>(ctx, p, DY, "gradp_y", e);
    }
    p.ntiles = 3;
    p.nops = 3;
    for (int c = 0; c < 3; ++c) p.in[c] = static_cast<const T *>(in[c]);
    const int xop[3] = {X3D_OP_DERXPV, X3D_OP_INTXPV, X3D_OP_INTXPV};
    for (int c = 0; c < 3; ++c) {
        p.ops[c] = sop<T>(B(ctx, xop[c]), c);
        set_flush(p.ops[c], out[c]);
        if (ucor) {
            p.ops[c].out2 = ucor[c];
            p.ops[c].base2 = ucor[c];
            p.ops[c].scale2 = -1.0;
        }
    }
    return run_stage<T>(ctx, p, DX, ucor ? "gradp_x_cor" : "gradp_x", e);
}

template <typename T>
static int gradp_t(x3d_ctx_s *ctx, void *const px[3], const double *pp3, void *const ucor[3], void *const s[6])
{
    const Ext e = box_ext(ctx);
    const void *const z_in[1] = {pp3};
    int rc = gradp_dir<T>(ctx, DZ, s, z_in, nullptr, e, s[5]);
    void *const y_out[3] = {s[2], s[3], s[4]};
    const void *const y_in[2] = {s[0], s[1]};
    if (!rc) rc = gradp_dir<T>(ctx, DY, y_out, y_in, nullptr, e, nullptr);
    const void *const x_in[3] = {s[2], s[3], s[4]};
    if (!rc) rc = gradp_dir<T>(ctx, DX, px, x_in, ucor, e, nullptr);
    return rc;
}

int fused_transeq(x3d_ctx_s *ctx, void *const du[3], const void *const u[3], bool step, double dt,
                  void *const unew[3])
{
    return ctx->precision == X3D_F32 ? transeq_t<float>(ctx, du, u, step, dt, unew)
                                     : transeq_t<double>(ctx, du, u, step, dt, unew);
}

int fused_divergence(x3d_ctx_s *ctx, double *pp3, const void *const u[3])
{
    void *s[5];
    for (int i = 0; i < 5; ++i)
        if (!(s[i] = ctx_scratch(ctx, i))) return set_error(ctx, X3D_ENOMEM, "scratch allocation failed");
    return ctx->precision == X3D_F32 ? divergence_t<float>(ctx, pp3, u, s) : divergence_t<double>(ctx, pp3, u, s);
}

// The fused divergence on caller-provided intermediate fields s[0..4] (each
// nx*ny*nz elements of the context precision); allocates nothing.
int fused_divergence_scratch(x3d_ctx_s *ctx, double *pp3, const void *const u[3], void *const s[5])
{
    return ctx->precision == X3D_F32 ? divergence_t<float>(ctx, pp3, u, s) : divergence_t<double>(ctx, pp3, u, s);
}

int fused_gradp(x3d_ctx_s *ctx, void *const px[3], const double *pp3, void *const ucor[3])
{
    void *s[6];
    for (int i = 0; i < 6; ++i)
        if (!(s[i] = ctx_scratch(ctx, i))) return set_error(ctx, X3D_ENOMEM, "scratch allocation failed");
    return ctx->precision == X3D_F32 ? gradp_t<float>(ctx, px, pp3, ucor, s) : gradp_t<double>(ctx, px, pp3, ucor, s);
}

// ---- the parts on one pencil (x3d_transeq_part etc.) ----------------------

int part_transeq(x3d_ctx_s *ctx, int dir, void *const du[3], const void *const u[3], const void *const *add,
                 void *const *unew, double dt, int nx, int ny, int nz)
{
    const Ext e{nx, ny, nz};
    return ctx->precision == X3D_F32 ? transeq_dir<float>(ctx, dir, du, u, add, unew, dt, e)
                                     : transeq_dir<double>(ctx, dir, du, u, add, unew, dt, e);
}

int part_divergence(x3d_ctx_s *ctx, int dir, void *const *out, const void *const *in, int nx, int ny, int nz)
{
    const Ext e{nx, ny, nz};
    return ctx->precision == X3D_F32 ? divergence_dir<float>(ctx, dir, out, in, e)
                                     : divergence_dir<double>(ctx, dir, out, in, e);
}

int part_gradp(x3d_ctx_s *ctx, int dir, void *const *out, const void *const *in, void *const *ucor, int nx, int ny,
               int nz)
{
    const Ext e{nx, ny, nz};
    return ctx->precision == X3D_F32 ? gradp_dir<float>(ctx, dir, out, in, ucor, e, nullptr)
                                     : gradp_dir<double>(ctx, dir, out, in, ucor, e, nullptr);
}

}  // namespace x3d
