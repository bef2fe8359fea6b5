// The C ABI (include/x3d_b200.h): argument checks, host-pointer staging,
// dispatch to the line-solve kernels, and the stage compositions of
// src/navier.f90, src/transeq.f90 and src/time_integrators.f90.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <new>
#include <string>
#include <vector>

#include "linesolve_chunk.h"
#include "x3d_internal.h"

using namespace x3d;

namespace x3d {

int set_error(x3d_ctx_s *ctx, int code, const std::string &msg)
{
    if (ctx) ctx->last_error = msg;
    return code;
}

int cuda_check(x3d_ctx_s *ctx, cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return X3D_OK;
    return set_error(ctx, X3D_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void *ctx_scratch(x3d_ctx_s *ctx, int idx)
{
    const size_t bytes = ctx->npts() * 8;  // large enough for either precision
    while ((int)ctx->scratch.size() <= idx) {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        ctx->scratch.push_back(p);
    }
    return ctx->scratch[idx];
}

}  // namespace x3d

namespace {

// Which table entry (kind, dir) each named operator instance is; derx and
// derxp are the same operator when periodic (first_deriv_imp_ only changes
// ffp for free-slip, src/x3d_operator_1d.f90:479-486).
struct Named {
    int kind, dir;
};
const Named kNamed[X3D_OP_COUNT] = {
    {DER, DX},   {DER, DX},   {DER, DY},   {DER, DY},   {DER, DZ},   {DER, DZ},   {DERVP, DX},
    {DERVP, DY}, {DERVP, DZ}, {DERPV, DX}, {DERPV, DY}, {DERPV, DZ}, {INTVP, DX}, {INTVP, DY},
    {INTVP, DZ}, {INTPV, DX}, {INTPV, DY}, {INTPV, DZ}, {DER2, DX},  {DER2, DY},  {DER2, DZ},
};

bool is_device_ptr(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// The device mirror of [p, p + bytes) when that range lies inside a host
// array registered with x3d_buf_register, else null.
void *resident_dev(const x3d_ctx_s *ctx, const void *p, size_t bytes)
{
    const char *c = static_cast<const char *>(p);
    for (const auto &r : ctx->resident) {
        const char *h = static_cast<const char *>(r.host);
        if (c >= h && c + bytes <= h + r.bytes) return static_cast<char *>(r.dev) + (c - h);
    }
    return nullptr;
}

// Host-pointer staging for one call: inputs are uploaded before the work,
// outputs downloaded after it, and the call then synchronises.
class Stager {
  public:
    explicit Stager(x3d_ctx_s *c) : ctx(c) {}
    ~Stager() { release(); }
    void *in(const void *p, size_t bytes) { return stage(const_cast<void *>(p), bytes, true, false); }
    void *out(void *p, size_t bytes) { return stage(p, bytes, false, true); }
    void *inout(void *p, size_t bytes) { return stage(p, bytes, true, true); }
    int status() const { return rc; }
    int finish(int work_rc)
    {
        if (work_rc) return work_rc;
        if (rc) return rc;
        if (!any_host) return X3D_OK;
        for (auto &it : items)
            if (it.out) {
                int r = cuda_check(ctx, cudaMemcpyAsync(it.user, it.dev, it.bytes, cudaMemcpyDeviceToHost, ctx->stream), "stage d2h");
                if (r) return r;
            }
        return cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "stage sync");
    }

  private:
    struct Item {
        void *user, *dev;
        size_t bytes;
        bool out;
    };
    x3d_ctx_s *ctx;
    std::vector<Item> items;
    size_t used = 0;  // staging-pool buffers taken by this call
    bool any_host = false;
    int rc = X3D_OK;
    void *stage(void *p, size_t bytes, bool upload, bool download)
    {
        if (!p || rc) return p;
        if (void *d = resident_dev(ctx, p, bytes)) return d;  // registered: no copies
        if (is_device_ptr(p)) return p;
        for (auto &it : items)  // the same host array passed twice maps to one device copy
            if (it.user == p) {
                it.out = it.out || download;
                return it.dev;
            }
        any_host = true;
        void *d = take(bytes);
        if (!d) {
            rc = set_error(ctx, X3D_ENOMEM, "staging allocation failed");
            return nullptr;
        }
        if (upload) {
            int r = cuda_check(ctx, cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, ctx->stream), "stage h2d");
            if (r) rc = r;
        }
        items.push_back({p, d, bytes, download});
        return d;
    }
    // The next device buffer of the context's staging pool, grown to bytes.
    // The pool outlives the call (freed by x3d_ctx_destroy), so repeated
    // calls on host arrays allocate nothing: allocating and mapping
    // hundreds of MB per call would cost more than the copies themselves.
    void *take(size_t bytes)
    {
        auto &pool = ctx->staging;
        if (used < pool.size() && pool[used].second >= bytes) return pool[used++].first;
        if (used < pool.size()) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(pool[used].first);
            pool[used] = {nullptr, 0};
        }
        void *d = nullptr;
        if (cudaMalloc(&d, bytes) != cudaSuccess) return nullptr;
        if (used < pool.size()) pool[used] = {d, bytes};
        else pool.push_back({d, bytes});
        ++used;
        return d;
    }
    // The pool's buffers may be taken by the next call only after this
    // call's copies are done.
    void release()
    {
        if (used) cudaStreamSynchronize(ctx->stream);
    }
};

int check_ctx(x3d_ctx_s *ctx)
{
    if (!ctx) return X3D_EINVAL;
    cudaSetDevice(ctx->device);
    return X3D_OK;
}

bool fp32(const x3d_ctx_s *ctx) { return ctx->precision == X3D_F32; }

// t(i,j,k) *= ppy(j) for a (nx, ny, nz) device field, ppy a host, device or
// registered array of ny doubles (the istret /= 0 multiply of dery_00,
// deryvp and derypv).
static int scale_by_metric(x3d_ctx_s *ctx, void *dt, const double *ppy, int nx, int ny, int nz)
{
    const double *dm = ppy;
    int rc = X3D_OK;
    if (const void *r = resident_dev(ctx, ppy, ny * sizeof(double))) {
        dm = static_cast<const double *>(r);
    } else if (!is_device_ptr(ppy)) {
        if (ctx->metric_len < ny) {
            if (ctx->d_metric) cudaFree(ctx->d_metric);
            ctx->d_metric = nullptr;
            ctx->metric_len = 0;
            if (cudaMalloc(&ctx->d_metric, ny * sizeof(double)) != cudaSuccess)
                return set_error(ctx, X3D_ENOMEM, "stretching metric allocation failed");
            ctx->metric_len = ny;
        }
        rc = cuda_check(ctx, cudaMemcpyAsync(ctx->d_metric, ppy, ny * sizeof(double), cudaMemcpyHostToDevice,
                                             ctx->stream),
                        "stretching metric upload");
        if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "stretching metric upload");
        dm = ctx->d_metric;
    }
    return rc ? rc : launch_scale_y(ctx, fp32(ctx), dt, dm, nx, ny, nz);
}

// One operator application on (nx,ny,nz) fields along dir; with ppy (a y
// operator of dery_00/deryvp/derypv given a stretching metric, host or
// device, ny values) the result is then multiplied by ppy(j).
int apply_op(x3d_ctx_s *ctx, void *t, const void *u, x3d_op_s *op, int want_kind, int want_dir,
             int nx, int ny, int nz, const double *ppy = nullptr)
{
    if (!op || !t || !u) return set_error(ctx, X3D_EINVAL, "null operator or field");
    if (op->h.kind != want_kind || op->h.dir != want_dir)
        return set_error(ctx, X3D_EINVAL, "operator kind/direction does not match the routine");
    if (nx <= 0 || ny <= 0 || nz <= 0) return set_error(ctx, X3D_EINVAL, "bad field shape");
    const int n = want_dir == DX ? nx : (want_dir == DY ? ny : nz);
    if (op->h.n != n) return set_error(ctx, X3D_EINVAL, "operator length differs from the line length");
    if (!op->h.periodic && (op->h.kind != DER || !op->h.ncl1))
        return set_error(ctx, X3D_EUNSUPPORTED,
                         "only periodic operators and the library's non-periodic first derivatives are supported");
    if (t == u) return set_error(ctx, X3D_EINVAL, "t and u must not alias (t is intent(out))");
    const size_t bytes = (size_t)nx * ny * nz * ctx->elem();
    Stager sg(ctx);
    void *du = sg.in(u, bytes);
    void *dt = sg.out(t, bytes);
    if (sg.status()) return sg.status();
    int rc = launch_linesolve(ctx, op, want_kind, want_dir, du, dt, nx, ny, nz, fp32(ctx));
    if (!rc && ppy) rc = scale_by_metric(ctx, dt, ppy, nx, ny, nz);
    return sg.finish(rc);
}

// A staggered operator along a non-periodic direction (src/x3d_staggered.f90,
// the nclx = .false. branches): input of n_in points along dir, output of
// n_out = n_in -/+ 1 (the pressure grid has nxm = nx - 1 points); nx, ny, nz
// are the velocity-grid extents.  ppy: as in apply_op, for the output's ny.
int apply_stag_np(x3d_ctx_s *ctx, void *t, const void *u, x3d_op_s *op, int kind, int dir, int n_in, int n_out,
                  int nx, int ny, int nz, const double *ppy = nullptr)
{
    if (!op || !t || !u) return set_error(ctx, X3D_EINVAL, "null operator or field");
    if (op->h.kind != kind || op->h.dir != dir)
        return set_error(ctx, X3D_EINVAL, "operator kind/direction does not match the routine");
    if (op->h.periodic) return set_error(ctx, X3D_EINVAL, "a periodic staggered operator needs nxm = nx");
    const bool vp = kind == DERVP || kind == INTVP;
    const int nv = dir == DX ? nx : (dir == DY ? ny : nz);
    if ((vp ? (n_in != nv || n_out != nv - 1) : (n_out != nv || n_in != nv - 1)) || op->h.n != n_out || nv < 9)
        return set_error(ctx, X3D_EINVAL, "extents do not match the non-periodic staggered grids");
    if (t == u) return set_error(ctx, X3D_EINVAL, "t and u must not alias (t is intent(out))");
    const int o1 = dir == DX ? ny : nx, o2 = dir == DZ ? ny : nz;
    const size_t es = ctx->elem();
    Stager sg(ctx);
    void *du = sg.in(u, (size_t)n_in * o1 * o2 * es);
    void *dt = sg.out(t, (size_t)n_out * o1 * o2 * es);
    if (sg.status()) return sg.status();
    int rc = launch_np_stag(ctx, op, dir, du, dt, n_in, o1, o2, fp32(ctx));
    if (!rc && ppy) rc = scale_by_metric(ctx, dt, ppy, nx, n_out, nz);
    return sg.finish(rc);
}

int thomas_call(x3d_ctx_s *ctx, int dir, void *tt, const double *ff, const double *fs,
                const double *fw, const double *perio, double alfa, int nx, int ny, int nz)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!tt || !ff || !fs || !fw) return set_error(ctx, X3D_EINVAL, "null argument");
    const int n = dir == DX ? nx : (dir == DY ? ny : nz);
    if (n < 8) return set_error(ctx, X3D_EUNSUPPORTED, "line length must be >= 8");
    // The coefficient arrays may live on either side; bring them to the host.
    auto fetch = [&](const double *p, std::vector<double> &v) {
        v.resize(n);
        if (is_device_ptr(p))
            return cudaMemcpy(v.data(), p, n * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess;
        std::memcpy(v.data(), p, n * sizeof(double));
        return true;
    };
    x3d_op_s op;
    op.h.kind = IDENT;
    op.h.dir = dir;
    op.h.n = n;
    op.h.alfa = alfa;
    op.h.periodic = perio ? 1 : 0;
    if (!fetch(ff, op.h.f) || !fetch(fs, op.h.s) || !fetch(fw, op.h.w))
        return set_error(ctx, X3D_ECUDA, "coefficient copy failed");
    if (perio && !fetch(perio, op.h.per)) return set_error(ctx, X3D_ECUDA, "coefficient copy failed");
    finish_op(op.h);
    rc = upload_op(&op);
    if (rc) {
        free_op(&op);
        return set_error(ctx, rc, "operator upload failed");
    }
    const size_t bytes = (size_t)nx * ny * nz * ctx->elem();
    Stager sg(ctx);
    void *d = sg.inout(tt, bytes);
    if (sg.status()) {
        free_op(&op);
        return sg.status();
    }
    rc = sg.finish(launch_linesolve(ctx, &op, IDENT, dir, d, d, nx, ny, nz, fp32(ctx)));
    cudaStreamSynchronize(ctx->stream);  // the temporary operator dies here
    free_op(&op);
    return rc;
}

int check_shape(x3d_ctx_s *ctx, int nx, int ny, int nz)
{
    if (nx != ctx->nx || ny != ctx->ny || nz != ctx->nz)
        return set_error(ctx, X3D_EINVAL, "field shape differs from the context grid");
    return X3D_OK;
}

}  // namespace

extern "C" {

// ---- context ----------------------------------------------------------------

int x3d_ctx_create(x3d_ctx *out, int nx, int ny, int nz, double xlx, double yly, double zlz,
                   int precision, int device)
{
    return x3d_ctx_create_bc(out, nx, ny, nz, xlx, yly, zlz, precision, device, nullptr);
}

int x3d_ctx_create_bc(x3d_ctx *out, int nx, int ny, int nz, double xlx, double yly, double zlz,
                      int precision, int device, const int *ncl_in)
{
    if (!out) return X3D_EINVAL;
    *out = nullptr;
    int ncl[6] = {0, 0, 0, 0, 0, 0};
    if (ncl_in)
        for (int i = 0; i < 6; ++i) ncl[i] = ncl_in[i];
    for (int d = 0; d < 3; ++d) {
        const int a = ncl[2 * d], b = ncl[2 * d + 1];
        if (a < 0 || a > 2 || b < 0 || b > 2) return X3D_EINVAL;
        if ((a == 0) != (b == 0)) return X3D_EINVAL;  // periodic means both ends
    }
    if (nx < 8 || ny < 8 || nz < 8) return X3D_EUNSUPPORTED;
    if (precision != X3D_F64 && precision != X3D_F32) return X3D_EINVAL;
    if (!(xlx > 0 && yly > 0 && zlz > 0)) return X3D_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return X3D_ECUDA;
    auto *ctx = new (std::nothrow) x3d_ctx_s;
    if (!ctx) return X3D_ENOMEM;
    ctx->nx = nx; ctx->ny = ny; ctx->nz = nz;
    ctx->xlx = xlx; ctx->yly = yly; ctx->zlz = zlz;
    // parameter(): dx = xlx/nxm with nxm = nx when periodic, nx - 1 otherwise
    // (src/parameters.f90:51-71)
    ctx->dx = xlx / (ncl[0] ? nx - 1 : nx);
    ctx->dy = yly / (ncl[2] ? ny - 1 : ny);
    ctx->dz = zlz / (ncl[4] ? nz - 1 : nz);
    for (int i = 0; i < 6; ++i) ctx->ncl[i] = ncl[i];
    ctx->periodic_all = !(ncl[0] || ncl[2] || ncl[4]);
    ctx->precision = precision;
    ctx->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete ctx;
        return X3D_ECUDA;
    }
    ctx->num_sms = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->d_err, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->d_red, 4 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&ctx->d_claim, sizeof(unsigned long long)) != cudaSuccess) {
        x3d_ctx_destroy(ctx);
        return X3D_ECUDA;
    }
    cudaMemset(ctx->d_err, 0, sizeof(int));
    ctx->stream = ctx->own_stream;
    const double dd[3] = {ctx->dx, ctx->dy, ctx->dz};
    const int nn[3] = {nx, ny, nz};
    for (int w = 0; w < X3D_OP_COUNT; ++w) {
        auto *op = new (std::nothrow) x3d_op_s;
        if (!op) {
            x3d_ctx_destroy(ctx);
            return X3D_ENOMEM;
        }
        op->builtin = true;
        const int d = kNamed[w].dir;
        int rc;
        if (!ncl[2 * d]) {
            rc = build_periodic_op(kNamed[w].kind, d, nn[d], dd[d], op->h);
        } else if (kNamed[w].kind == DER) {
            // derx (npaire 0) and derxp (npaire 1), x3d_operator_1d_init :140-141
            rc = build_nonperiodic_der(d, nn[d], dd[d], ncl[2 * d], ncl[2 * d + 1], (w & 1) ? 1 : 0, op->h);
        } else if (kNamed[w].kind != DER2) {
            // staggered operators with the parities x3d_operator_1d_init binds
            // (:152-189): derxvp 1, derxpv 0, intxvp 1, intxpv 1
            const int k = kNamed[w].kind;
            rc = build_nonperiodic_stag(k, d, nn[d], dd[d], ncl[2 * d], ncl[2 * d + 1], k == DERPV ? 0 : 1,
                                        op->h);
        } else {
            delete op;  // defined for periodic directions only
            continue;
        }
        ctx->builtin[w] = op;
        if (!rc) rc = upload_op(op);
        if (rc) {
            x3d_ctx_destroy(ctx);
            return rc;
        }
    }
    *out = ctx;
    return X3D_OK;
}

int x3d_ctx_destroy(x3d_ctx ctx)
{
    if (!ctx) return X3D_EINVAL;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto *&op : ctx->builtin) {
        if (op) {
            free_op(op);
            delete op;
        }
        op = nullptr;
    }
    poisson_free(ctx);
    for (void *p : ctx->scratch) cudaFree(p);
    ctx->scratch.clear();
    for (auto &b : ctx->staging) cudaFree(b.first);
    ctx->staging.clear();
    for (auto &r : ctx->resident) cudaFree(r.dev);
    ctx->resident.clear();
    if (ctx->step_exec) cudaGraphExecDestroy(ctx->step_exec);
    if (ctx->step_graph) cudaGraphDestroy(ctx->step_graph);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->d_red) cudaFree(ctx->d_red);
    if (ctx->d_claim) cudaFree(ctx->d_claim);
    if (ctx->d_metric) cudaFree(ctx->d_metric);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return X3D_OK;
}

int x3d_ctx_set_stream(x3d_ctx ctx, void *stream)
{
    if (!ctx) return X3D_EINVAL;
    ctx->stream = static_cast<cudaStream_t>(stream);
    return X3D_OK;
}

int x3d_ctx_launch_count(x3d_ctx ctx, unsigned long long *count)
{
    if (!ctx || !count) return X3D_EINVAL;
    *count = ctx->launches;
    return X3D_OK;
}

int x3d_ctx_last_kernel(x3d_ctx ctx, int *cfg)
{
    if (!ctx || !cfg) return X3D_EINVAL;
    *cfg = ctx->last_cfg;
    return X3D_OK;
}

int x3d_ctx_get_stream(x3d_ctx ctx, void **stream)
{
    if (!ctx || !stream) return X3D_EINVAL;
    *stream = ctx->stream;
    return X3D_OK;
}

int x3d_ctx_sync(x3d_ctx ctx)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "stream sync");
    if (rc) return rc;
    int flag = 0;
    rc = cuda_check(ctx, cudaMemcpy(&flag, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost), "error flag read");
    if (rc) return rc;
    if (flag) {
        cudaMemset(ctx->d_err, 0, sizeof(int));
        return set_error(ctx, X3D_ETIMEOUT, "a device-side bounded wait gave up (code " + std::to_string(flag) + ")");
    }
    return X3D_OK;
}

int x3d_roofline_probe(x3d_ctx ctx, int pattern, int w, int ctas_per_sm, const void *in, void *const *outs, int nx,
                       int ny, int nz)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!in || !outs || nx < 1 || ny < 1 || nz < 1 || pattern < 0 || pattern > 6)
        return set_error(ctx, X3D_EINVAL, "bad probe request");
    float *o[6];
    for (int k = 0; k < 6; ++k) {
        if (!outs[k] || !is_device_ptr(outs[k])) return set_error(ctx, X3D_EINVAL, "probe outputs must be device arrays");
        o[k] = static_cast<float *>(outs[k]);
    }
    if (!is_device_ptr(in)) return set_error(ctx, X3D_EINVAL, "probe input must be a device array");
    if (ctas_per_sm < 0 || ctas_per_sm > 32) return set_error(ctx, X3D_EINVAL, "ctas_per_sm must be 0..32");
    return launch_roofline_probe(ctx, pattern, w, ctas_per_sm, static_cast<const float *>(in), o, nx, ny, nz);
}

int x3d_ctx_selftest_timeout(x3d_ctx ctx, double limit_s)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!(limit_s > 0.0 && limit_s <= 1.0)) return set_error(ctx, X3D_EINVAL, "limit must be in (0, 1] s");
    return launch_wait_selftest(ctx, (uint64_t)(limit_s * 1e9));
}

const char *x3d_ctx_last_error(x3d_ctx ctx)
{
    if (!ctx) return "null context";
    return ctx->last_error.c_str();
}

int x3d_ctx_geometry(x3d_ctx ctx, int *dims, double *lengths, double *spacing, int *precision)
{
    if (!ctx) return X3D_EINVAL;
    if (dims) { dims[0] = ctx->nx; dims[1] = ctx->ny; dims[2] = ctx->nz; }
    if (lengths) { lengths[0] = ctx->xlx; lengths[1] = ctx->yly; lengths[2] = ctx->zlz; }
    if (spacing) { spacing[0] = ctx->dx; spacing[1] = ctx->dy; spacing[2] = ctx->dz; }
    if (precision) *precision = ctx->precision;
    return X3D_OK;
}

// ---- operators ------------------------------------------------------------------

int x3d_op_builtin(x3d_ctx ctx, int which, x3d_op *op)
{
    if (!ctx || !op) return X3D_EINVAL;
    if (which < 0 || which >= X3D_OP_COUNT) return set_error(ctx, X3D_EINVAL, "unknown operator instance");
    if (!ctx->builtin[which])
        return set_error(ctx, X3D_EUNSUPPORTED,
                         "operator not defined: only first derivatives exist along a non-periodic direction");
    *op = ctx->builtin[which];
    return X3D_OK;
}

int x3d_op_create(x3d_ctx ctx, int kind, int dir, int n, int npaire, double alfa, const double *f,
                  const double *s, const double *w, const double *periodic, const double *rhs,
                  x3d_op *out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || !f || !s || !w || !rhs) return set_error(ctx, X3D_EINVAL, "null argument");
    if (kind < DER || kind > INTPV || dir < DX || dir > DZ) return set_error(ctx, X3D_EINVAL, "bad kind or direction");
    if (n < 8) return set_error(ctx, X3D_EUNSUPPORTED, "line length must be >= 8");
    const bool stag = kind == DERVP || kind == DERPV || kind == INTVP || kind == INTPV;
    if (!periodic && !stag)
        return set_error(ctx, X3D_EUNSUPPORTED,
                         "a non-periodic first or second derivative needs its boundary closures (x3d_ctx_create_bc)");
    auto *op = new (std::nothrow) x3d_op_s;
    if (!op) return X3D_ENOMEM;
    op->h.kind = kind;
    op->h.dir = dir;
    op->h.n = n;
    op->h.npaire = npaire;
    op->h.periodic = periodic ? 1 : 0;
    op->h.alfa = alfa;
    op->h.a = rhs[0]; op->h.b = rhs[1]; op->h.c = rhs[2]; op->h.d = rhs[3];
    op->h.f.assign(f, f + n);
    op->h.s.assign(s, s + n);
    op->h.w.assign(w, w + n);
    if (periodic) op->h.per.assign(periodic, periodic + n);
    else op->h.per.clear();
    finish_op(op->h);
    rc = upload_op(op);
    if (rc) {
        free_op(op);
        delete op;
        return set_error(ctx, rc, "operator upload failed");
    }
    *out = op;
    return X3D_OK;
}

int x3d_op_destroy(x3d_ctx ctx, x3d_op op)
{
    if (!ctx || !op) return X3D_EINVAL;
    if (op->builtin) return set_error(ctx, X3D_EINVAL, "built-in operators belong to the context");
    cudaStreamSynchronize(ctx->stream);
    free_op(op);
    delete op;
    return X3D_OK;
}

int x3d_op_info(x3d_op op, int *meta, double *scal, double *f, double *s, double *w, double *periodic)
{
    if (!op) return X3D_EINVAL;
    const OpHost &h = op->h;
    if (meta) { meta[0] = h.n; meta[1] = h.kind; meta[2] = h.dir; meta[3] = h.npaire; }
    if (scal) { scal[0] = h.alfa; scal[1] = h.a; scal[2] = h.b; scal[3] = h.c; scal[4] = h.d; }
    if (f) std::memcpy(f, h.f.data(), h.n * sizeof(double));
    if (s) std::memcpy(s, h.s.data(), h.n * sizeof(double));
    if (w) std::memcpy(w, h.w.data(), h.n * sizeof(double));
    if (periodic) {
        if (h.per.empty()) std::memset(periodic, 0, h.n * sizeof(double));
        else std::memcpy(periodic, h.per.data(), h.n * sizeof(double));
    }
    return X3D_OK;
}

// ---- derivatives ------------------------------------------------------------------

#define X3D_APPLY(kind, dir, t, u, op, nx, ny, nz)              \
    do {                                                        \
        int rc_ = check_ctx(ctx);                               \
        if (rc_) return rc_;                                    \
        return apply_op(ctx, t, u, op, kind, dir, nx, ny, nz);  \
    } while (0)

int x3d_derx(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nx, int ny, int nz)
{ X3D_APPLY(DER, DX, tx, ux, op, nx, ny, nz); }
int x3d_dery(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, const double *ppy, int nx, int ny, int nz)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    return apply_op(ctx, ty, uy, op, DER, DY, nx, ny, nz, ppy);
}
int x3d_derz(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nz)
{ X3D_APPLY(DER, DZ, tz, uz, op, nx, ny, nz); }
int x3d_derxx(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nx, int ny, int nz)
{ X3D_APPLY(DER2, DX, tx, ux, op, nx, ny, nz); }
int x3d_deryy(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, int nx, int ny, int nz)
{ X3D_APPLY(DER2, DY, ty, uy, op, nx, ny, nz); }
int x3d_derzz(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nz)
{ X3D_APPLY(DER2, DZ, tz, uz, op, nx, ny, nz); }

// ---- staggered ----------------------------------------------------------------------
// Periodic only: the pressure-grid length equals the velocity-grid length.
#define X3D_STAG(kind, dir, t, u, op, n_in, n_out, nx, ny, nz)                                      \
    do {                                                                                            \
        int rc_ = check_ctx(ctx);                                                                   \
        if (rc_) return rc_;                                                                        \
        if ((n_in) != (n_out))                                                                      \
            return apply_stag_np(ctx, t, u, op, kind, dir, n_in, n_out, nx, ny, nz);                \
        return apply_op(ctx, t, u, op, kind, dir, nx, ny, nz);                                      \
    } while (0)

int x3d_derxvp(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nx, int nxm, int ny, int nz)
{ X3D_STAG(DERVP, DX, tx, ux, op, nx, nxm, nx, ny, nz); }
int x3d_interxvp(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nx, int nxm, int ny, int nz)
{ X3D_STAG(INTVP, DX, tx, ux, op, nx, nxm, nx, ny, nz); }
int x3d_derxpv(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nxm, int nx, int ny, int nz)
{ X3D_STAG(DERPV, DX, tx, ux, op, nxm, nx, nx, ny, nz); }
int x3d_interxpv(x3d_ctx ctx, void *tx, const void *ux, x3d_op op, int nxm, int nx, int ny, int nz)
{ X3D_STAG(INTPV, DX, tx, ux, op, nxm, nx, nx, ny, nz); }
int x3d_interyvp(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, int nx, int ny, int nym, int nz)
{ X3D_STAG(INTVP, DY, ty, uy, op, ny, nym, nx, ny, nz); }
int x3d_deryvp(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, const double *ppyi, int nx, int ny, int nym, int nz)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (ny != nym) return apply_stag_np(ctx, ty, uy, op, DERVP, DY, ny, nym, nx, ny, nz, ppyi);
    return apply_op(ctx, ty, uy, op, DERVP, DY, nx, ny, nz, ppyi);
}
int x3d_interypv(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, int nx, int nym, int ny, int nz)
{ X3D_STAG(INTPV, DY, ty, uy, op, nym, ny, nx, ny, nz); }
int x3d_derypv(x3d_ctx ctx, void *ty, const void *uy, x3d_op op, const double *ppy, int nx, int nym, int ny, int nz)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (ny != nym) return apply_stag_np(ctx, ty, uy, op, DERPV, DY, nym, ny, nx, ny, nz, ppy);
    return apply_op(ctx, ty, uy, op, DERPV, DY, nx, ny, nz, ppy);
}
int x3d_derzvp(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nz, int nzm)
{ X3D_STAG(DERVP, DZ, tz, uz, op, nz, nzm, nx, ny, nz); }
int x3d_interzvp(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nz, int nzm)
{ X3D_STAG(INTVP, DZ, tz, uz, op, nz, nzm, nx, ny, nz); }
int x3d_derzpv(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nzm, int nz)
{ X3D_STAG(DERPV, DZ, tz, uz, op, nzm, nz, nx, ny, nz); }
int x3d_interzpv(x3d_ctx ctx, void *tz, const void *uz, x3d_op op, int nx, int ny, int nzm, int nz)
{ X3D_STAG(INTPV, DZ, tz, uz, op, nzm, nz, nx, ny, nz); }

// ---- batch ----------------------------------------------------------------------------

int x3d_apply(x3d_ctx ctx, x3d_op op, const void *in, void *out)
{
    const x3d_work item{op, in, out};
    return x3d_apply_batch(ctx, &item, 1);
}

int x3d_apply_batch(x3d_ctx ctx, const x3d_work *items, int count)
{
    const TraceRange trace("apply_batch");
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (count < 0 || (count > 0 && !items)) return set_error(ctx, X3D_EINVAL, "bad work-list");
    const size_t bytes = ctx->npts() * ctx->elem();
    for (int i = 0; i < count; ++i) {
        const x3d_op_s *op = items[i].op;
        if (!op || !items[i].in || !items[i].out) return set_error(ctx, X3D_EINVAL, "null work item");
        const int n = op->h.dir == DX ? ctx->nx : (op->h.dir == DY ? ctx->ny : ctx->nz);
        if (op->h.n != n) return set_error(ctx, X3D_EINVAL, "operator does not fit the grid");
        if (!op->h.periodic && (op->h.kind != DER || !op->h.ncl1))
            return set_error(ctx, X3D_EUNSUPPORTED,
                             "only periodic operators and the library's non-periodic first derivatives are supported");
        for (int j = 0; j < count; ++j)
            if (items[i].out == items[j].in) return set_error(ctx, X3D_EINVAL, "an output aliases an input");
    }
    Stager sg(ctx);
    std::vector<const void *> din(count);
    std::vector<void *> dout(count);
    for (int i = 0; i < count; ++i) din[i] = sg.in(items[i].in, bytes);
    for (int i = 0; i < count; ++i) dout[i] = sg.out(items[i].out, bytes);
    if (sg.status()) return sg.status();
    // Items that read the same input along the same direction share one
    // staged read: up to six of them go into one multi-output launch.
    std::vector<char> done(count, 0);
    for (int i = 0; i < count && !rc; ++i) {
        if (done[i]) continue;
        const x3d_op_s *gops[6];
        int gkind[6];
        void *gout[6];
        int k = 0;
        for (int j = i; j < count && k < 6; ++j) {
            if (done[j] || din[j] != din[i] || items[j].op->h.dir != items[i].op->h.dir) continue;
            gops[k] = items[j].op;
            gkind[k] = items[j].op->h.kind;
            gout[k] = dout[j];
            ++k;
            done[j] = 1;
        }
        rc = launch_group(ctx, items[i].op->h.dir, din[i], gops, gkind, gout, k, ctx->nx, ctx->ny,
                          ctx->nz, fp32(ctx));
    }
    return sg.finish(rc);
}

int x3d_autotune(x3d_ctx ctx, int max_group)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (max_group < 1 || max_group > 6) return set_error(ctx, X3D_EINVAL, "max_group must be 1..6");
    if (cudaStreamCaptureStatus st; cudaStreamIsCapturing(ctx->stream, &st) == cudaSuccess &&
                                    st != cudaStreamCaptureStatusNone)
        return set_error(ctx, X3D_EINVAL, "cannot autotune during stream capture");
    void *buf[7];
    for (int i = 0; i < 7; ++i)
        if (!(buf[i] = ctx_scratch(ctx, i))) return set_error(ctx, X3D_ENOMEM, "scratch allocation failed");
    rc = cuda_check(ctx, cudaMemsetAsync(buf[0], 0, ctx->npts() * ctx->elem(), ctx->stream), "memset");
    const int kinds[6] = {DER, DER2, DERVP, DERPV, INTVP, INTPV};
    const int sizes[4] = {1, 2, 3, 6};
    for (int dir = 0; dir < 3 && !rc; ++dir)
        for (int g : sizes) {
            if (g > max_group || rc) continue;
            const x3d_op_s *ops[6];
            void *outs[6];
            for (int k = 0; k < g; ++k) {
                const int idx = [&] {
                    for (int w = 0; w < X3D_OP_COUNT; ++w)
                        if (ctx->builtin[w] && ctx->builtin[w]->h.kind == kinds[k] && ctx->builtin[w]->h.dir == dir)
                            return w;
                    return -1;
                }();
                if (idx < 0) {  // only first derivatives along a non-periodic direction
                    g = 0;
                    break;
                }
                ops[k] = ctx->builtin[idx];
                outs[k] = buf[1 + k];
            }
            if (g) rc = autotune_group(ctx, dir, buf[0], ops, kinds, outs, g, fp32(ctx), 3, nullptr);
        }
    if (rc || !ctx->periodic_all) return rc;  // the Euler stages need every direction periodic
    // the fused stages of the Euler step (transeq + int_time, divergence,
    // gradp + cor_vel), run once on scratch fields 7..13 with every
    // configuration timed; fields 0..5 are the stages' own intermediates
    void *u[3], *du[3];
    for (int i = 0; i < 3 && !rc; ++i) {
        u[i] = ctx_scratch(ctx, 7 + i);
        du[i] = ctx_scratch(ctx, 10 + i);
        if (!u[i] || !du[i]) return set_error(ctx, X3D_ENOMEM, "scratch allocation failed");
        rc = cuda_check(ctx, cudaMemsetAsync(u[i], 0, ctx->npts() * ctx->elem(), ctx->stream), "memset");
        if (!rc) rc = cuda_check(ctx, cudaMemsetAsync(du[i], 0, ctx->npts() * ctx->elem(), ctx->stream), "memset");
    }
    double *pp3 = static_cast<double *>(ctx_scratch(ctx, 13));
    if (!pp3) return set_error(ctx, X3D_ENOMEM, "scratch allocation failed");
    if (rc) return rc;
    ctx->stage_tuning = true;
    const void *uc[3] = {u[0], u[1], u[2]};
    rc = fused_transeq(ctx, du, uc, true, 0.0, u);
    if (!rc || rc == X3D_EUNSUPPORTED) rc = fused_divergence(ctx, pp3, uc);
    if (!rc || rc == X3D_EUNSUPPORTED) rc = fused_gradp(ctx, du, pp3, nullptr);
    if (!rc || rc == X3D_EUNSUPPORTED) rc = fused_gradp(ctx, du, pp3, u);
    ctx->stage_tuning = false;
    // a grid no fused stage can take keeps the unfused path
    return rc == X3D_EUNSUPPORTED ? X3D_OK : rc;
}

int x3d_ctx_set_kernel(x3d_ctx ctx, int cfg)
{
    if (!ctx || cfg < -1 || cfg >= kAllConfigs) return X3D_EINVAL;
    ctx->tuned.clear();
    ctx->stage_tuned.clear();
    ctx->stage_ms.clear();
    ctx->default_cfg = cfg < 0 ? 0 : cfg;
    return X3D_OK;
}

int x3d_autotune_choice(x3d_ctx ctx, int dir, int group, int *cfg)
{
    if (!ctx || !cfg) return X3D_EINVAL;
    const std::string key = std::to_string(dir) + ":" + std::to_string(ctx->nx) + "x" +
                            std::to_string(ctx->ny) + "x" + std::to_string(ctx->nz) + ":" +
                            (fp32(ctx) ? "f32" : "f64") + ":" + std::to_string(group);
    const auto it = ctx->tuned.find(key);
    *cfg = it == ctx->tuned.end() ? -1 : it->second;
    return X3D_OK;
}

int x3d_autotune_stage_choice(x3d_ctx ctx, const char *stage, int *cfg)
{
    if (!ctx || !stage || !cfg) return X3D_EINVAL;
    const auto it = ctx->stage_tuned.find(stage);
    *cfg = it == ctx->stage_tuned.end() ? -1 : it->second;
    return X3D_OK;
}

int x3d_ctx_set_stage_choice(x3d_ctx ctx, const char *stage, int value)
{
    if (!ctx || !stage || !*stage) return X3D_EINVAL;
    const std::string s = stage;
    const auto ends = [&](const char *suf) {
        const size_t n = std::strlen(suf);
        return s.size() > n && s.compare(s.size() - n, n, suf) == 0;
    };
    if (value < -1) return set_error(ctx, X3D_EINVAL, "stage choice below -1");
    if ((ends(".split") || s == "poisson_x") && value > 1)
        return set_error(ctx, X3D_EINVAL, "a split or poisson_x choice is 0 or 1");
    if (!ends(".split") && !ends(".parts") && s != "poisson_x" && value >= 0 && !is_stage_cfg(value))
        return set_error(ctx, X3D_EINVAL, "stage configurations are 0..15 and 17..20");
    if (value == -1) ctx->stage_tuned.erase(s);
    else ctx->stage_tuned[s] = value;
    return X3D_OK;
}

// ---- Thomas ------------------------------------------------------------------------

int x3d_xthomas(x3d_ctx ctx, void *tt, const double *ff, const double *fs, const double *fw,
                const double *perio, double alfa, int nx, int ny, int nz)
{ return thomas_call(ctx, DX, tt, ff, fs, fw, perio, alfa, nx, ny, nz); }
int x3d_ythomas(x3d_ctx ctx, void *tt, const double *ff, const double *fs, const double *fw,
                const double *perio, double alfa, int nx, int ny, int nz)
{ return thomas_call(ctx, DY, tt, ff, fs, fw, perio, alfa, nx, ny, nz); }
int x3d_zthomas(x3d_ctx ctx, void *tt, const double *ff, const double *fs, const double *fw,
                const double *perio, double alfa, int nx, int ny, int nz)
{ return thomas_call(ctx, DZ, tt, ff, fs, fw, perio, alfa, nx, ny, nz); }

// ---- transposes ---------------------------------------------------------------------

static int transpose_copy(x3d_ctx ctx, const void *in, void *out, int is_complex)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!in || !out) return set_error(ctx, X3D_EINVAL, "null field");
    const size_t bytes = ctx->npts() * ctx->elem() * (is_complex ? 2 : 1);
    Stager sg(ctx);
    void *di = sg.in(in, bytes);
    void *dout = sg.out(out, bytes);
    if (sg.status()) return sg.status();
    return sg.finish(launch_copy(ctx, dout, di, bytes));
}

int x3d_transpose_x_to_y(x3d_ctx ctx, const void *in, void *out, int c) { return transpose_copy(ctx, in, out, c); }
int x3d_transpose_y_to_z(x3d_ctx ctx, const void *in, void *out, int c) { return transpose_copy(ctx, in, out, c); }
int x3d_transpose_z_to_y(x3d_ctx ctx, const void *in, void *out, int c) { return transpose_copy(ctx, in, out, c); }
int x3d_transpose_y_to_x(x3d_ctx ctx, const void *in, void *out, int c) { return transpose_copy(ctx, in, out, c); }

int x3d_copy_blocks(x3d_ctx ctx, void *dst, const void *src, int elem_bytes, const x3d_block *blocks, int count)
{
    const int rc = check_ctx(ctx);
    if (rc) return rc;
    if (elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16)
        return set_error(ctx, X3D_EINVAL, "elem_bytes must be 4, 8 or 16");
    if (count < 0 || (count > 0 && !blocks)) return set_error(ctx, X3D_EINVAL, "bad block list");
    if (count == 0) return X3D_OK;
    if (!dst || !src || !is_device_ptr(dst) || !is_device_ptr(src))
        return set_error(ctx, X3D_EINVAL, "block copies take device arrays");
    for (int i = 0; i < count; ++i) {
        const x3d_block &b = blocks[i];
        if (b.nx < 0 || b.ny < 0 || b.nz < 0 || b.src_offset < 0 || b.dst_offset < 0 || b.src_ystride < 0 ||
            b.src_zstride < 0 || b.dst_ystride < 0 || b.dst_zstride < 0)
            return set_error(ctx, X3D_EINVAL, "negative block extent, offset or stride");
    }
    return copy_blocks(ctx, dst, src, elem_bytes, blocks, count);
}

// ---- Poisson -------------------------------------------------------------------------

// The Euler-step compositions use the staggered operators, which exist only
// when every direction is periodic (the reference's Poisson solver likewise
// stops on other boundary conditions, src/poisson.f90:104-108).
static int need_periodic(x3d_ctx_s *ctx)
{
    return ctx->periodic_all ? X3D_OK
                             : set_error(ctx, X3D_EUNSUPPORTED,
                                         "this routine needs periodic boundaries in every direction");
}

int x3d_poisson(x3d_ctx ctx, double *rhs)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!rhs) return set_error(ctx, X3D_EINVAL, "null field");
    Stager sg(ctx);
    double *d = static_cast<double *>(sg.inout(rhs, ctx->ppts() * sizeof(double)));
    if (sg.status()) return sg.status();
    return sg.finish(ctx->periodic_all ? poisson_solve(ctx, d) : poisson_solve_mirror(ctx, d));
}

int x3d_poisson_zpencil(x3d_ctx ctx, void *spec, int nxh_loc, int i0, int ny_loc, int j0)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = need_periodic(ctx))) return rc;
    if (!spec || !is_device_ptr(spec)) return set_error(ctx, X3D_EINVAL, "spec must be a device array");
    return poisson_zpencil(ctx, spec, nxh_loc, i0, ny_loc, j0);
}

int x3d_poisson_zlines(x3d_ctx ctx, void *spec, int ny_loc, int j0)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    return x3d_poisson_zpencil(ctx, spec, ctx->nx / 2 + 1, 0, ny_loc, j0);
}

// ---- navier ----------------------------------------------------------------------------

// divergence (src/navier.f90:98-236) with 1x1 transposes elided: the fused
// stage kernels, or one launch per operator when no fused kernel fits.
static int divergence_unfused(x3d_ctx_s *ctx, double *pp3, const void *ux, const void *uy, const void *uz);
static int divergence_dev(x3d_ctx_s *ctx, double *pp3, const void *ux, const void *uy, const void *uz)
{
    const TraceRange trace("divergence");
    const void *u[3] = {ux, uy, uz};
    const int rc = fused_divergence(ctx, pp3, u);
    return rc == X3D_EUNSUPPORTED ? divergence_unfused(ctx, pp3, ux, uy, uz) : rc;
}

static int divergence_unfused(x3d_ctx_s *ctx, double *pp3, const void *ux, const void *uy, const void *uz)
{
    const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    const bool f = fp32(ctx);
    const size_t N = ctx->npts();
    void *s[5];
    for (int i = 0; i < 5; ++i)
        if (!(s[i] = ctx_scratch(ctx, i))) return set_error(ctx, X3D_ENOMEM, "scratch allocation failed");
    x3d_op_s **B = ctx->builtin;
    int rc = 0;
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERXVP], DERVP, DX, ux, s[0], nx, ny, nz, f);  // pp1
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTXVP], INTVP, DX, uy, s[1], nx, ny, nz, f);  // pgy1
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTXVP], INTVP, DX, uz, s[2], nx, ny, nz, f);  // pgz1
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTYVP], INTVP, DY, s[0], s[3], nx, ny, nz, f);  // upi2
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERYVP], DERVP, DY, s[1], s[4], nx, ny, nz, f);  // duydypi2
    rc = rc ? rc : launch_add(ctx, f, s[4], s[4], s[3], N);
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTYVP], INTVP, DY, s[2], s[3], nx, ny, nz, f);  // upi2
    if (!f) {
        rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTZVP], INTVP, DZ, s[4], pp3, nx, ny, nz, f);
        rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERZVP], DERVP, DZ, s[3], s[0], nx, ny, nz, f);  // po3
        rc = rc ? rc : launch_add(ctx, false, pp3, pp3, s[0], N);
    } else {
        rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTZVP], INTVP, DZ, s[4], s[0], nx, ny, nz, f);
        rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERZVP], DERVP, DZ, s[3], s[1], nx, ny, nz, f);
        rc = rc ? rc : launch_add(ctx, true, s[0], s[0], s[1], N);
        rc = rc ? rc : launch_convert(ctx, pp3, false, s[0], true, N);
    }
    return rc;
}

// gradp (src/navier.f90:249-359) with 1x1 transposes elided; with ucor set
// the x stage also applies cor_vel (u -= grad p).
static int gradp_unfused(x3d_ctx_s *ctx, void *px, void *py, void *pz, const double *pp3);
static int gradp_dev(x3d_ctx_s *ctx, void *px, void *py, void *pz, const double *pp3,
                     void *const *ucor = nullptr)
{
    const TraceRange trace("gradp + cor_vel");
    void *p[3] = {px, py, pz};
    int rc = fused_gradp(ctx, p, pp3, ucor);
    if (rc != X3D_EUNSUPPORTED) return rc;
    rc = gradp_unfused(ctx, px, py, pz, pp3);
    if (!rc && ucor) rc = launch_sub3(ctx, fp32(ctx), ucor[0], ucor[1], ucor[2], px, py, pz, ctx->npts());
    return rc;
}

static int gradp_unfused(x3d_ctx_s *ctx, void *px, void *py, void *pz, const double *pp3)
{
    const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    const bool f = fp32(ctx);
    const size_t N = ctx->npts();
    void *s[6];
    for (int i = 0; i < 6; ++i)
        if (!(s[i] = ctx_scratch(ctx, i))) return set_error(ctx, X3D_ENOMEM, "scratch allocation failed");
    x3d_op_s **B = ctx->builtin;
    int rc = 0;
    const void *p = pp3;
    if (f) {
        rc = launch_convert(ctx, s[5], true, pp3, false, N);
        p = s[5];
    }
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTZPV], INTPV, DZ, p, s[0], nx, ny, nz, f);     // ppi3
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERZPV], DERPV, DZ, p, s[1], nx, ny, nz, f);     // pgz3
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTYPV], INTPV, DY, s[0], s[2], nx, ny, nz, f);  // ppi2
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERYPV], DERPV, DY, s[0], s[3], nx, ny, nz, f);  // pgy2
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTYPV], INTPV, DY, s[1], s[4], nx, ny, nz, f);  // pgzi2
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERXPV], DERPV, DX, s[2], px, nx, ny, nz, f);
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTXPV], INTPV, DX, s[3], py, nx, ny, nz, f);
    rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_INTXPV], INTPV, DX, s[4], pz, nx, ny, nz, f);
    return rc;
}

// momentum_rhs_eq (src/transeq.f90:44-355) with 1x1 transposes elided; with
// step set, int_time's u = dt du + u is applied too.
static int momentum_unfused(x3d_ctx_s *ctx, void *du[3], const void *u[3]);
static int momentum_dev(x3d_ctx_s *ctx, void *du[3], const void *u[3], bool step = false,
                        double dt = 0.0)
{
    const TraceRange trace("momentum_rhs_eq");
    void *un[3] = {const_cast<void *>(u[0]), const_cast<void *>(u[1]), const_cast<void *>(u[2])};
    int rc = fused_transeq(ctx, du, u, step, dt, un);
    if (rc != X3D_EUNSUPPORTED) return rc;
    rc = momentum_unfused(ctx, du, u);
    if (!rc && step) rc = launch_axpy3(ctx, fp32(ctx), un[0], un[1], un[2], du[0], du[1], du[2], dt, ctx->npts());
    return rc;
}

static int momentum_unfused(x3d_ctx_s *ctx, void *du[3], const void *u[3])
{
    const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    const bool f = fp32(ctx);
    const size_t N = ctx->npts();
    void *s[4];
    for (int i = 0; i < 4; ++i)
        if (!(s[i] = ctx_scratch(ctx, i))) return set_error(ctx, X3D_ENOMEM, "scratch allocation failed");
    x3d_op_s **B = ctx->builtin;
    void *ta = s[0], *td = s[1], *tg = s[2], *t3 = s[3];
    int rc = 0;
    for (int c = 0; c < 3 && !rc; ++c) {
        const void *uc = u[c];
        rc = rc ? rc : launch_mul(ctx, f, ta, u[0], uc, N);
        rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERXP], DER, DX, ta, td, nx, ny, nz, f);
        rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERX], DER, DX, uc, ta, nx, ny, nz, f);
        rc = rc ? rc : launch_fma_acc(ctx, f, du[c], td, u[0], ta, N);
        rc = rc ? rc : launch_mul(ctx, f, td, uc, u[1], N);
        rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERY], DER, DY, td, tg, nx, ny, nz, f);
        rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERYP], DER, DY, uc, td, nx, ny, nz, f);
        rc = rc ? rc : launch_fma_acc(ctx, f, tg, tg, u[1], td, N);
        rc = rc ? rc : launch_mul(ctx, f, td, uc, u[2], N);
        rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERZ], DER, DZ, td, t3, nx, ny, nz, f);
        rc = rc ? rc : launch_linesolve(ctx, B[X3D_OP_DERZP], DER, DZ, uc, td, nx, ny, nz, f);
        rc = rc ? rc : launch_fma_acc(ctx, f, t3, t3, u[2], td, N);
        rc = rc ? rc : launch_add(ctx, f, tg, tg, t3, N);
        rc = rc ? rc : launch_add(ctx, f, du[c], du[c], tg, N);
    }
    return rc;
}

int x3d_divergence(x3d_ctx ctx, double *pp3, const void *ux1, const void *uy1, const void *uz1, int)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = need_periodic(ctx))) return rc;
    if (!pp3 || !ux1 || !uy1 || !uz1) return set_error(ctx, X3D_EINVAL, "null field");
    const size_t b = ctx->npts() * ctx->elem();
    Stager sg(ctx);
    const void *u = sg.in(ux1, b), *v = sg.in(uy1, b), *w = sg.in(uz1, b);
    double *p = static_cast<double *>(sg.out(pp3, ctx->npts() * sizeof(double)));
    if (sg.status()) return sg.status();
    return sg.finish(divergence_dev(ctx, p, u, v, w));
}

int x3d_gradp(x3d_ctx ctx, void *px1, void *py1, void *pz1, const double *pp3)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = need_periodic(ctx))) return rc;
    if (!pp3 || !px1 || !py1 || !pz1) return set_error(ctx, X3D_EINVAL, "null field");
    const size_t b = ctx->npts() * ctx->elem();
    Stager sg(ctx);
    const double *p = static_cast<const double *>(sg.in(pp3, ctx->npts() * sizeof(double)));
    void *x = sg.out(px1, b), *y = sg.out(py1, b), *z = sg.out(pz1, b);
    if (sg.status()) return sg.status();
    return sg.finish(gradp_dev(ctx, x, y, z, p));
}

int x3d_cor_vel(x3d_ctx ctx, void *ux, void *uy, void *uz, const void *px, const void *py, const void *pz)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!ux || !uy || !uz || !px || !py || !pz) return set_error(ctx, X3D_EINVAL, "null field");
    const size_t b = ctx->npts() * ctx->elem();
    Stager sg(ctx);
    void *u = sg.inout(ux, b), *v = sg.inout(uy, b), *w = sg.inout(uz, b);
    const void *a = sg.in(px, b), *bb = sg.in(py, b), *c = sg.in(pz, b);
    if (sg.status()) return sg.status();
    return sg.finish(launch_sub3(ctx, fp32(ctx), u, v, w, a, bb, c, ctx->npts()));
}

int x3d_solve_poisson(x3d_ctx ctx, double *pp3, void *px1, void *py1, void *pz1, const void *ux1,
                      const void *uy1, const void *uz1)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = need_periodic(ctx))) return rc;
    if (!pp3 || !px1 || !py1 || !pz1 || !ux1 || !uy1 || !uz1) return set_error(ctx, X3D_EINVAL, "null field");
    const size_t b = ctx->npts() * ctx->elem();
    Stager sg(ctx);
    const void *u = sg.in(ux1, b), *v = sg.in(uy1, b), *w = sg.in(uz1, b);
    double *p = static_cast<double *>(sg.out(pp3, ctx->npts() * sizeof(double)));
    void *x = sg.out(px1, b), *y = sg.out(py1, b), *z = sg.out(pz1, b);
    if (sg.status()) return sg.status();
    rc = divergence_dev(ctx, p, u, v, w);
    rc = rc ? rc : poisson_solve(ctx, p);
    rc = rc ? rc : gradp_dev(ctx, x, y, z, p);
    return sg.finish(rc);
}

int x3d_div_stats(x3d_ctx ctx, const double *pp3, double *out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!pp3 || !out) return set_error(ctx, X3D_EINVAL, "null argument");
    Stager sg(ctx);
    const double *p = static_cast<const double *>(sg.in(pp3, ctx->npts() * sizeof(double)));
    if (sg.status()) return sg.status();
    return sg.finish(reduce_absmax_mean(ctx, p, ctx->npts(), out));
}

// ---- transeq / time integration --------------------------------------------------------

// ---- the step's parts on one pencil ------------------------------------------------------

// A pencil of the context's box along dir: whole lines along dir, at least
// one line, and every listed field a device array.
static int check_part(x3d_ctx_s *ctx, int dir, int nx, int ny, int nz, std::initializer_list<const void *> fields)
{
    int rc = need_periodic(ctx);
    if (rc) return rc;
    if (dir < 0 || dir > 2) return set_error(ctx, X3D_EINVAL, "dir must be 0, 1 or 2");
    const int ext[3] = {nx, ny, nz}, box[3] = {ctx->nx, ctx->ny, ctx->nz};
    for (int d = 0; d < 3; ++d)
        if (ext[d] < 1 || ext[d] > box[d]) return set_error(ctx, X3D_EINVAL, "pencil extents outside the box");
    if (ext[dir] != box[dir]) return set_error(ctx, X3D_EINVAL, "a pencil holds whole lines along its direction");
    for (const void *f : fields)
        if (!f || !is_device_ptr(f)) return set_error(ctx, X3D_EINVAL, "pencil parts take device arrays");
    return X3D_OK;
}

int x3d_transeq_part(x3d_ctx ctx, int dir, void *const *du, const void *const *u, const void *const *add,
                     void *const *unew, double dt, int nx, int ny, int nz)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!du || !u) return set_error(ctx, X3D_EINVAL, "null field list");
    if ((rc = check_part(ctx, dir, nx, ny, nz, {du[0], du[1], du[2], u[0], u[1], u[2]}))) return rc;
    if (add && (rc = check_part(ctx, dir, nx, ny, nz, {add[0], add[1], add[2]}))) return rc;
    if (unew && (rc = check_part(ctx, dir, nx, ny, nz, {unew[0], unew[1], unew[2]}))) return rc;
    const TraceRange trace("momentum_rhs_eq part");
    return part_transeq(ctx, dir, du, u, add, unew, dt, nx, ny, nz);
}

int x3d_divergence_part(x3d_ctx ctx, int dir, void *const *out, const void *const *in, int nx, int ny, int nz)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || !in) return set_error(ctx, X3D_EINVAL, "null field list");
    if (dir == 0) rc = check_part(ctx, dir, nx, ny, nz, {out[0], out[1], out[2], in[0], in[1], in[2]});
    else if (dir == 1) rc = check_part(ctx, dir, nx, ny, nz, {out[0], out[1], in[0], in[1], in[2]});
    else rc = check_part(ctx, dir, nx, ny, nz, {out[0], in[0], in[1]});
    if (rc) return rc;
    const TraceRange trace("divergence part");
    return part_divergence(ctx, dir, out, in, nx, ny, nz);
}

int x3d_gradp_part(x3d_ctx ctx, int dir, void *const *out, const void *const *in, void *const *ucor, int nx,
                   int ny, int nz)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || !in) return set_error(ctx, X3D_EINVAL, "null field list");
    if (dir == 2) rc = check_part(ctx, dir, nx, ny, nz, {out[0], out[1], in[0]});
    else if (dir == 1) rc = check_part(ctx, dir, nx, ny, nz, {out[0], out[1], out[2], in[0], in[1]});
    else rc = check_part(ctx, dir, nx, ny, nz, {out[0], out[1], out[2], in[0], in[1], in[2]});
    if (!rc && ucor && dir == 0) rc = check_part(ctx, dir, nx, ny, nz, {ucor[0], ucor[1], ucor[2]});
    if (rc) return rc;
    const TraceRange trace("gradp part");
    return part_gradp(ctx, dir, out, in, dir == 0 ? ucor : nullptr, nx, ny, nz);
}

int x3d_momentum_rhs_eq(x3d_ctx ctx, void *dux1, void *duy1, void *duz1, const void *ux1,
                        const void *uy1, const void *uz1)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = need_periodic(ctx))) return rc;
    if (!dux1 || !duy1 || !duz1 || !ux1 || !uy1 || !uz1) return set_error(ctx, X3D_EINVAL, "null field");
    const size_t b = ctx->npts() * ctx->elem();
    Stager sg(ctx);
    const void *u[3] = {sg.in(ux1, b), sg.in(uy1, b), sg.in(uz1, b)};
    void *du[3] = {sg.out(dux1, b), sg.out(duy1, b), sg.out(duz1, b)};
    if (sg.status()) return sg.status();
    return sg.finish(momentum_dev(ctx, du, u));
}

int x3d_int_time(x3d_ctx ctx, void *ux1, void *uy1, void *uz1, const void *dux1, const void *duy1,
                 const void *duz1, double gdt)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!dux1 || !duy1 || !duz1 || !ux1 || !uy1 || !uz1) return set_error(ctx, X3D_EINVAL, "null field");
    const size_t b = ctx->npts() * ctx->elem();
    Stager sg(ctx);
    void *u = sg.inout(ux1, b), *v = sg.inout(uy1, b), *w = sg.inout(uz1, b);
    const void *a = sg.in(dux1, b), *bb = sg.in(duy1, b), *c = sg.in(duz1, b);
    if (sg.status()) return sg.status();
    return sg.finish(launch_axpy3(ctx, fp32(ctx), u, v, w, a, bb, c, gdt, ctx->npts()));
}

// One timestep on device fields (src/xcompact3d.f90:80-95).
static int euler_dev(x3d_ctx_s *ctx, void *u[3], void *du[3], double *p, void *px, void *py, void *pz, double dt)
{
    const TraceRange trace("euler_step");
    const void *uc[3] = {u[0], u[1], u[2]};
    int rc = momentum_dev(ctx, du, uc, true, dt);             // calculate_transeq_rhs + int_time
    rc = rc ? rc : divergence_dev(ctx, p, u[0], u[1], u[2]);  // solve_poisson: divergence
    rc = rc ? rc : poisson_solve(ctx, p);                     //                poisson
    rc = rc ? rc : gradp_dev(ctx, px, py, pz, p, u);          //                gradp + cor_vel
    return rc;
}

int x3d_euler_step(x3d_ctx ctx, void *ux1, void *uy1, void *uz1, void *dux1, void *duy1, void *duz1,
                   double *pp3, void *px1, void *py1, void *pz1, double dt)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = need_periodic(ctx))) return rc;
    if (!ux1 || !uy1 || !uz1 || !dux1 || !duy1 || !duz1 || !pp3 || !px1 || !py1 || !pz1)
        return set_error(ctx, X3D_EINVAL, "null field");
    const size_t b = ctx->npts() * ctx->elem();
    Stager sg(ctx);
    void *u[3] = {sg.inout(ux1, b), sg.inout(uy1, b), sg.inout(uz1, b)};
    void *du[3] = {sg.out(dux1, b), sg.out(duy1, b), sg.out(duz1, b)};
    double *p = static_cast<double *>(sg.out(pp3, ctx->npts() * sizeof(double)));
    void *px = sg.out(px1, b), *py = sg.out(py1, b), *pz = sg.out(pz1, b);
    if (sg.status()) return sg.status();
    return sg.finish(euler_dev(ctx, u, du, p, px, py, pz, dt));
}

int x3d_step_capture(x3d_ctx ctx, void *ux1, void *uy1, void *uz1, void *dux1, void *duy1, void *duz1,
                     double *pp3, void *px1, void *py1, void *pz1, double dt)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = need_periodic(ctx))) return rc;
    if (!ctx->stream || ctx->stream == cudaStreamLegacy || ctx->stream == cudaStreamPerThread)
        return set_error(ctx, X3D_EUNSUPPORTED, "capture needs the context on a created stream");
    const size_t b = ctx->npts() * ctx->elem();
    void *const user[10] = {ux1, uy1, uz1, dux1, duy1, duz1, pp3, px1, py1, pz1};
    void *dev[10];
    for (int i = 0; i < 10; ++i) {
        const size_t bytes = i == 6 ? ctx->npts() * sizeof(double) : b;
        if (!user[i]) return set_error(ctx, X3D_EINVAL, "null field");
        dev[i] = resident_dev(ctx, user[i], bytes);
        if (!dev[i] && is_device_ptr(user[i])) dev[i] = user[i];
        if (!dev[i]) return set_error(ctx, X3D_EINVAL, "capture needs device or registered fields");
    }
    // everything the step allocates on first use, before the capture
    if (!ctx_scratch(ctx, 5)) return set_error(ctx, X3D_ENOMEM, "scratch allocation failed");
    if ((rc = poisson_setup(ctx))) return rc;
    if ((rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "capture"))) return rc;
    if (ctx->step_exec) cudaGraphExecDestroy(ctx->step_exec);
    if (ctx->step_graph) cudaGraphDestroy(ctx->step_graph);
    ctx->step_exec = nullptr;
    ctx->step_graph = nullptr;
    rc = cuda_check(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    if (rc) return rc;
    void *u[3] = {dev[0], dev[1], dev[2]}, *du[3] = {dev[3], dev[4], dev[5]};
    const int work = euler_dev(ctx, u, du, static_cast<double *>(dev[6]), dev[7], dev[8], dev[9], dt);
    cudaGraph_t g = nullptr;
    rc = cuda_check(ctx, cudaStreamEndCapture(ctx->stream, &g), "end capture");
    if (work || rc) {
        if (g) cudaGraphDestroy(g);
        return work ? work : rc;
    }
    cudaGraphExec_t e = nullptr;
    if ((rc = cuda_check(ctx, cudaGraphInstantiate(&e, g, 0), "graph instantiate"))) {
        cudaGraphDestroy(g);
        return rc;
    }
    ctx->step_graph = g;
    ctx->step_exec = e;
    return X3D_OK;
}

int x3d_step_launch(x3d_ctx ctx)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!ctx->step_exec) return set_error(ctx, X3D_EINVAL, "no captured step");
    return cuda_check(ctx, cudaGraphLaunch(ctx->step_exec, ctx->stream), "graph launch");
}

// ---- device-resident mirrors ------------------------------------------------------------

int x3d_buf_register(x3d_ctx ctx, void *host, size_t nbytes, void **dev)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!host || !nbytes) return set_error(ctx, X3D_EINVAL, "null or empty host array");
    if (is_device_ptr(host)) return set_error(ctx, X3D_EINVAL, "already a device pointer");
    const char *h = static_cast<const char *>(host);
    for (const auto &r : ctx->resident) {
        const char *o = static_cast<const char *>(r.host);
        if (h < o + r.bytes && o < h + nbytes) return set_error(ctx, X3D_EINVAL, "overlaps a registered array");
    }
    void *d = nullptr;
    if (cudaMalloc(&d, nbytes) != cudaSuccess) return set_error(ctx, X3D_ENOMEM, "mirror allocation failed");
    rc = cuda_check(ctx, cudaMemcpyAsync(d, host, nbytes, cudaMemcpyHostToDevice, ctx->stream), "mirror upload");
    if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "mirror upload");
    if (rc) {
        cudaFree(d);
        return rc;
    }
    ctx->resident.push_back({host, d, nbytes});
    if (dev) *dev = d;
    return X3D_OK;
}

static x3d_ctx_s::Resident *find_resident(x3d_ctx_s *ctx, const void *host)
{
    for (auto &r : ctx->resident)
        if (r.host == host) return &r;
    return nullptr;
}

int x3d_buf_unregister(x3d_ctx ctx, void *host)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    for (size_t i = 0; i < ctx->resident.size(); ++i)
        if (ctx->resident[i].host == host) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(ctx->resident[i].dev);
            ctx->resident.erase(ctx->resident.begin() + i);
            return X3D_OK;
        }
    return set_error(ctx, X3D_EINVAL, "not a registered array");
}

int x3d_sync_to_device(x3d_ctx ctx, void *host)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    auto *r = find_resident(ctx, host);
    if (!r) return set_error(ctx, X3D_EINVAL, "not a registered array");
    rc = cuda_check(ctx, cudaMemcpyAsync(r->dev, r->host, r->bytes, cudaMemcpyHostToDevice, ctx->stream),
                    "sync to device");
    return rc ? rc : cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync to device");
}

int x3d_sync_to_host(x3d_ctx ctx, void *host)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    auto *r = find_resident(ctx, host);
    if (!r) return set_error(ctx, X3D_EINVAL, "not a registered array");
    rc = cuda_check(ctx, cudaMemcpyAsync(r->host, r->dev, r->bytes, cudaMemcpyDeviceToHost, ctx->stream),
                    "sync to host");
    return rc ? rc : cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync to host");
}

// ---- mom ----------------------------------------------------------------------------------

int x3d_vel(x3d_ctx ctx, void *u, void *v, void *w)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!u || !v || !w) return set_error(ctx, X3D_EINVAL, "null field");
    const size_t b = ctx->npts() * ctx->elem();
    Stager sg(ctx);
    void *a = sg.out(u, b), *bb = sg.out(v, b), *c = sg.out(w, b);
    if (sg.status()) return sg.status();
    return sg.finish(launch_vel(ctx, fp32(ctx), a, bb, c));
}

int x3d_test_rms(x3d_ctx ctx, int which, const void *du, double *rms)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!du || !rms || which < 0 || which > 2) return set_error(ctx, X3D_EINVAL, "bad argument");
    Stager sg(ctx);
    const void *d = sg.in(du, ctx->npts() * ctx->elem());
    if (sg.status()) return sg.status();
    return sg.finish(reduce_test_rms(ctx, fp32(ctx), which, d, rms));
}

}  // extern "C"
