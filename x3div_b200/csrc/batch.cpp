// Batches of independent periodic boxes of uneven sizes: the derivative
// sweep of every box in one persistent launch (BatchJob work-list, see
// linesolve_chunk.cu), capturable as a CUDA graph.  Boxes of one shape share
// a context, hence its FP64 operator precompute.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "linesolve_chunk.h"
#include "x3d_internal.h"

using namespace x3d;

struct x3d_batch_s {
    int precision = X3D_F32;
    int device = 0;
    int num_sms = 148;
    size_t smem_optin = 0;
    std::vector<x3d_box> boxes;
    std::vector<x3d_ctx> shape_ctx;  // owned, one per distinct (dims, lengths)
    std::vector<int> box_shape;      // box -> shape_ctx index
    cudaStream_t own_stream = nullptr, stream = nullptr;
    unsigned long long *d_counter = nullptr;
    int *d_err = nullptr;
    void *d_jobs = nullptr;
    size_t jobs_cap = 0;
    int njobs = 0;
    long total_tiles = 0;
    size_t tile_cap = 0;
    int variant = 0;  // the batch kernel's variant the job list needs (BatchVariant)
    int grid = 0;
    // jobs the persistent kernel cannot take run as per-box grouped launches
    struct Fallback {
        int box, dir;
        const void *in;
        const x3d_op_s *ops[6];
        int kinds[6];
        void *outs[6];
        int nops;
    };
    std::vector<Fallback> fallback;
    long long points = 0;  // operator-application points per run
    // the bound sweep (x3d_batch_bind_sweep), kept for x3d_batch_autotune
    int nfields = 0, nops = 0;
    std::vector<void *> fields, outs;
    // per (box shape, direction): chunk length (0: the long one) and the
    // most lines per tile (0: as many as the threads allow), set by
    // x3d_batch_autotune; and the lines per tile each shape's jobs got
    std::vector<int> choice_L, choice_W, choice_X, planned_W;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    std::string last_error;
};

namespace {

int bfail(x3d_batch_s *b, int code, const std::string &msg)
{
    if (b) b->last_error = msg;
    return code;
}

template <typename T>
const LineOp<T> &lop(const x3d_op_s *op);
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

// The work-list of the bound sweep: every (box, field, direction) job, or
// only those of box shape `shape` and direction `dir` (>= 0), each planned
// with its shape and direction's choice of chunk length and tile width, or
// with (L, w_req) where L > 0.  Jobs the kernel cannot take go to the
// fallback list (for the whole work-list only).
template <typename T>
int make_jobs(x3d_batch_s *b, std::vector<BatchJob<T>> &jobs, size_t *tile_cap_out, long *tiles_out,
              int shape, int dir, int L_force, int w_force, int x_force = 0)
{
    const int nfields = b->nfields, nops_per_dir = b->nops;
    void *const *fields = b->fields.data();
    void *const *outs = b->outs.data();
    const bool whole = shape < 0;
    if (whole) {
        b->fallback.clear();
        b->points = 0;
    }
    size_t tile_cap = 0;
    long tiles = 0;
    const int kinds[6] = {DER, DER2, DERVP, DERPV, INTVP, INTPV};
    for (size_t i = 0; i < b->boxes.size(); ++i) {
        if (!whole && b->box_shape[i] != shape) continue;
        x3d_ctx_s *ctx = b->shape_ctx[b->box_shape[i]];
        const int dims[3] = {ctx->nx, ctx->ny, ctx->nz};
        for (int f = 0; f < nfields; ++f) {
            const void *in = fields[i * nfields + f];
            for (int d = 0; d < 3; ++d) {
                if (!whole && d != dir) continue;
                BatchJob<T> J;
                std::memset(&J, 0, sizeof(J));
                J.in = static_cast<const T *>(in);
                J.nops = nops_per_dir;
                J.dir = d;
                J.n = dims[d];
                J.nx = dims[0];
                J.ny = dims[1];
                J.nz = dims[2];
                typename x3d_batch_s::Fallback fb{};
                fb.box = (int)i;
                fb.dir = d;
                fb.in = in;
                fb.nops = nops_per_dir;
                for (int k = 0; k < nops_per_dir; ++k) {
                    const x3d_op_s *op = nullptr;
                    for (int w = 0; w < X3D_OP_COUNT; ++w)
                        if (ctx->builtin[w]->h.kind == kinds[k] && ctx->builtin[w]->h.dir == d) {
                            op = ctx->builtin[w];
                            break;
                        }
                    J.op[k] = lop<T>(op);
                    J.kind[k] = kinds[k];
                    J.out[k] = static_cast<T *>(outs[((i * nfields + f) * 3 + d) * 6 + k]);
                    fb.ops[k] = op;
                    fb.kinds[k] = kinds[k];
                    fb.outs[k] = J.out[k];
                }
                if (whole) b->points += (long long)nops_per_dir * dims[0] * dims[1] * dims[2];
                const int sd = b->box_shape[i] * 3 + d;
                const int L = L_force > 0 ? L_force : (b->choice_L[sd] > 0 ? b->choice_L[sd] : kChunkLong<T>);
                const int w = L_force > 0 ? w_force : b->choice_W[sd];
                const int xs = L_force > 0 ? x_force : b->choice_X[sd];
                size_t tb = 0;
                if (plan_batch_job<T>(J, L, w, xs, &tb)) {
                    // one box shape's operators along d at one chunk length
                    J.rclass = sd * 2 + (J.L == kChunkLong<T> ? 0 : 1);
                    J.tile0 = tiles;
                    tiles += J.ntiles;
                    tile_cap = std::max(tile_cap, tb);
                    jobs.push_back(J);
                    if (whole) b->planned_W[sd] = J.W;
                } else if (whole) {
                    b->fallback.push_back(fb);
                }
            }
        }
    }
    *tile_cap_out = tile_cap;
    *tiles_out = tiles;
    return X3D_OK;
}

template <typename T>
int bind_typed(x3d_batch_s *b)
{
    std::vector<BatchJob<T>> jobs;
    size_t tile_cap = 0;
    long tiles = 0;
    make_jobs<T>(b, jobs, &tile_cap, &tiles, -1, -1, 0, 0);
    b->njobs = (int)jobs.size();
    b->total_tiles = tiles;
    b->tile_cap = tile_cap;
    b->variant = batch_variant<T>(jobs.data(), (int)jobs.size());
    if (!jobs.empty()) {
        const size_t bytes = jobs.size() * sizeof(BatchJob<T>);
        if (bytes > b->jobs_cap) {
            if (b->d_jobs) cudaFree(b->d_jobs);
            b->d_jobs = nullptr;
            b->jobs_cap = 0;
            if (cudaMalloc(&b->d_jobs, bytes) != cudaSuccess) return bfail(b, X3D_ENOMEM, "job list allocation failed");
            b->jobs_cap = bytes;
        }
        if (cudaMemcpy(b->d_jobs, jobs.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess)
            return bfail(b, X3D_ECUDA, "job list upload failed");
        const int rc = prepare_batch<T>(tile_cap, b->variant, b->smem_optin, b->num_sms, &b->grid);
        if (rc) {
            b->njobs = 0;
            b->total_tiles = 0;
            return bfail(b, rc, "batch kernel cannot fit its tiles in shared memory");
        }
    }
    return X3D_OK;
}

template <typename T>
int run_typed(x3d_batch_s *b)
{
    if (b->njobs > 0) {
        const int rc = launch_batch<T>(b->stream, b->grid, static_cast<const BatchJob<T> *>(b->d_jobs), b->njobs,
                                       b->total_tiles, b->d_counter, b->tile_cap, b->variant, b->d_err);
        if (rc) return bfail(b, rc, std::string("batch launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    }
    for (auto &fb : b->fallback) {
        x3d_ctx_s *ctx = b->shape_ctx[b->box_shape[fb.box]];
        cudaStream_t keep = ctx->stream;
        ctx->stream = b->stream;
        const int rc = launch_group(ctx, fb.dir, fb.in, fb.ops, fb.kinds, fb.outs, fb.nops, ctx->nx, ctx->ny,
                                    ctx->nz, b->precision == X3D_F32);
        ctx->stream = keep;
        if (rc) return bfail(b, rc, ctx->last_error);
    }
    return X3D_OK;
}

void drop_graph(x3d_batch_s *b)
{
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
}

}  // namespace

namespace {

// Times the batch kernel on the jobs of one box shape and direction with
// each candidate and keeps the fastest: the long and the short chunk, each
// with as many lines per tile as the threads allow and with half as many,
// and for x jobs each with outputs straight out and staged in shared memory.
template <typename T>
int autotune_typed(x3d_batch_s *b)
{
    const int nshapes = (int)b->shape_ctx.size();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    void *d_tmp = nullptr;
    size_t tmp_cap = 0;
    int rc = X3D_OK;
    for (int sh = 0; sh < nshapes && !rc; ++sh)
        for (int d = 0; d < 3 && !rc; ++d) {
            float best = -1.f;
            int bestL = 0, bestW = 0, bestX = 0;
            const int Ls[2] = {kChunkLong<T>, kChunkShort<T>};
            for (int cand = 0; cand < (d == 0 ? 8 : 4) && !rc; ++cand) {
                    const int li = cand & 1, half = (cand >> 1) & 1, xs = cand >> 2;
                    std::vector<BatchJob<T>> jobs;
                    size_t cap = 0;
                    long tiles = 0;
                    // the widest tile first, to learn the width to halve
                    int w = 0;
                    if (half) {
                        std::vector<BatchJob<T>> probe;
                        make_jobs<T>(b, probe, &cap, &tiles, sh, d, Ls[li], 0);
                        if (probe.empty()) continue;
                        w = probe[0].W / 2;
                        if (w < (int)(16 / sizeof(T))) continue;
                    }
                    make_jobs<T>(b, jobs, &cap, &tiles, sh, d, Ls[li], w, xs);
                    if (jobs.empty()) continue;
                    const size_t bytes = jobs.size() * sizeof(BatchJob<T>);
                    if (bytes > tmp_cap) {
                        if (d_tmp) cudaFree(d_tmp);
                        d_tmp = nullptr;
                        if (cudaMalloc(&d_tmp, bytes) != cudaSuccess) {
                            rc = bfail(b, X3D_ENOMEM, "autotune job list allocation failed");
                            break;
                        }
                        tmp_cap = bytes;
                    }
                    if (cudaMemcpy(d_tmp, jobs.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
                        rc = bfail(b, X3D_ECUDA, "autotune job list upload failed");
                        break;
                    }
                    int grid = 0;
                    const int var = batch_variant<T>(jobs.data(), (int)jobs.size());
                    if (prepare_batch<T>(cap, var, b->smem_optin, b->num_sms, &grid)) continue;
                    auto run = [&]() {
                        return launch_batch<T>(b->stream, grid, static_cast<const BatchJob<T> *>(d_tmp),
                                               (int)jobs.size(), tiles, b->d_counter, cap, var, b->d_err);
                    };
                    if ((rc = run())) break;
                    float ms = 0.f;
                    for (int r = 0; r < 3 && !rc; ++r) {
                        cudaEventRecord(e0, b->stream);
                        rc = run();
                        cudaEventRecord(e1, b->stream);
                        cudaEventSynchronize(e1);
                        float m = 0.f;
                        cudaEventElapsedTime(&m, e0, e1);
                        ms = r == 0 ? m : std::min(ms, m);
                    }
                    if (!rc && (best < 0.f || ms < best)) {
                        best = ms;
                        bestL = Ls[li];
                        bestW = w;
                        bestX = xs;
                    }
                }
            if (best >= 0.f) {
                b->choice_L[sh * 3 + d] = bestL;
                b->choice_W[sh * 3 + d] = bestW;
                b->choice_X[sh * 3 + d] = bestX;
            }
        }
    if (d_tmp) {
        cudaStreamSynchronize(b->stream);
        cudaFree(d_tmp);
    }
    // Each shape was timed alone; in the whole launch the largest tile (and
    // the staging rows, if any job stages) sizes every CTA, so fewer may fit
    // an SM than in a shape's trial, and a job list with any short chunk or
    // staged x job needs a wider kernel variant.  The whole work-list is
    // timed with the choices; with them but no x staging; with the chosen
    // lines per tile of the long-chunk choices only (the narrowest variant);
    // and with the defaults.  The fastest of the four is kept.
    auto time_whole = [&](float *ms) {
        int r = bind_typed<T>(b);
        if (r) return r;
        if ((r = run_typed<T>(b))) return r;
        for (int k = 0; k < 3 && !r; ++k) {
            cudaEventRecord(e0, b->stream);
            r = run_typed<T>(b);
            cudaEventRecord(e1, b->stream);
            cudaEventSynchronize(e1);
            float m = 0.f;
            cudaEventElapsedTime(&m, e0, e1);
            *ms = k == 0 ? m : std::min(*ms, m);
        }
        return r;
    };
    if (!rc) {
        struct Set {
            std::vector<int> L, W, X;
        };
        const size_t ns = b->choice_L.size();
        const std::vector<int> zero(ns, 0);
        const Set tuned{b->choice_L, b->choice_W, b->choice_X};
        Set long_only{zero, zero, zero};
        for (size_t i = 0; i < ns; ++i)
            if (tuned.L[i] == kChunkLong<T>) long_only.W[i] = tuned.W[i];
        const Set sets[4] = {tuned, {tuned.L, tuned.W, zero}, long_only, {zero, zero, zero}};
        float best = -1.f;
        int pick = 0;
        for (int k = 0; k < 4 && !rc; ++k) {
            b->choice_L = sets[k].L;
            b->choice_W = sets[k].W;
            b->choice_X = sets[k].X;
            float ms = 0.f;
            rc = time_whole(&ms);
            if (!rc && (best < 0.f || ms < best)) {
                best = ms;
                pick = k;
            }
        }
        b->choice_L = sets[pick].L;
        b->choice_W = sets[pick].W;
        b->choice_X = sets[pick].X;
        if (!rc) rc = bind_typed<T>(b);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

}  // namespace

extern "C" {

int x3d_batch_create(x3d_batch *out, const x3d_box *boxes, int nboxes, int precision, int device)
{
    if (!out || !boxes || nboxes < 1) return X3D_EINVAL;
    *out = nullptr;
    if (precision != X3D_F32 && precision != X3D_F64) return X3D_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return X3D_ECUDA;
    auto *b = new (std::nothrow) x3d_batch_s;
    if (!b) return X3D_ENOMEM;
    b->precision = precision;
    b->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete b;
        return X3D_ECUDA;
    }
    b->num_sms = prop.multiProcessorCount;
    b->smem_optin = prop.sharedMemPerBlockOptin;
    std::map<std::tuple<int, int, int, double, double, double>, int> shapes;
    for (int i = 0; i < nboxes; ++i) {
        const x3d_box &bx = boxes[i];
        const auto key = std::make_tuple(bx.nx, bx.ny, bx.nz, bx.xlx, bx.yly, bx.zlz);
        auto it = shapes.find(key);
        if (it == shapes.end()) {
            x3d_ctx c = nullptr;
            const int rc = x3d_ctx_create(&c, bx.nx, bx.ny, bx.nz, bx.xlx, bx.yly, bx.zlz, precision, device);
            if (rc) {
                x3d_batch_destroy(b);
                return rc;
            }
            it = shapes.emplace(key, (int)b->shape_ctx.size()).first;
            b->shape_ctx.push_back(c);
        }
        b->boxes.push_back(bx);
        b->box_shape.push_back(it->second);
    }
    b->choice_L.assign(b->shape_ctx.size() * 3, 0);
    b->choice_W.assign(b->shape_ctx.size() * 3, 0);
    b->choice_X.assign(b->shape_ctx.size() * 3, 0);
    b->planned_W.assign(b->shape_ctx.size() * 3, 0);
    if (cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&b->d_counter, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&b->d_err, sizeof(int)) != cudaSuccess) {
        x3d_batch_destroy(b);
        return X3D_ECUDA;
    }
    cudaMemset(b->d_err, 0, sizeof(int));
    b->stream = b->own_stream;
    *out = b;
    return X3D_OK;
}

int x3d_batch_destroy(x3d_batch b)
{
    if (!b) return X3D_EINVAL;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (x3d_ctx c : b->shape_ctx) x3d_ctx_destroy(c);
    if (b->d_jobs) cudaFree(b->d_jobs);
    if (b->d_counter) cudaFree(b->d_counter);
    if (b->d_err) cudaFree(b->d_err);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    delete b;
    return X3D_OK;
}

int x3d_batch_set_stream(x3d_batch b, void *stream)
{
    if (!b) return X3D_EINVAL;
    b->stream = static_cast<cudaStream_t>(stream);
    drop_graph(b);
    return X3D_OK;
}

const char *x3d_batch_last_error(x3d_batch b) { return b ? b->last_error.c_str() : "null batch"; }

int x3d_batch_bind_sweep(x3d_batch b, int nfields, void *const *fields, void *const *outs, int nops)
{
    if (!b || nfields < 1 || !fields || !outs || nops < 1 || nops > 6) return X3D_EINVAL;
    cudaSetDevice(b->device);
    const size_t nin = b->boxes.size() * (size_t)nfields;
    for (size_t i = 0; i < nin; ++i)
        if (!fields[i]) return bfail(b, X3D_EINVAL, "null input field");
    for (size_t i = 0; i < nin * 18; ++i)
        if ((int)(i % 6) < nops && !outs[i]) return bfail(b, X3D_EINVAL, "null output field");
    drop_graph(b);
    b->nfields = nfields;
    b->nops = nops;
    b->fields.assign(fields, fields + nin);
    b->outs.assign(outs, outs + nin * 18);
    return b->precision == X3D_F32 ? bind_typed<float>(b) : bind_typed<double>(b);
}


int x3d_batch_autotune(x3d_batch b)
{
    if (!b) return X3D_EINVAL;
    if (b->nfields < 1) return bfail(b, X3D_EINVAL, "bind a sweep before tuning it");
    cudaSetDevice(b->device);
    if (cudaStreamCaptureStatus st; cudaStreamIsCapturing(b->stream, &st) == cudaSuccess &&
                                    st != cudaStreamCaptureStatusNone)
        return bfail(b, X3D_EINVAL, "cannot autotune during stream capture");
    drop_graph(b);
    const int rc = b->precision == X3D_F32 ? autotune_typed<float>(b) : autotune_typed<double>(b);
    if (rc) return rc;
    return x3d_batch_sync(b);
}

int x3d_batch_choice(x3d_batch b, int box, int dir, int *chunk, int *lines)
{
    if (!b || box < 0 || box >= (int)b->boxes.size() || dir < 0 || dir > 2) return X3D_EINVAL;
    const int sd = b->box_shape[box] * 3 + dir;
    const bool f32 = b->precision == X3D_F32;
    if (chunk) *chunk = b->choice_L[sd] > 0 ? b->choice_L[sd] : (f32 ? kChunkLong<float> : kChunkLong<double>);
    if (lines) *lines = b->planned_W[sd];
    return X3D_OK;
}

int x3d_batch_run(x3d_batch b)
{
    const TraceRange trace("batch_run");
    if (!b) return X3D_EINVAL;
    cudaSetDevice(b->device);
    return b->precision == X3D_F32 ? run_typed<float>(b) : run_typed<double>(b);
}

int x3d_batch_capture(x3d_batch b)
{
    if (!b) return X3D_EINVAL;
    cudaSetDevice(b->device);
    drop_graph(b);
    // Capture on the batch's own stream (the legacy default stream cannot be
    // captured); x3d_batch_replay launches the graph on the batch's stream.
    cudaStream_t user = b->stream;
    if (cudaStreamSynchronize(user) != cudaSuccess) return bfail(b, X3D_ECUDA, "stream sync failed");
    b->stream = b->own_stream;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        b->stream = user;
        return bfail(b, X3D_ECUDA, "stream capture could not start");
    }
    const int rc = x3d_batch_run(b);
    const cudaError_t e = cudaStreamEndCapture(b->stream, &b->graph);
    b->stream = user;
    if (rc) return rc;
    if (e != cudaSuccess) return bfail(b, X3D_ECUDA, "stream capture failed");
    if (cudaGraphInstantiate(&b->gexec, b->graph, 0) != cudaSuccess) {
        drop_graph(b);
        return bfail(b, X3D_ECUDA, "graph instantiation failed");
    }
    return X3D_OK;
}

int x3d_batch_replay(x3d_batch b)
{
    if (!b) return X3D_EINVAL;
    if (!b->gexec) return bfail(b, X3D_EINVAL, "no captured graph");
    cudaSetDevice(b->device);
    return cudaGraphLaunch(b->gexec, b->stream) == cudaSuccess ? X3D_OK : bfail(b, X3D_ECUDA, "graph launch failed");
}

int x3d_batch_sync(x3d_batch b)
{
    if (!b) return X3D_EINVAL;
    cudaSetDevice(b->device);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bfail(b, X3D_ECUDA, "batch stream sync failed");
    int flag = 0;
    if (cudaMemcpy(&flag, b->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return bfail(b, X3D_ECUDA, "batch error flag read failed");
    if (flag) {
        cudaMemset(b->d_err, 0, sizeof(int));
        return bfail(b, X3D_ETIMEOUT, "a device-side bounded wait gave up");
    }
    return X3D_OK;
}

int x3d_batch_info(x3d_batch b, long long *points, long long *tiles, int *jobs, int *fallback_jobs)
{
    if (!b) return X3D_EINVAL;
    if (points) *points = b->points;
    if (tiles) *tiles = b->total_tiles;
    if (jobs) *jobs = b->njobs;
    if (fallback_jobs) *fallback_jobs = (int)b->fallback.size();
    return X3D_OK;
}

}  // extern "C"
