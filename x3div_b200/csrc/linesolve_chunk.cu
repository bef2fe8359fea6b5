// Chunked periodic line solves: the fast path for whole-field operator
// applications, and the multi-operator variant that applies up to six
// operators to one staged input (one read of the field, K writes).
//
// The reference sweeps each line serially (?thomas_12, src/thomas.f90:61-84):
//   forward  z_i = r_i - s_i z_{i-1}          backward y_i = (z_i - f_i y_{i+1}) w_i
// then corrects for periodicity with the precomputed vector p
// (xthomas_0 :49-55):  x = y - p (y_1 - alfa y_n) / (1 + p_1 - alfa p_n).
//
// Here a line of n points is cut into C chunks of L points; thread (l, c)
// owns chunk c of line l and keeps it in registers.  Each recurrence is
// affine in its incoming value, so a chunk is swept locally from zero and
// later shifted by  multiplier * carry, where the multiplier is the running
// product of the reference's own factors (-s_i forward, -f_i w_i backward):
//   1. stencil r_i for the chunk (window of L+8 input values, read once for
//      all K operators);
//   2. local forward sweep -> chunk end value and multiplier, plus the chunk's
//      share of y_0 = sum_i g_i r_i (g = first row of M^-1, FP64);
//   -- barrier -- every thread scans the chunk ends (C fused multiply-adds)
//      for its carry and for z_{n-1}, so ss = (y_0 - alfa z_{n-1} w_{n-1})
//      / (1 + p_0 - alfa p_{n-1}) is known before the backward sweep;
//   3. fix the forward values, local backward sweep -> chunk start value and
//      multiplier;
//   -- barrier -- scan for the backward carry;
//   4. fix the backward values, subtract ss p_i, store.
// Two barriers per operator, no intermediate field in shared memory, and the
// same arithmetic as the reference Thomas + Sherman-Morrison up to rounding.
//
// Staging: y/z tiles of W x-adjacent lines arrive by TMA tensor loads and
// results go straight to global memory, coalesced across the W lines; x
// tiles arrive as W padded rows by 1-D bulk copies and results leave as
// 16-byte vector stores of each thread's contiguous chunk.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "ptx.cuh"
#include "x3d_internal.h"
#include "linesolve_chunk.h"

namespace x3d {

constexpr uint64_t kChunkWaitNs = 2000000000ull;

template <int KIND, typename T>
__device__ __forceinline__ T stencil_at(const T *v, const LineOp<T> &op)
{
    // v[k] = u_{i-4+k}
    if constexpr (KIND == DER) return op.a * (v[5] - v[3]) + op.b * (v[6] - v[2]);
    if constexpr (KIND == DER2)
        return op.a * ((v[5] - v[4]) - (v[4] - v[3])) + op.b * ((v[6] - v[4]) - (v[4] - v[2]));
    if constexpr (KIND == DERVP) return op.a * (v[5] - v[4]) + op.b * (v[6] - v[3]);
    if constexpr (KIND == DERPV) return op.a * (v[4] - v[3]) + op.b * (v[5] - v[2]);
    if constexpr (KIND == INTVP)
        return op.a * (v[5] + v[4]) + op.b * (v[6] + v[3]) + op.c * (v[7] + v[2]) + op.d * (v[8] + v[1]);
    if constexpr (KIND == INTPV)
        return op.a * (v[4] + v[3]) + op.b * (v[5] + v[2]) + op.c * (v[6] + v[1]) + op.d * (v[7] + v[0]);
    return v[4];
}

template <int KIND, typename T, int L>
__device__ __forceinline__ void chunk_stencil(const T (&w)[L + 8], T (&r)[L], const LineOp<T> &op)
{
#pragma unroll
    for (int j = 0; j < L; ++j) r[j] = stencil_at<KIND>(w + j, op);
}

template <typename T, int L>
__device__ __forceinline__ void chunk_stencil_kind(int kind, const T (&w)[L + 8], T (&r)[L],
                                                   const LineOp<T> &op)
{
    switch (kind) {
    case DER: chunk_stencil<DER, T, L>(w, r, op); break;
    case DER2: chunk_stencil<DER2, T, L>(w, r, op); break;
    case DERVP: chunk_stencil<DERVP, T, L>(w, r, op); break;
    case DERPV: chunk_stencil<DERPV, T, L>(w, r, op); break;
    case INTVP: chunk_stencil<INTVP, T, L>(w, r, op); break;
    case INTPV: chunk_stencil<INTPV, T, L>(w, r, op); break;
    default: chunk_stencil<IDENT, T, L>(w, r, op); break;
    }
}

// Scratch in shared memory after the input tile: per (chunk, line) the
// forward end value / multiplier / y_0 share and the backward start value /
// multiplier.
template <typename T>
struct ChunkScratch {
    T *fz, *fm, *bz, *bm;
    double *fg;
};

// Steps 1-4 for one operator; the solved values end in r[] (chunk-local).
// load(w) fills the L+8 input window u[cs-4 .. cs+L+3] (indices mod n) from
// the staged tile; the window is dead once the stencil is evaluated.
template <typename T, int W, int L, typename Load>
__device__ __forceinline__ void chunk_solve(const LineOp<T> &op, int kind, const Load &load,
                                            T (&r)[L], const ChunkScratch<T> &sc, int l, int c,
                                            int C, int cs, int nv)
{
    {
        T w[L + 8];
        load(w);
        chunk_stencil_kind<T, L>(kind, w, r, op);
    }
    // local forward sweep
    T zh = T(0), m = T(1);
    double gp = 0.0;
    const bool has_g = cs < op.glen;
#pragma unroll
    for (int j = 0; j < L; ++j) {
        if (j < nv) {
            const int i = cs + j;
            const T s = __ldg(op.s + i);
            if (has_g) gp = fma(__ldg(op.g + i), (double)r[j], gp);
            zh = r[j] - s * zh;
            m = -s * m;
            r[j] = zh;
        }
    }
    const int q = c * W + l;
    sc.fz[q] = zh;
    sc.fm[q] = m;
    sc.fg[q] = gp;
    __syncthreads();
    // forward carries, y_0 and z_{n-1}
    T carry = T(0), run = T(0);
    double y0 = 0.0;
    const int cg = min(C, (op.glen + L - 1) / L);
    for (int cc = 0; cc < C; ++cc) {
        if (cc == c) carry = run;
        const int qq = cc * W + l;
        run = sc.fz[qq] + sc.fm[qq] * run;
        if (cc < cg) y0 += sc.fg[qq];
    }
    const T zlast = run;
    const int n = op.n;
    const double ss =
        op.periodic ? (y0 - op.alfa * ((double)zlast * (double)__ldg(op.w + (n - 1)))) / op.den : 0.0;
    // fix forward values, local backward sweep
    m = T(1);
#pragma unroll
    for (int j = 0; j < L; ++j) {
        if (j < nv) {
            m = -__ldg(op.s + cs + j) * m;
            r[j] = r[j] + m * carry;
        }
    }
    T yh = T(0), mb = T(1);
#pragma unroll
    for (int j = L - 1; j >= 0; --j) {
        if (j < nv) {
            const int i = cs + j;
            const T fw = __ldg(op.fw + i);
            yh = r[j] * __ldg(op.w + i) - fw * yh;
            mb = -fw * mb;
            r[j] = yh;
        }
    }
    sc.bz[q] = yh;
    sc.bm[q] = mb;
    __syncthreads();
    T bcarry = T(0);
    for (int cc = C - 1; cc > c; --cc) {
        const int qq = cc * W + l;
        bcarry = sc.bz[qq] + sc.bm[qq] * bcarry;
    }
    const T sst = (T)ss;
    mb = T(1);
#pragma unroll
    for (int j = L - 1; j >= 0; --j) {
        if (j < nv) {
            const int i = cs + j;
            mb = -__ldg(op.fw + i) * mb;
            r[j] = r[j] + mb * bcarry - sst * __ldg(op.p + i);
        }
    }
}

template <typename T>
__device__ __forceinline__ ChunkScratch<T> carve_scratch(unsigned char *base, int C, int W)
{
    ChunkScratch<T> sc;
    T *t = reinterpret_cast<T *>(base);
    const int q = C * W;
    sc.fz = t;
    sc.fm = t + q;
    sc.bz = t + 2 * q;
    sc.bm = t + 3 * q;
    sc.fg = reinterpret_cast<double *>(base + (((size_t)4 * q * sizeof(T) + 15) & ~(size_t)15));
    return sc;
}

// ---------------------------------------------------------------------------
// y- and z-lines.
template <typename T, int W, int L>
__global__ void __launch_bounds__(512) ls_chunk_yz(const __grid_constant__ CUtensorMap tmap,
                                                    const __grid_constant__ ChunkOps<T> ops, int nx,
                                                    int ny, int dir, int box_n, int nbox,
                                                    size_t tile_bytes, int *err)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bar;
    T *tile = reinterpret_cast<T *>(smem_raw);
    const int n = ops.op[0].n;
    const int C = blockDim.x / W;
    const int t = threadIdx.x;
    const int l = t % W, c = t / W;
    const int tiles_x = (nx + W - 1) / W;
    const int x0 = (blockIdx.x % tiles_x) * W;
    const int o = blockIdx.x / tiles_x;
    if (t == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (t == 0) {
        mbar_arrive_expect_tx(&bar, (uint32_t)((size_t)nbox * box_n * W * sizeof(T)));
        for (int b = 0; b < nbox; ++b) {
            if (dir == DY)
                tma_load_3d(tile + (size_t)b * box_n * W, &tmap, &bar, x0, b * box_n, o);
            else
                tma_load_3d(tile + (size_t)b * box_n * W, &tmap, &bar, x0, o, b * box_n);
        }
    }
    const bool ok = mbar_wait_bounded(&bar, 0, kChunkWaitNs);
    if (!__syncthreads_and(ok)) {
        if (t == 0) atomicExch(err, 1);
        mbar_wait_bounded(&bar, 0, kChunkWaitNs);
        return;
    }
    const ChunkScratch<T> sc = carve_scratch<T>(smem_raw + tile_bytes, C, W);
    const int cs = c * L;
    const int nv = min(L, n - cs);
    const T *col = tile + l;
    const bool wraps = cs < 4 || cs + L + 4 > n;
    auto load = [&](T(&w)[L + 8]) {
        if (!wraps) {
#pragma unroll
            for (int j = 0; j < L + 8; ++j) w[j] = col[(cs - 4 + j) * W];
        } else {
#pragma unroll
            for (int j = 0; j < L + 8; ++j) {
                int idx = (cs - 4 + j) % n;
                idx = idx < 0 ? idx + n : idx;
                w[j] = col[idx * W];
            }
        }
    };
    const bool live = x0 + l < nx;
    const size_t ostride = dir == DY ? (size_t)nx : (size_t)nx * ny;
    const size_t obase = (size_t)(x0 + l) + (dir == DY ? (size_t)nx * ny * o : (size_t)nx * o) +
                         (size_t)cs * ostride;
    T r[L];
    for (int k = 0; k < ops.nops; ++k) {
        chunk_solve<T, W, L>(ops.op[k], ops.kind[k], load, r, sc, l, c, C, cs, nv);
        if (live) {
            T *dst = ops.out[k] + obase;
#pragma unroll
            for (int j = 0; j < L; ++j)
                if (j < nv) dst[(size_t)j * ostride] = r[j];
        }
    }
}

// ---------------------------------------------------------------------------
// x-lines.
template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
    static constexpr int N = 4;
    using type = float4;
};
template <>
struct Vec4<double> {
    static constexpr int N = 2;
    using type = double2;
};

template <typename T, int W, int L>
__global__ void __launch_bounds__(512) ls_chunk_x(const T *__restrict__ in,
                                                   const __grid_constant__ ChunkOps<T> ops,
                                                   long nlines, int pitch, size_t tile_bytes, int *err)
{
    using VT = typename Vec4<T>::type;
    constexpr int V = Vec4<T>::N;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bar;
    T *tile = reinterpret_cast<T *>(smem_raw);
    const int n = ops.op[0].n;
    const int C = blockDim.x / W;
    const int t = threadIdx.x;
    const int l = t % W, c = t / W;
    const long l0 = (long)blockIdx.x * W;
    const int rows = (int)min((long)W, nlines - l0);
    const uint32_t row_bytes = (uint32_t)(n * sizeof(T));
    if (t == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (t == 0) {
        mbar_arrive_expect_tx(&bar, row_bytes * (uint32_t)rows);
        for (int rr = 0; rr < rows; ++rr)
            bulk_load(tile + (size_t)rr * pitch, in + (size_t)(l0 + rr) * n, row_bytes, &bar);
    }
    const bool ok = mbar_wait_bounded(&bar, 0, kChunkWaitNs);
    if (!__syncthreads_and(ok)) {
        if (t == 0) atomicExch(err, 1);
        mbar_wait_bounded(&bar, 0, kChunkWaitNs);
        return;
    }
    const ChunkScratch<T> sc = carve_scratch<T>(smem_raw + tile_bytes, C, W);
    const int cs = c * L;
    const int nv = min(L, n - cs);
    const int lr = l < rows ? l : 0;  // rows past the end compute on row 0 and store nothing
    const T *row = tile + (size_t)lr * pitch;
    auto load = [&](T(&w)[L + 8]) {
#pragma unroll
        for (int j = 0; j < L + 8; j += V) {
            int idx = (cs - 4 + j) % n;
            idx = idx < 0 ? idx + n : idx;
            const VT q = *reinterpret_cast<const VT *>(row + idx);
            const T *e = reinterpret_cast<const T *>(&q);
#pragma unroll
            for (int v = 0; v < V; ++v) w[j + v] = e[v];
        }
    };
    T r[L];
    for (int k = 0; k < ops.nops; ++k) {
        chunk_solve<T, W, L>(ops.op[k], ops.kind[k], load, r, sc, l, c, C, cs, nv);
        if (l < rows) {
            T *dst = ops.out[k] + (size_t)(l0 + l) * n + cs;
#pragma unroll
            for (int j = 0; j < L; j += V) {
                if (j < nv) {
                    VT q;
                    T *e = reinterpret_cast<T *>(&q);
#pragma unroll
                    for (int v = 0; v < V; ++v) e[v] = r[j + v];
                    *reinterpret_cast<VT *>(dst + j) = q;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Host side.

static PFN_cuTensorMapEncodeTiled_v12000 encode_tiled()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

static size_t scratch_bytes(int C, int W, size_t es)
{
    return (((size_t)4 * C * W * es + 15) & ~(size_t)15) + (size_t)C * W * sizeof(double);
}

template <typename T, int W, int L>
static int launch_chunk_cfg(x3d_ctx_s *ctx, const ChunkOps<T> &ops, int dir, const T *in, int nx,
                            int ny, int nz)
{
    const int n = ops.op[0].n;
    const size_t es = sizeof(T);
    const int C = (n + L - 1) / L;
    const int threads = C * W;
    if (threads > 512 || threads % 32) return X3D_EUNSUPPORTED;
    cudaStream_t st = ctx->stream;
    if (dir == DX) {
        constexpr int V = Vec4<T>::N;
        if (n % V || (reinterpret_cast<uintptr_t>(in) & 15)) return X3D_EUNSUPPORTED;
        for (int k = 0; k < ops.nops; ++k)
            if (reinterpret_cast<uintptr_t>(ops.out[k]) & 15) return X3D_EUNSUPPORTED;
        int pitch = n + V;
        while (((size_t)pitch * es / 16) % 2 == 0) pitch += V;
        const size_t tile = ((size_t)W * pitch * es + 127) & ~(size_t)127;
        const size_t smem = tile + scratch_bytes(C, W, es);
        if (smem + 1024 > ctx->smem_optin) return X3D_EUNSUPPORTED;
        auto kern = ls_chunk_x<T, W, L>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        const long nlines = (long)ny * nz;
        ++ctx->launches;
        kern<<<(unsigned)((nlines + W - 1) / W), threads, smem, st>>>(in, ops, nlines, pitch, tile, ctx->d_err);
        return cuda_check(ctx, cudaGetLastError(), "ls_chunk_x launch");
    }
    auto enc = encode_tiled();
    if (!enc || ((size_t)nx * es) % 16 || (reinterpret_cast<uintptr_t>(in) & 15)) return X3D_EUNSUPPORTED;
    const int nb = (n + 255) / 256;
    int box_n = (n + nb - 1) / nb;
    const int align_rows = (int)(128 / (W * es) > 0 ? 128 / (W * es) : 1);
    box_n = (box_n + align_rows - 1) / align_rows * align_rows;
    if (box_n > 256) return X3D_EUNSUPPORTED;
    const size_t tile = ((size_t)nb * box_n * W * es + 127) & ~(size_t)127;
    const size_t smem = tile + scratch_bytes(C, W, es);
    if (smem + 1024 > ctx->smem_optin) return X3D_EUNSUPPORTED;
    CUtensorMap tmap;
    cuuint64_t gdim[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    cuuint64_t gstride[2] = {(cuuint64_t)nx * es, (cuuint64_t)nx * ny * es};
    cuuint32_t box[3] = {(cuuint32_t)W, 1, 1};
    box[dir == DY ? 1 : 2] = (cuuint32_t)box_n;
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(&tmap, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                     const_cast<T *>(in), gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return X3D_EUNSUPPORTED;
    auto kern = ls_chunk_yz<T, W, L>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const long tiles_x = (nx + W - 1) / W;
    const long grid = tiles_x * (dir == DY ? nz : ny);
    ++ctx->launches;
    kern<<<(unsigned)grid, threads, smem, st>>>(tmap, ops, nx, ny, dir, box_n, nb, tile, ctx->d_err);
    return cuda_check(ctx, cudaGetLastError(), "ls_chunk_yz launch");
}

template <typename T>
int launch_chunk(x3d_ctx_s *ctx, const ChunkOps<T> &ops, int dir, const T *in, int nx, int ny, int nz,
                 int cfg)
{
    // cfg selects (lines per CTA, chunk length); see chunk_configs().
    switch (cfg) {
    case 0: return launch_chunk_cfg<T, 16, (sizeof(T) == 4 ? 32 : 16)>(ctx, ops, dir, in, nx, ny, nz);
    case 1: return launch_chunk_cfg<T, 32, (sizeof(T) == 4 ? 32 : 16)>(ctx, ops, dir, in, nx, ny, nz);
    case 2: return launch_chunk_cfg<T, 16, (sizeof(T) == 4 ? 16 : 8)>(ctx, ops, dir, in, nx, ny, nz);
    case 3: return launch_chunk_cfg<T, 8, (sizeof(T) == 4 ? 32 : 16)>(ctx, ops, dir, in, nx, ny, nz);
    default: return X3D_EUNSUPPORTED;
    }
}

template int launch_chunk<float>(x3d_ctx_s *, const ChunkOps<float> &, int, const float *, int, int, int, int);
template int launch_chunk<double>(x3d_ctx_s *, const ChunkOps<double> &, int, const double *, int, int, int, int);

}  // namespace x3d
