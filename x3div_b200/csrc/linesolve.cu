// Batched periodic line solves: explicit compact stencil + Thomas sweep +
// Sherman-Morrison correction, one kernel per operator application.
//
// Reference algorithm: derx_00 / dery_00 / derz_00 (src/x3d_derive.f90:111-152,
// 279-339, 503-558) and the periodic branches of src/x3d_staggered.f90 compute
// the RHS into the output, then ?thomas_0 (src/thomas.f90:34-58, 87-111,
// 139-163) sweeps it forward, backward and once more for the periodic
// correction: four passes over the field.  Here every line stays on chip from
// the stencil to the corrected value, so each application reads its input
// once and writes its output once:
//   forward pass : r_i = stencil(u), z_i = r_i - s_i z_{i-1}, y_0 += g_i r_i
//   between      : ss = (y_0 - alfa y_{n-1}) / (1 + p_0 - alfa p_{n-1}) in FP64
//   backward pass: y_i = z_i w_i - (f_i w_i) y_{i+1}, out_i = y_i - ss p_i
// where g is the first row of M^-1 (precomputed once in FP64), so the
// Sherman-Morrison scalar is known before the backward pass starts.
//
// Kernels
//   ls_yz_tma : y- and z-lines.  A CTA owns W x-adjacent lines; the whole
//               W x n tile is brought into shared memory by TMA tensor loads,
//               one thread sweeps one line (lane-contiguous, bank-conflict
//               free), and the backward pass stores straight to global
//               memory, coalesced across the W lanes.
//   ls_x_bulk : x-lines (contiguous).  W rows are staged by 1-D bulk copies
//               into rows padded to an odd number of 16-byte granules, so a
//               thread reading its own row with 16-byte vectors is bank
//               conflict free; results are written back in place and stored
//               with 1-D bulk copies.
//   ls_generic: any shape/alignment (odd sizes, unaligned pointers, lines
//               too long for shared memory); one thread per line straight
//               from global memory.  Correctness path, not a fast path.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>

#include "linesolve_chunk.h"
#include "ptx.cuh"
#include "x3d_internal.h"

namespace x3d {

constexpr uint64_t kWaitLimitNs = 2000000000ull;  // bounded mbarrier waits: 2 s

// ---------------------------------------------------------------------------
// Stencils on a 9-point window v[k] = u_{i-4+k}; the grouping follows the
// reference expressions (e.g. afix*(u(i+1)-u(i-1)) + bfix*(u(i+2)-u(i-2))).
// The second derivative, absent from the reference, takes differences of
// differences, which are exact for neighbouring values (Sterbenz), so its
// rounding error does not grow like 1/h^2 on fine grids.
template <int KIND, typename T>
__device__ __forceinline__ T stencil(const T *v, const LineOp<T> &op)
{
    if constexpr (KIND == DER) return op.a * (v[5] - v[3]) + op.b * (v[6] - v[2]);
    if constexpr (KIND == DER2)
        return op.a * ((v[5] - v[4]) - (v[4] - v[3])) + op.b * ((v[6] - v[4]) - (v[4] - v[2]));
    if constexpr (KIND == DERVP) return op.a * (v[5] - v[4]) + op.b * (v[6] - v[3]);
    if constexpr (KIND == DERPV) return op.a * (v[4] - v[3]) + op.b * (v[5] - v[2]);
    if constexpr (KIND == INTVP)
        return op.a * (v[5] + v[4]) + op.b * (v[6] + v[3]) + op.c * (v[7] + v[2]) + op.d * (v[8] + v[1]);
    if constexpr (KIND == INTPV)
        return op.a * (v[4] + v[3]) + op.b * (v[5] + v[2]) + op.c * (v[6] + v[1]) + op.d * (v[7] + v[0]);
    if constexpr (KIND == IDENT) return v[4];
    return T(0);
}

// Right-hand side at the first two and last two points of a non-periodic
// first-derivative line (der?_ij, src/x3d_derive.f90:171-210): v is the same
// 9-point window (v[k] = u_{i-4+k}; entries past the line's ends are never
// used here).  Free slip (ncl = 1) mirrors the field (npaire = 1: even, so
// the derivative vanishes at the wall; npaire = 0: odd); Dirichlet (ncl = 2)
// uses the one-sided closures.  Other points keep the interior stencil r.
template <typename T>
__device__ __forceinline__ T der_closure(int i, int n, const T *v, const LineOp<T> &op, T r)
{
    const T a = op.a, b = op.b;
    if (i == 0) {
        if (op.ncl1 == 1) return op.npaire == 1 ? T(0) : a * (v[5] + v[5]) + b * (v[6] + v[6]);
        return op.cl[0] * v[4] + op.cl[1] * v[5] + op.cl[2] * v[6];
    }
    if (i == 1) {
        if (op.ncl1 == 1)
            return op.npaire == 1 ? a * (v[5] - v[3]) + b * (v[6] - v[4]) : a * (v[5] - v[3]) + b * (v[6] + v[4]);
        return op.cl[3] * (v[5] - v[3]);
    }
    if (i == n - 2) {
        if (op.ncln == 1)
            return op.npaire == 1 ? a * (v[5] - v[3]) + b * (v[4] - v[2]) : a * (v[5] - v[3]) + b * ((-v[4]) - v[2]);
        return op.cl[4] * (v[5] - v[3]);
    }
    if (i == n - 1) {
        if (op.ncln == 1) return op.npaire == 1 ? T(0) : a * ((-v[3]) - v[3]) + b * ((-v[2]) - v[2]);
        return -op.cl[5] * v[4] - op.cl[6] * v[3] - op.cl[7] * v[2];
    }
    return r;
}

template <typename T>
__device__ __forceinline__ T ldg(const T *p)
{
    return __ldg(p);
}

// Column accessors: element i of one line.
template <typename T>
struct StridedRef {
    T *base;
    size_t stride;
    __device__ __forceinline__ T ld(int i) const { return base[(size_t)i * stride]; }
    __device__ __forceinline__ void st(int i, T v) const { base[(size_t)i * stride] = v; }
};

// One line, scalar accesses.  src supplies u (read ahead of the in-place
// z stores when src and zb alias), zb holds the forward-pass values, dst
// receives the results.
template <int KIND, typename T, typename Src, typename ZB, typename Dst>
__device__ __forceinline__ void solve_line(const Src &src, const ZB &zb, const Dst &dst,
                                           const LineOp<T> &op)
{
    const int n = op.n;
    T v[9];
    v[0] = src.ld(n - 4);
    v[1] = src.ld(n - 3);
    v[2] = src.ld(n - 2);
    v[3] = src.ld(n - 1);
    v[4] = src.ld(0);
    v[5] = src.ld(1);
    v[6] = src.ld(2);
    v[7] = src.ld(3);
    v[8] = src.ld(4);
    const T h0 = v[4], h1 = v[5], h2 = v[6], h3 = v[7];
    T z = T(0);
    double acc = 0.0;
    int i = 0;
    const int nmain = n - 5;
    const bool closed = KIND == DER && !op.periodic;
#pragma unroll 4
    for (; i < nmain; ++i) {
        T r = stencil<KIND>(v, op);
        if (closed && i < 2) r = der_closure(i, n, v, op, r);
        z = r - ldg(op.s + i) * z;
        acc = fma(ldg(op.g + i), (double)r, acc);
        zb.st(i, z);
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = v[k + 1];
        v[8] = src.ld(i + 5);
    }
    for (; i < n; ++i) {
        T r = stencil<KIND>(v, op);
        if (closed && (i < 2 || i >= n - 2)) r = der_closure(i, n, v, op, r);
        z = r - ldg(op.s + i) * z;
        acc = fma(ldg(op.g + i), (double)r, acc);
        zb.st(i, z);
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = v[k + 1];
        const int k = i + 5 - n;
        v[8] = k == 0 ? h0 : (k == 1 ? h1 : (k == 2 ? h2 : h3));
    }
    const T ylast = z * ldg(op.w + (n - 1));
    const double ss = op.periodic ? (acc - op.alfa * (double)ylast) / op.den : 0.0;
    const T sst = (T)ss;
    T y = T(0);
    if (op.periodic) {
#pragma unroll 4
        for (int j = n - 1; j >= 0; --j) {
            y = zb.ld(j) * ldg(op.w + j) - ldg(op.fw + j) * y;
            dst.st(j, y - sst * ldg(op.p + j));
        }
    } else {
#pragma unroll 4
        for (int j = n - 1; j >= 0; --j) {
            y = zb.ld(j) * ldg(op.w + j) - ldg(op.fw + j) * y;
            dst.st(j, y);
        }
    }
}

// ---------------------------------------------------------------------------
// y- and z-lines through TMA tiles.
template <typename T, int KIND, int W>
__global__ void __launch_bounds__(W) ls_yz_tma(const __grid_constant__ CUtensorMap tmap,
                                               T *__restrict__ out, const LineOp<T> op, int nx,
                                               int ny, int dir, int box_n, int nbox, int *err)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bar;
    T *tile = reinterpret_cast<T *>(smem_raw);
    const int tiles_x = (nx + W - 1) / W;
    const int x0 = (blockIdx.x % tiles_x) * W;
    const int o = blockIdx.x / tiles_x;
    const int lane = threadIdx.x;
    if (lane == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (lane == 0) {
        mbar_arrive_expect_tx(&bar, (uint32_t)((size_t)nbox * box_n * W * sizeof(T)));
        for (int b = 0; b < nbox; ++b) {
            if (dir == DY)
                tma_load_3d(tile + (size_t)b * box_n * W, &tmap, &bar, x0, b * box_n, o);
            else
                tma_load_3d(tile + (size_t)b * box_n * W, &tmap, &bar, x0, o, b * box_n);
        }
    }
    if (!mbar_wait_bounded(&bar, 0, kWaitLimitNs)) {
        if (lane == 0) atomicExch(err, 1);
        mbar_wait_bounded(&bar, 0, kWaitLimitNs);
        return;
    }
    if (x0 + lane >= nx) return;
    const size_t ostride = dir == DY ? (size_t)nx : (size_t)nx * ny;
    T *orow = out + (x0 + lane) + (dir == DY ? (size_t)nx * ny * o : (size_t)nx * o);
    const StridedRef<T> col{tile + lane, (size_t)W};
    const StridedRef<T> dst{orow, ostride};
    solve_line<KIND, T>(col, col, dst, op);
}

// ---------------------------------------------------------------------------
// x-lines: vector sweeps over padded shared-memory rows.
template <typename T>
struct Vec;
template <>
struct Vec<float> {
    static constexpr int N = 4;
    using type = float4;
};
template <>
struct Vec<double> {
    static constexpr int N = 2;
    using type = double2;
};

template <typename T, int V>
__device__ __forceinline__ void ldv(const T *p, T *dst)
{
    const typename Vec<T>::type q = *reinterpret_cast<const typename Vec<T>::type *>(p);
    const T *e = reinterpret_cast<const T *>(&q);
#pragma unroll
    for (int k = 0; k < V; ++k) dst[k] = e[k];
}

template <typename T, int V>
__device__ __forceinline__ void stv(T *p, const T *src)
{
    typename Vec<T>::type q;
    T *e = reinterpret_cast<T *>(&q);
#pragma unroll
    for (int k = 0; k < V; ++k) e[k] = src[k];
    *reinterpret_cast<typename Vec<T>::type *>(p) = q;
}

// In-place solve of one contiguous row of n (n % V == 0) values in shared memory.
template <int KIND, typename T>
__device__ __forceinline__ void solve_row_vec(T *row, const LineOp<T> &op)
{
    constexpr int V = Vec<T>::N;
    const int n = op.n;
    T wb[8 + V];  // wb[k] = u_{i-4+k}
    T head[4];    // u_0..u_3 for the wrap-around at the end of the row
    ldv<T, V>(row + n - 4, wb);
    if constexpr (V == 2) ldv<T, V>(row + n - 2, wb + 2);
#pragma unroll
    for (int k = 0; k < V + 4; k += V) ldv<T, V>(row + k, wb + 4 + k);
#pragma unroll
    for (int k = 0; k < 4; ++k) head[k] = wb[4 + k];
    T z = T(0);
    double acc = 0.0;
    const bool closed = KIND == DER && !op.periodic;
    for (int i = 0; i < n; i += V) {
        T zv[V];
#pragma unroll
        for (int q = 0; q < V; ++q) {
            T r = stencil<KIND>(wb + q, op);
            if (closed && (i + q < 2 || i + q >= n - 2)) r = der_closure(i + q, n, wb + q, op, r);
            z = r - ldg(op.s + i + q) * z;
            acc = fma(ldg(op.g + i + q), (double)r, acc);
            zv[q] = z;
        }
        stv<T, V>(row + i, zv);
#pragma unroll
        for (int k = 0; k < 8; ++k) wb[k] = wb[k + V];
        const int j = i + V + 4;  // first element of the next vector
        if (j < n) {
            ldv<T, V>(row + j, wb + 8);
        } else {
            const int h = j - n;  // 0 (V=4) or 0, 2 (V=2)
#pragma unroll
            for (int q = 0; q < V; ++q) wb[8 + q] = h == 0 ? head[q] : head[(2 + q) & 3];
        }
    }
    const T ylast = z * ldg(op.w + (n - 1));
    const double ss = op.periodic ? (acc - op.alfa * (double)ylast) / op.den : 0.0;
    const T sst = (T)ss;
    T y = T(0);
    for (int i = n - V; i >= 0; i -= V) {
        T zv[V], xv[V];
        ldv<T, V>(row + i, zv);
#pragma unroll
        for (int q = V - 1; q >= 0; --q) {
            y = zv[q] * ldg(op.w + i + q) - ldg(op.fw + i + q) * y;
            xv[q] = op.periodic ? y - sst * ldg(op.p + i + q) : y;
        }
        stv<T, V>(row + i, xv);
    }
}

template <typename T, int KIND, int W>
__global__ void __launch_bounds__(W) ls_x_bulk(const T *__restrict__ in, T *__restrict__ out,
                                               const LineOp<T> op, long nlines, int pitch, int *err)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bar;
    T *tile = reinterpret_cast<T *>(smem_raw);
    const int n = op.n;
    const long l0 = (long)blockIdx.x * W;
    const int rows = (int)min((long)W, nlines - l0);
    const int lane = threadIdx.x;
    const uint32_t row_bytes = (uint32_t)(n * sizeof(T));
    if (lane == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (lane == 0) {
        mbar_arrive_expect_tx(&bar, row_bytes * (uint32_t)rows);
        for (int r = 0; r < rows; ++r)
            bulk_load(tile + (size_t)r * pitch, in + (size_t)(l0 + r) * n, row_bytes, &bar);
    }
    if (!mbar_wait_bounded(&bar, 0, kWaitLimitNs)) {
        if (lane == 0) atomicExch(err, 1);
        mbar_wait_bounded(&bar, 0, kWaitLimitNs);
        return;
    }
    if (lane < rows) {
        T *row = tile + (size_t)lane * pitch;
        solve_row_vec<KIND, T>(row, op);
        fence_proxy_async_smem();
        bulk_store(out + (size_t)(l0 + lane) * n, row, row_bytes);
        bulk_commit();
        bulk_wait_read_all();
    }
}

// ---------------------------------------------------------------------------
// Generic path: one thread per line in global memory.
template <typename T, int KIND>
__global__ void ls_generic(const T *in, T *out, const LineOp<T> op, int nx, int ny, int nz, int dir)
{
    long nl;
    size_t st;
    if (dir == DX) { nl = (long)ny * nz; st = 1; }
    else if (dir == DY) { nl = (long)nx * nz; st = nx; }
    else { nl = (long)nx * ny; st = (size_t)nx * ny; }
    const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    size_t base;
    if (dir == DX) base = (size_t)l * nx;
    else if (dir == DY) base = (size_t)(l % nx) + (size_t)nx * ny * (size_t)(l / nx);
    else base = (size_t)l;
    const StridedRef<T> src{const_cast<T *>(in) + base, st};
    const StridedRef<T> zb{out + base, st};
    solve_line<KIND, T>(src, zb, zb, op);
}

// ---------------------------------------------------------------------------
// Non-periodic staggered operators (the nclx = .false. branches of
// src/x3d_staggered.f90): one thread per line, from an input line of n_in
// points to an output line of op.n = n_in -/+ 1 points.  Every boundary row
// of the reference is the interior stencil applied to a reflected input:
//   velocity-grid input (vp), npaire 1: u(1-k) = u(1+k), u(n+k) = u(n-k),
//     a mirror about the end points (the walls);
//   velocity-grid input, the odd closure of derxvp's other branch (:83-101,
//     and deryvp's only one, :595-622): u(1-k) = 2 u(1) - u(1+k), likewise
//     at n;
//   pressure-grid input (pv), npaire 1: p(1-k) = p(k), p(nm+k) = p(nm+1-k),
//     a mirror about the walls half a cell outside.
// E.g. derxvp's tx(1) = a(u(2)-u(1)) + b(u(3)-u(2)) is the interior
// a(u(i+1)-u(i)) + b(u(i+2)-u(i-1)) with u(0) = u(2), and derxpv's
// tx(1) = 0 is the interior with p(0) = p(1), p(-1) = p(2).  The solve is the
// plain Thomas of ?thomas_12 (src/thomas.f90:61-84).  Lines of the other two
// directions are enumerated as (o1, o2), the input's and output's extents
// there.
enum { kReflEven = 0, kReflOdd = 1 };

template <typename T, int KIND>
__global__ void ls_np_stag(const T *__restrict__ in, T *__restrict__ out, const LineOp<T> op, int n_in, int o1,
                           int o2, int dir, int refl)
{
    constexpr bool VP = KIND == DERVP || KIND == INTVP;
    const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= (long)o1 * o2) return;
    const int m = op.n;
    size_t bi, bo, st;
    if (dir == DX) {
        bi = (size_t)l * n_in;
        bo = (size_t)l * m;
        st = 1;
    } else if (dir == DY) {
        const size_t i = (size_t)(l % o1), k = (size_t)(l / o1);
        bi = i + (size_t)o1 * n_in * k;
        bo = i + (size_t)o1 * m * k;
        st = (size_t)o1;
    } else {
        bi = bo = (size_t)l;
        st = (size_t)o1 * o2;
    }
    const T *u = in + bi;
    T *t = out + bo;
    auto ld = [&](int k) -> T {
        if (k >= 0 && k < n_in) return u[(size_t)k * st];
        if (VP) {
            const T v = u[(size_t)(k < 0 ? -k : 2 * (n_in - 1) - k) * st];
            if (refl == kReflOdd) {
                const T e = u[(size_t)(k < 0 ? 0 : n_in - 1) * st];
                return (e + e) - v;
            }
            return v;
        }
        return u[(size_t)(k < 0 ? -1 - k : 2 * n_in - 1 - k) * st];
    };
    T v[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) v[k] = ld(k - 4);
    T z = T(0);
    for (int i = 0; i < m; ++i) {
        z = stencil<KIND>(v, op) - ldg(op.s + i) * z;
        t[(size_t)i * st] = z;
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = v[k + 1];
        v[8] = ld(i + 5);
    }
    T y = T(0);
    for (int i = m - 1; i >= 0; --i) {
        y = t[(size_t)i * st] * ldg(op.w + i) - ldg(op.fw + i) * y;
        t[(size_t)i * st] = y;
    }
}

// ---------------------------------------------------------------------------
// Host side.

template <typename T>
static const LineOp<T> &lineop(const x3d_op_s *op);
template <>
const LineOp<float> &lineop<float>(const x3d_op_s *op)
{
    return op->opf;
}
template <>
const LineOp<double> &lineop<double>(const x3d_op_s *op)
{
    return op->opd;
}

static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename T, int KIND>
static int run_kind(x3d_ctx_s *ctx, const x3d_op_s *op, int dir, const T *in, T *out, int nx,
                    int ny, int nz)
{
    const LineOp<T> &lo = lineop<T>(op);
    const int n = lo.n;
    const size_t es = sizeof(T);
    cudaStream_t st = ctx->stream;
    const bool ptr_ok = aligned16(in) && aligned16(out);
    constexpr int V = Vec<T>::N;
    constexpr int W = sizeof(T) == 4 ? 32 : 16;

    if (dir == DX) {
        const long nlines = (long)ny * nz;
        int pitch = n + V;  // odd number of 16-byte granules per row
        while (((size_t)pitch * es / 16) % 2 == 0) pitch += V;
        const size_t smem = (size_t)W * pitch * es;
        if (ptr_ok && n % V == 0 && smem + 1024 <= ctx->smem_optin && in != out) {
            auto kern = ls_x_bulk<T, KIND, W>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            const long grid = (nlines + W - 1) / W;
            ++ctx->launches;
            kern<<<(unsigned)grid, W, smem, st>>>(in, out, lo, nlines, pitch, ctx->d_err);
            return cuda_check(ctx, cudaGetLastError(), "ls_x_bulk launch");
        }
    } else {
        const int nb = (n + 255) / 256;
        const int box_n = (n + nb - 1) / nb;
        const size_t smem = (size_t)nb * box_n * W * es;
        auto enc = encode_tiled();
        if (enc && ptr_ok && ((size_t)nx * es) % 16 == 0 && smem + 1024 <= ctx->smem_optin) {
            CUtensorMap tmap;
            cuuint64_t gdim[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
            cuuint64_t gstride[2] = {(cuuint64_t)nx * es, (cuuint64_t)nx * ny * es};
            cuuint32_t box[3] = {(cuuint32_t)W, 1, 1};
            box[dir == DY ? 1 : 2] = (cuuint32_t)box_n;
            cuuint32_t estr[3] = {1, 1, 1};
            CUresult r = enc(&tmap, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                             3, const_cast<T *>(in), gdim, gstride, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r == CUDA_SUCCESS) {
                auto kern = ls_yz_tma<T, KIND, W>;
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                const long tiles_x = (nx + W - 1) / W;
                const long grid = tiles_x * (dir == DY ? nz : ny);
                ++ctx->launches;
                kern<<<(unsigned)grid, W, smem, st>>>(tmap, out, lo, nx, ny, dir, box_n, nb, ctx->d_err);
                return cuda_check(ctx, cudaGetLastError(), "ls_yz_tma launch");
            }
        }
    }
    long nl = dir == DX ? (long)ny * nz : (dir == DY ? (long)nx * nz : (long)nx * ny);
    const int bs = 128;
    ++ctx->launches;
    ls_generic<T, KIND><<<(unsigned)((nl + bs - 1) / bs), bs, 0, st>>>(in, out, lo, nx, ny, nz, dir);
    return cuda_check(ctx, cudaGetLastError(), "ls_generic launch");
}

template <typename T>
static int run_typed(x3d_ctx_s *ctx, const x3d_op_s *op, int kind, int dir, const void *in,
                     void *out, int nx, int ny, int nz)
{
    const T *i = static_cast<const T *>(in);
    T *o = static_cast<T *>(out);
    switch (kind) {
    case DER: return run_kind<T, DER>(ctx, op, dir, i, o, nx, ny, nz);
    case DER2: return run_kind<T, DER2>(ctx, op, dir, i, o, nx, ny, nz);
    case DERVP: return run_kind<T, DERVP>(ctx, op, dir, i, o, nx, ny, nz);
    case DERPV: return run_kind<T, DERPV>(ctx, op, dir, i, o, nx, ny, nz);
    case INTVP: return run_kind<T, INTVP>(ctx, op, dir, i, o, nx, ny, nz);
    case INTPV: return run_kind<T, INTPV>(ctx, op, dir, i, o, nx, ny, nz);
    case IDENT: return run_kind<T, IDENT>(ctx, op, dir, i, o, nx, ny, nz);
    default: return set_error(ctx, X3D_EINVAL, "unknown operator kind");
    }
}

// ---------------------------------------------------------------------------
// Dispatch.  Candidates for a group of operators sharing one input and one
// direction: the chunked kernel in each of its configurations (one launch
// for the whole group), then one thread-per-line launch per operator, then
// the generic kernel.  The autotuner times the candidates once per
// (direction, grid, precision, group size) and remembers the fastest.

static int run_tpl(x3d_ctx_s *ctx, int dir, const void *in, const x3d_op_s *const *ops,
                   const int *kinds, void *const *outs, int nops, int nx, int ny, int nz, bool fp32)
{
    for (int k = 0; k < nops; ++k) {
        const int rc = fp32 ? run_typed<float>(ctx, ops[k], kinds[k], dir, in, outs[k], nx, ny, nz)
                            : run_typed<double>(ctx, ops[k], kinds[k], dir, in, outs[k], nx, ny, nz);
        if (rc) return rc;
    }
    ctx->last_cfg = kChunkConfigs;
    return X3D_OK;
}

template <typename T>
static int run_chunk(x3d_ctx_s *ctx, int dir, const void *in, const x3d_op_s *const *ops,
                     const int *kinds, void *const *outs, int nops, int nx, int ny, int nz, int cfg)
{
    const LineOp<T> *lops[kMaxStageOps];
    for (int k = 0; k < nops; ++k) {
        lops[k] = &lineop<T>(ops[k]);
        if (kinds[k] == IDENT || outs[k] == in) return X3D_EUNSUPPORTED;  // in-place Thomas: other paths
    }
    const StageProgram<T> prog = plain_program<T>(static_cast<const T *>(in), lops, kinds, outs, nops);
    return launch_stage<T>(ctx, prog, dir, nx, ny, nz, cfg);
}

// cfg: a chunked configuration (is_stage_cfg), or kChunkConfigs for one
// thread per line.
static int run_cfg(x3d_ctx_s *ctx, int cfg, int dir, const void *in, const x3d_op_s *const *ops,
                   const int *kinds, void *const *outs, int nops, int nx, int ny, int nz, bool fp32)
{
    if (is_stage_cfg(cfg))
        return fp32 ? run_chunk<float>(ctx, dir, in, ops, kinds, outs, nops, nx, ny, nz, cfg)
                    : run_chunk<double>(ctx, dir, in, ops, kinds, outs, nops, nx, ny, nz, cfg);
    return run_tpl(ctx, dir, in, ops, kinds, outs, nops, nx, ny, nz, fp32);
}

static std::string tune_key(int dir, int nx, int ny, int nz, bool fp32, int nops)
{
    return std::to_string(dir) + ":" + std::to_string(nx) + "x" + std::to_string(ny) + "x" +
           std::to_string(nz) + ":" + (fp32 ? "f32" : "f64") + ":" + std::to_string(nops);
}

int launch_group(x3d_ctx_s *ctx, int dir, const void *in, const x3d_op_s *const *ops,
                 const int *kinds, void *const *outs, int nops, int nx, int ny, int nz, bool fp32)
{
    if (nops < 1 || nops > kMaxStageOps) return set_error(ctx, X3D_EINVAL, "bad operator group");
    const auto it = ctx->tuned.find(tune_key(dir, nx, ny, nz, fp32, nops));
    const int first = it != ctx->tuned.end() ? it->second : ctx->default_cfg;
    int rc = run_cfg(ctx, first, dir, in, ops, kinds, outs, nops, nx, ny, nz, fp32);
    if (rc != X3D_EUNSUPPORTED) return rc;
    for (int cfg = 0; cfg < kAllConfigs; ++cfg) {
        if (cfg == first) continue;
        rc = run_cfg(ctx, cfg, dir, in, ops, kinds, outs, nops, nx, ny, nz, fp32);
        if (rc != X3D_EUNSUPPORTED) return rc;
    }
    return set_error(ctx, X3D_EUNSUPPORTED, "no kernel accepts this operator group");
}

int launch_linesolve(x3d_ctx_s *ctx, const x3d_op_s *op, int kind, int dir, const void *in,
                     void *out, int nx, int ny, int nz, bool fp32)
{
    return launch_group(ctx, dir, in, &op, &kind, &out, 1, nx, ny, nz, fp32);
}

// Times every candidate on the given buffers (outputs are overwritten) and
// records the fastest.  Not callable during stream capture.
int autotune_group(x3d_ctx_s *ctx, int dir, const void *in, const x3d_op_s *const *ops,
                   const int *kinds, void *const *outs, int nops, bool fp32, int reps, float *best_ms)
{
    const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int best = -1;
    float bt = 0.f;
    for (int cfg = 0; cfg < kAllConfigs; ++cfg) {
        int rc = run_cfg(ctx, cfg, dir, in, ops, kinds, outs, nops, nx, ny, nz, fp32);  // warm-up / probe
        if (rc == X3D_EUNSUPPORTED) continue;
        if (rc) break;
        cudaEventRecord(a, ctx->stream);
        for (int r = 0; r < reps; ++r) run_cfg(ctx, cfg, dir, in, ops, kinds, outs, nops, nx, ny, nz, fp32);
        cudaEventRecord(b, ctx->stream);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (best < 0 || ms < bt) {
            best = cfg;
            bt = ms;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (best < 0) return set_error(ctx, X3D_EUNSUPPORTED, "no kernel accepts this operator group");
    ctx->tuned[tune_key(dir, nx, ny, nz, fp32, nops)] = best;
    if (best_ms) *best_ms = bt / reps;
    return X3D_OK;
}

// Which non-periodic branches the reference has (src/x3d_staggered.f90):
// derxvp and derzvp one for npaire 1 and one for the rest (:64, :944),
// deryvp only the odd one, for npaire 0 (:595); every other staggered
// routine only npaire 1.  Without a branch the reference computes nothing;
// here the call returns X3D_EUNSUPPORTED.
int launch_np_stag(x3d_ctx_s *ctx, const x3d_op_s *op, int dir, const void *in, void *out, int n_in, int o1, int o2,
                   bool fp32)
{
    const int kind = op->h.kind, np = op->h.npaire;
    int refl = kReflEven;
    if (kind == DERVP) {
        if (dir == DY) {
            if (np != 0)
                return set_error(ctx, X3D_EUNSUPPORTED,
                                 "deryvp has a non-periodic branch for npaire 0 only (src/x3d_staggered.f90:595)");
            refl = kReflOdd;
        } else {
            refl = np == 1 ? kReflEven : kReflOdd;
        }
    } else if (np != 1) {
        return set_error(ctx, X3D_EUNSUPPORTED,
                         "this staggered routine has a non-periodic branch for npaire 1 only (src/x3d_staggered.f90)");
    }
    const long nl = (long)o1 * o2;
    const int bs = 128;
    const unsigned grid = (unsigned)((nl + bs - 1) / bs);
    auto go = [&](auto kern, const auto *i, auto *o, const auto &lo) {
        ++ctx->launches;
        kern<<<grid, bs, 0, ctx->stream>>>(i, o, lo, n_in, o1, o2, dir, refl);
        return cuda_check(ctx, cudaGetLastError(), "ls_np_stag launch");
    };
    if (fp32) {
        const float *i = static_cast<const float *>(in);
        float *o = static_cast<float *>(out);
        switch (kind) {
        case DERVP: return go(ls_np_stag<float, DERVP>, i, o, op->opf);
        case INTVP: return go(ls_np_stag<float, INTVP>, i, o, op->opf);
        case DERPV: return go(ls_np_stag<float, DERPV>, i, o, op->opf);
        default: return go(ls_np_stag<float, INTPV>, i, o, op->opf);
        }
    }
    const double *i = static_cast<const double *>(in);
    double *o = static_cast<double *>(out);
    switch (kind) {
    case DERVP: return go(ls_np_stag<double, DERVP>, i, o, op->opd);
    case INTVP: return go(ls_np_stag<double, INTVP>, i, o, op->opd);
    case DERPV: return go(ls_np_stag<double, DERPV>, i, o, op->opd);
    default: return go(ls_np_stag<double, INTPV>, i, o, op->opd);
    }
}

}  // namespace x3d
