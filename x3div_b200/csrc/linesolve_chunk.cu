// Chunked periodic line solves: the fast path for whole-field operator
// applications, and the stage kernels that fuse several operators, their
// pointwise products and their sums into one pass over the staged inputs.
//
// The reference sweeps each line serially (?thomas_12, src/thomas.f90:61-84)
// with the LU factors of its periodic matrix, then corrects for periodicity
// with the precomputed vector p (xthomas_0 :49-55).  The matrix that pair
// inverts is exactly the circulant (alfa, 1, alfa), which factors as
//   M = (1 + rho^2)^-1 (1 - rho E^-1)(1 - rho E),  alfa rho^2 + rho + alfa = 0,
// |rho| < 1.  So y = M^-1 r is two first-order periodic recurrences with one
// constant coefficient:
//   forward  v_i = (1 + rho^2) r_i + rho v_{i-1}     backward  y_i = v_i + rho y_{i+1}
// (the factor 1 + rho^2 is folded into the RHS scalars).
//
// A line of n points is cut into C chunks of L points; thread (l, c) owns
// chunk c of line l and keeps it in registers.  Each recurrence is affine in
// its incoming value, so a chunk is swept locally from zero and later
// shifted by rho^k * carry:
//   1. stencil r_i for the chunk from an L+8 window of the staged input;
//   2. local forward sweep, chunk end value to shared memory;
//   -- barrier -- each thread folds the end values of the chunks before it
//      (depth chunks, or the whole line divided by 1 - rho^n) into its
//      carry, fixes its values and sweeps backward locally;
//   -- barrier -- the same for the backward carry from the chunks after it.
// Every chunk does the same work: no tables, no per-line scalar, two
// barriers per operator and one HBM read and write per application.
//
// A stage (StageProgram) runs up to six such operators over up to three
// staged inputs, combining the results in a register accumulator and
// writing only what the program flushes, so e.g. one x-pencil pass of
// momentum_rhs_eq (src/transeq.f90:99-116, six derx calls and their
// products and sums for three velocity components) is one kernel.
//
// Staging: y/z tiles of W x-adjacent lines arrive by TMA tensor loads and
// results go straight to global memory, coalesced across the W lines; x
// tiles arrive as W padded rows by 1-D bulk copies and results leave as
// 16-byte vector stores of each thread's contiguous chunk.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "linesolve_chunk.h"
#include "ptx.cuh"
#include "x3d_internal.h"

namespace x3d {

constexpr uint64_t kChunkWaitNs = 2000000000ull;

// Two x-adjacent y/z lines' values in one 64-bit register pair, computed with
// the packed FP32 instructions of sm_100: per lane the same IEEE operations
// (round-to-nearest add, multiply, fused multiply-add) as the scalar code,
// for half the instructions.
struct F2 {
    float2 v;
    F2() = default;
    __device__ __forceinline__ explicit F2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ explicit F2(float2 x) : v(x) {}
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
// a - b as b * (-1) + a: one rounding of the exact difference, as a subtraction
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 &operator+=(F2 &a, F2 b) { return a = a + b; }
// fma for the scalar types too, so that the unqualified calls below resolve
// to the exact overload inside this namespace
__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) { return F2(__ffma2_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ float fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma(double a, double b, double c) { return ::fma(a, b, c); }

// Value type of a stage kernel that carries PR lines per thread.
template <typename T, int PR>
struct PairOf {
    using type = T;
};
template <>
struct PairOf<float, 2> {
    using type = F2;
};

// PR consecutive values of U (one per line of a pair), as one load or store.
template <typename U, int PR>
struct Lanes {
    using type = U;
};
template <>
struct Lanes<float, 2> {
    using type = float2;
};
template <>
struct Lanes<double, 2> {
    using type = double2;
};

// Launch bounds of the stage kernels: up to 512 threads with the registers
// of one such CTA per SM (128 per thread), so that no configuration spills
// its chunk; a paired kernel with long chunks keeps twice the values per
// thread and is limited to 256 threads.
template <typename T, int L, int PR>
constexpr int kStageThreads = PR == 2 && L == kChunkLong<T> ? 256 : 512;

// RHS scalars of a stencil (the operator's, times 1 + rho^2).
template <typename T>
struct Coef {
    T a, b, c, d;
};

template <int KIND, typename T>
__device__ __forceinline__ T stencil_at(const T *v, const Coef<T> &k)
{
    // v[m] = u_{i-4+m}.  The packed type needs its fused multiply-adds
    // spelled out; the scalar types leave contraction to the compiler.
    if constexpr (!std::is_same<T, F2>::value) {
        if constexpr (KIND == DER) return k.a * (v[5] - v[3]) + k.b * (v[6] - v[2]);
        if constexpr (KIND == DER2)
            return k.a * ((v[5] - v[4]) - (v[4] - v[3])) + k.b * ((v[6] - v[4]) - (v[4] - v[2]));
        if constexpr (KIND == DERVP) return k.a * (v[5] - v[4]) + k.b * (v[6] - v[3]);
        if constexpr (KIND == DERPV) return k.a * (v[4] - v[3]) + k.b * (v[5] - v[2]);
        if constexpr (KIND == INTVP)
            return k.a * (v[5] + v[4]) + k.b * (v[6] + v[3]) + k.c * (v[7] + v[2]) + k.d * (v[8] + v[1]);
        if constexpr (KIND == INTPV)
            return k.a * (v[4] + v[3]) + k.b * (v[5] + v[2]) + k.c * (v[6] + v[1]) + k.d * (v[7] + v[0]);
        return v[4];
    }
    if constexpr (KIND == DER) return fma(k.a, v[5] - v[3], k.b * (v[6] - v[2]));
    if constexpr (KIND == DER2)
        return fma(k.a, (v[5] - v[4]) - (v[4] - v[3]), k.b * ((v[6] - v[4]) - (v[4] - v[2])));
    if constexpr (KIND == DERVP) return fma(k.a, v[5] - v[4], k.b * (v[6] - v[3]));
    if constexpr (KIND == DERPV) return fma(k.a, v[4] - v[3], k.b * (v[5] - v[2]));
    if constexpr (KIND == INTVP)
        return fma(k.a, v[5] + v[4], fma(k.b, v[6] + v[3], fma(k.c, v[7] + v[2], k.d * (v[8] + v[1]))));
    if constexpr (KIND == INTPV)
        return fma(k.a, v[4] + v[3], fma(k.b, v[5] + v[2], fma(k.c, v[6] + v[1], k.d * (v[7] + v[0]))));
    return v[4];
}

// r[OFF + j] for j < N from a window w of N + 8 values (w[m] = u_{OFF+j-4+m}).
template <int KIND, typename T, int N, int L, int OFF>
__device__ __forceinline__ void chunk_stencil(const T (&w)[N + 8], T (&r)[L], const Coef<T> &k)
{
#pragma unroll
    for (int j = 0; j < N; ++j) r[OFF + j] = stencil_at<KIND>(w + j, k);
}

template <typename T, int N, int L, int OFF, typename S>
__device__ __forceinline__ void chunk_stencil_kind(int kind, const T (&w)[N + 8], T (&r)[L],
                                                   const LineOp<S> &op)
{
    const Coef<T> k{T(op.ca), T(op.cb), T(op.cc), T(op.cd)};
    switch (kind) {
    case DER: chunk_stencil<DER, T, N, L, OFF>(w, r, k); break;
    case DER2: chunk_stencil<DER2, T, N, L, OFF>(w, r, k); break;
    case DERVP: chunk_stencil<DERVP, T, N, L, OFF>(w, r, k); break;
    case DERPV: chunk_stencil<DERPV, T, N, L, OFF>(w, r, k); break;
    case INTVP: chunk_stencil<INTVP, T, N, L, OFF>(w, r, k); break;
    case INTPV: chunk_stencil<INTPV, T, N, L, OFF>(w, r, k); break;
    default: chunk_stencil<IDENT, T, N, L, OFF>(w, r, k); break;
    }
}

// The explicit right-hand side of a whole chunk, in P parts of L/P points,
// each from its own window of L/P + 8 staged values, so that only one part's
// window is live next to r.  load(w, J0) fills w[m] = u_{cs+J0-4+m}.
template <typename T, int L, int P, int I = 0, typename Load, typename S>
__device__ __forceinline__ void chunk_rhs(int kind, const Load &load, T (&r)[L], const LineOp<S> &op)
{
    if constexpr (I < P) {
        constexpr int N = L / P;
        {
            T w[N + 8];
            load(w, std::integral_constant<int, I * N>{});
            chunk_stencil_kind<T, N, L, I * N>(kind, w, r, op);
        }
        chunk_rhs<T, L, P, I + 1>(kind, load, r, op);
    }
}

// Staged lines carry periodic halos, so a chunk's window never wraps:
// shared-memory row (y/z tiles) or element (x rows) kHalo + i holds point i
// of the line for -4 <= i < n + 4, and the rows past that up to the end of
// the last chunk's window exist but hold values that are never used.
constexpr int kHalo = 4;

// Fills the halos of ntiles staged y/z tiles of W columns whose point i sits
// in row h0 + i: rows h0-4 .. h0-1 from points n-4 .. n-1, rows h0+n ..
// h0+n+3 from points 0 .. 3.
template <typename T>
__device__ __forceinline__ void fill_halos_yz(unsigned char *base, size_t tile_bytes, int ntiles, int n, int W,
                                              int h0)
{
    const int per = 8 * W;
    for (int i = threadIdx.x; i < per * ntiles; i += blockDim.x) {
        const int ti = i / per, r = i - ti * per;
        const int h = r / W, x = r - h * W;
        T *tp = reinterpret_cast<T *>(base + ti * tile_bytes);
        const int dst = h < 4 ? h0 - 4 + h : h0 + n + h - 4;
        const int src = h < 4 ? h0 + n - 4 + h : h0 + h - 4;
        tp[dst * W + x] = tp[src * W + x];
    }
}

// Scratch in shared memory after the input tiles: per (chunk, line) the
// forward end value and the backward start value of the local sweeps.
template <typename T>
struct ChunkScratch {
    T *fz, *bz;
};

// Carry into chunk c: the end values e of the chunks before it (STEP = 1,
// forward sweep) or the start values of the chunks after it (STEP = -1,
// backward), folded from the farthest in over depth chunks, or over the
// whole line once and scaled by 1 / (1 - rho^n).  A chunk propagates an
// incoming carry by rho^L (rho^nv for the last, possibly short, chunk); the
// first chunk folded multiplies zero, so only a later visit to chunk C-1
// needs its own multiplier.  The visits run as at most two unwrapped
// segments of e.
template <typename T, int STEP>
__device__ __forceinline__ T chunk_carry(const T *e, int K, T mf, T ml, T wrap, int W, int l, int c, int C)
{
    const bool full = K >= C;
    T carry = T(0);
    if (STEP == 1) {
        int s = full ? c : c - K;
        s = s < 0 ? s + C : s;
        const int n1 = min(K, C - s);  // chunks s .. s+n1-1, then 0 .. K-n1-1
        const T *p = e + s * W + l;
#pragma unroll 4
        for (int k = 1; k < n1; ++k, p += W) carry = fma(mf, carry, *p);
        carry = fma(s + n1 == C ? ml : mf, carry, *p);
        p = e + l;
#pragma unroll 4
        for (int k = n1; k < K; ++k, p += W) carry = fma(mf, carry, *p);
    } else {
        int s = full ? c : c + K;
        s = s >= C ? s - C : s;
        const int n1 = min(K, s + 1);  // chunks s .. s-n1+1, then C-1 .. C-K+n1
        const T *p = e + s * W + l;
#pragma unroll 4
        for (int k = 0; k < n1; ++k, p -= W) carry = fma(mf, carry, *p);
        if (K > n1) {
            p = e + (C - 1) * W + l;
            carry = fma(ml, carry, *p);
            p -= W;
#pragma unroll 4
            for (int k = n1 + 1; k < K; ++k, p -= W) carry = fma(mf, carry, *p);
        }
    }
    return full ? carry * wrap : carry;
}

// 16-byte vector of T.
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
template <>
struct Vec4<F2> {
    static constexpr int N = 2;
    using type = float4;
};

// Shared-memory copy of the carry responses of a stage's operators, laid
// out [operator][4][L] (see StageOp::resp), made once per CTA.
template <typename V, int L, typename S>
__device__ __forceinline__ void load_resp(const StageProgram<S> &prog, V *dst)
{
    const int total = prog.nops * 4 * L;
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        const int k = i / (4 * L), rem = i - k * 4 * L, a = rem / L, j = rem - a * L;
        dst[i] = V(prog.ops[k].resp[a][j]);
    }
}

// Solves one operator for one chunk; the solved values end in r[] (chunk
// local).  load(w, J0) fills a window u[cs+J0-4 ...] of the size of w from the
// staged line and its periodic halos; nv = points of the chunk inside the
// line (L except for the last chunk of a ragged line).  The carry fixes are
// folded into two precomputed responses: both local sweeps run before the
// first barrier (the backward one on the local forward values), and since
// the solve is linear,
//   y_j = y_j(local) + F h_j + B g_j,
//   h_j = sum_{m=j}^{len-1} rho^(2m-j+1),   g_j = rho^(len-j),
// with F the true v just before the chunk and B the true y just after it.
// The chunk's start value for the backward scan is y_0(local) + F h_0, so
// each thread publishes it after finding its own F.  h and g (resp[0..1],
// or resp[2..3] for a short last chunk) come from this operator's block of
// the shared-memory copy as 16-byte vectors, so each fix is one fused
// multiply-add per carry and half a load per point.
//
// keep = nh | ng << 8 (full chunks): the fixes by h_j for j >= nh and by
// g_j for j < L - ng are dropped, their responses being below 2^-32 (FP32)
// or 2^-62 (FP64) of the largest, far under the sweep's rounding (for the
// first derivative, rho = -0.38, that is all h past the 24th point and all g
// before the 8th; operators with |rho| < 0.2 keep half of each).  They go in
// blocks of 8 points, chosen by tests uniform across the CTA.
// Only kernels whose registers allow it (TRIM) compile the trimmed form.
template <typename T, int L, bool TRIM = false, typename Load, typename S>
__device__ __forceinline__ void chunk_solve_resp(const LineOp<S> &op, int kind, const T *resp, const Load &load,
                                                 T (&r)[L], const ChunkScratch<T> &sc, int W, int l, int c,
                                                 int C, int nv, int q, int keep = 0)
{
    constexpr int ti = L == kChunkLong<S> ? 0 : 1;
    // operator fields into registers once (the parameters are read through
    // a generic pointer, and would be read again after every barrier)
    const T rho = T(op.rho), mf = T(op.mfull[ti]), ml = T(op.mlast[ti]), wrap = T(op.wrap);
    const int K = op.depth[ti];
    chunk_rhs<T, L, 2>(kind, load, r, op);
    // local forward sweep; the chunk's end value goes straight to shared
    // memory (for a short last chunk, the value at point nv - 1, captured in
    // the sweep: selecting it from r afterwards would index r at run time
    // and move the whole array to local memory)
    T v = T(0);
    if (nv == L) {
#pragma unroll
        for (int j = 0; j < L; ++j) {
            v = fma(rho, v, r[j]);
            r[j] = v;
        }
        sc.fz[q] = v;
    } else {
#pragma unroll
        for (int j = 0; j < L; ++j) {
            v = fma(rho, v, r[j]);
            if (j + 1 == nv) sc.fz[q] = v;
            r[j] = j < nv ? v : T(0);
        }
    }
    T y = T(0);
#pragma unroll
    for (int j = L - 1; j >= 0; --j) {
        y = fma(rho, y, r[j]);
        r[j] = y;
    }
    __syncthreads();
    const T F = chunk_carry<T, 1>(sc.fz, K, mf, ml, wrap, W, l, c, C);
    const T *h = resp + (nv == L ? 0 : 2 * L);
    const T *g = h + L;
    sc.bz[q] = fma(F, h[0], y);
    __syncthreads();
    const T B = chunk_carry<T, -1>(sc.bz, K, mf, ml, wrap, W, l, c, C);
    using VT = typename Vec4<T>::type;
    constexpr int V = Vec4<T>::N;
    const int nh = keep & 0xff, ng = keep >> 8;
    if (TRIM && nv == L && keep && (nh < L || ng < L)) {
        constexpr int B8 = L < 8 ? L : 8;
#pragma unroll
        for (int j0 = 0; j0 < L; j0 += B8) {
            const bool dh = j0 < nh, dg = j0 + B8 > L - ng;
            if (dh && dg) {
#pragma unroll
                for (int j = j0; j < j0 + B8; j += V) {
                    const VT hv = *reinterpret_cast<const VT *>(h + j);
                    const VT gv = *reinterpret_cast<const VT *>(g + j);
                    const T *he = reinterpret_cast<const T *>(&hv);
                    const T *ge = reinterpret_cast<const T *>(&gv);
#pragma unroll
                    for (int v = 0; v < V; ++v) r[j + v] = fma(F, he[v], fma(B, ge[v], r[j + v]));
                }
            } else if (dh) {
#pragma unroll
                for (int j = j0; j < j0 + B8; j += V) {
                    const VT hv = *reinterpret_cast<const VT *>(h + j);
                    const T *he = reinterpret_cast<const T *>(&hv);
#pragma unroll
                    for (int v = 0; v < V; ++v) r[j + v] = fma(F, he[v], r[j + v]);
                }
            } else if (dg) {
#pragma unroll
                for (int j = j0; j < j0 + B8; j += V) {
                    const VT gv = *reinterpret_cast<const VT *>(g + j);
                    const T *ge = reinterpret_cast<const T *>(&gv);
#pragma unroll
                    for (int v = 0; v < V; ++v) r[j + v] = fma(B, ge[v], r[j + v]);
                }
            }
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < L; j += V) {
        const VT hv = *reinterpret_cast<const VT *>(h + j);
        const VT gv = *reinterpret_cast<const VT *>(g + j);
        const T *he = reinterpret_cast<const T *>(&hv);
        const T *ge = reinterpret_cast<const T *>(&gv);
#pragma unroll
        for (int v = 0; v < V; ++v) r[j + v] = fma(F, he[v], fma(B, ge[v], r[j + v]));
    }
}

template <typename T>
__device__ __forceinline__ ChunkScratch<T> carve_scratch(unsigned char *base, int C, int W)
{
    ChunkScratch<T> sc;
    T *t = reinterpret_cast<T *>(base);
    sc.fz = t;
    sc.bz = t + C * W;
    return sc;
}

// acc (+)= m * r, with m = 1 or the staged tile value at the point;
// tile_at(ti, j) returns TV consecutive tile values from point j (a 16-byte
// vector along an x row, one value per point down a y/z column).
template <typename T, int L, int TV, typename S, typename TileAt>
__device__ __forceinline__ void accumulate(const StageOp<S> &so, T (&acc)[L], const T (&r)[L],
                                           int nv, const TileAt &tile_at)
{
    if (so.mul_tile < 0) {
        if (so.accumulate) {
#pragma unroll
            for (int j = 0; j < L; ++j) acc[j] += r[j];
        } else {
#pragma unroll
            for (int j = 0; j < L; ++j) acc[j] = r[j];
        }
    } else if (so.accumulate) {
        // points past a short chunk's end read staged halo/padding rows and
        // are never stored
#pragma unroll
        for (int j = 0; j < L; j += TV) {
            const auto tv = tile_at(so.mul_tile, j);
            const T *te = reinterpret_cast<const T *>(&tv);
#pragma unroll
            for (int v = 0; v < TV; ++v) acc[j + v] = fma(te[v], r[j + v], acc[j + v]);
        }
    } else {
#pragma unroll
        for (int j = 0; j < L; j += TV) {
            const auto tv = tile_at(so.mul_tile, j);
            const T *te = reinterpret_cast<const T *>(&tv);
#pragma unroll
            for (int v = 0; v < TV; ++v) acc[j + v] = te[v] * r[j + v];
        }
    }
}

// ---------------------------------------------------------------------------
// y- and z-lines.
struct StageMaps {
    CUtensorMap m[kMaxStageTiles];   // inputs
    CUtensorMap hm[kMaxStageTiles];  // the same inputs in boxes of kHalo rows: the periodic halos
    CUtensorMap pm[kMaxStageOps];    // base (else base2) arrays prefetched into L2 (ops with prefetch_base)
};

// Flush fields of a stage operator, read from the parameters once per
// flush rather than at every store.
template <typename T>
struct FlushArgs {
    void *out;
    const void *base;
    void *out2;
    const void *base2;
    double sign, scale2;
    bool f64, plain;
    const T *b2s;  // base2 from a staged tile: this thread's point cs there, or null
    int b2step;    // elements between consecutive points of the line in that tile
    __device__ FlushArgs(const StageOp<T> &so, const T *b2s_ = nullptr, int b2step_ = 1)
        : out(so.out), base(so.base), out2(so.out2), base2(so.base2), sign(so.sign), scale2(so.scale2),
          f64(so.out_f64 != 0), b2s(b2s_), b2step(b2step_)
    {
        plain = !base && !out2 && !f64 && sign == 1.0;
    }
};

// General flush of a y/z chunk in blocks of up to 8 points: every load of a
// block (base, base2) is issued before its stores.  base and base2 are often
// the output arrays themselves (du += ..., u = u + dt du in place), so a load
// placed after a store could not be moved ahead of it, and each point would
// wait for memory in turn.  V holds PR x-adjacent lines (PR = 1 or 2), moved
// as one PR-wide load or store of U.
template <typename T, typename V, typename U, int L>
__device__ __forceinline__ void flush_yz_blocked(const FlushArgs<T> &fa, const V (&res)[L], size_t obase,
                                                 size_t ostride, int nv)
{
    constexpr int PR = sizeof(V) / sizeof(T);
    using UP = typename Lanes<U, PR>::type;
    constexpr int B = L < 8 ? L : 8;
    const U *base = static_cast<const U *>(fa.base);
    const U *base2 = static_cast<const U *>(fa.base2);
    U *out = static_cast<U *>(fa.out);
    U *out2 = static_cast<U *>(fa.out2);
    const U sign = (U)fa.sign, scale2 = (U)fa.scale2;
#pragma unroll
    for (int j0 = 0; j0 < L; j0 += B) {
        UP bv[B], b2v[B];
#pragma unroll
        for (int i = 0; i < B; ++i) {
            const size_t p = obase + (size_t)(j0 + i) * ostride;
            const bool in = j0 + i < nv;
            bv[i] = base && in ? *reinterpret_cast<const UP *>(base + p) : UP{};
            if constexpr (std::is_same<T, U>::value) {
                if (fa.b2s) b2v[i] = *reinterpret_cast<const UP *>(fa.b2s + (j0 + i) * fa.b2step);
                else b2v[i] = base2 && in ? *reinterpret_cast<const UP *>(base2 + p) : UP{};
            } else {
                b2v[i] = base2 && in ? *reinterpret_cast<const UP *>(base2 + p) : UP{};
            }
        }
#pragma unroll
        for (int i = 0; i < B; ++i) {
            if (j0 + i < nv) {
                const size_t p = obase + (size_t)(j0 + i) * ostride;
                const T *rv = reinterpret_cast<const T *>(&res[j0 + i]);
                const U *bl = reinterpret_cast<const U *>(&bv[i]);
                const U *b2l = reinterpret_cast<const U *>(&b2v[i]);
                UP o;
                U *ol = reinterpret_cast<U *>(&o);
#pragma unroll
                for (int e = 0; e < PR; ++e) ol[e] = bl[e] + sign * (U)rv[e];
                *reinterpret_cast<UP *>(out + p) = o;
                if (out2) {
                    UP o2;
                    U *o2l = reinterpret_cast<U *>(&o2);
#pragma unroll
                    for (int e = 0; e < PR; ++e) o2l[e] = b2l[e] + scale2 * ol[e];
                    *reinterpret_cast<UP *>(out2 + p) = o2;
                }
            }
        }
    }
}

// The general flush of a whole chunk (nv == L) in the forms the Euler-step
// stages use, with every test hoisted out of the point loop and the
// addresses stepped by pointer increments:
//   HB:  out = base + sign * res (else out = sign * res)
//   B2T: out2 = base2 + scale2 * out, base2 read from the staged tile b2s
// U = double writes FP64 outputs.
template <typename T, typename V, typename U, int L, bool HB, bool B2T>
__device__ __forceinline__ void flush_yz_whole(const FlushArgs<T> &fa, const V (&res)[L], size_t obase,
                                               size_t ostride)
{
    constexpr int PR = sizeof(V) / sizeof(T);
    using UP = typename Lanes<U, PR>::type;
    constexpr int B = L < 8 ? L : 8;
    const U *bp = static_cast<const U *>(fa.base) + obase;
    U *op = static_cast<U *>(fa.out) + obase;
    U *op2 = static_cast<U *>(fa.out2) + obase;
    const T *b2p = fa.b2s;
    const int b2step = fa.b2step;
    const U sign = (U)fa.sign, scale2 = (U)fa.scale2;
#pragma unroll
    for (int j0 = 0; j0 < L; j0 += B) {
        UP bv[B];
        if constexpr (HB) {
#pragma unroll
            for (int i = 0; i < B; ++i) bv[i] = *reinterpret_cast<const UP *>(bp + (size_t)i * ostride);
            bp += (size_t)B * ostride;
        }
#pragma unroll
        for (int i = 0; i < B; ++i) {
            const T *rv = reinterpret_cast<const T *>(&res[j0 + i]);
            UP o;
            U *ol = reinterpret_cast<U *>(&o);
            if constexpr (HB) {
                const U *bl = reinterpret_cast<const U *>(&bv[i]);
#pragma unroll
                for (int e = 0; e < PR; ++e) ol[e] = bl[e] + sign * (U)rv[e];
            } else {
#pragma unroll
                for (int e = 0; e < PR; ++e) ol[e] = sign * (U)rv[e];
            }
            *reinterpret_cast<UP *>(op + (size_t)i * ostride) = o;
            if constexpr (B2T) {
                const V b2 = *reinterpret_cast<const V *>(b2p + (j0 + i) * b2step);
                const T *b2l = reinterpret_cast<const T *>(&b2);
                UP o2;
                U *o2l = reinterpret_cast<U *>(&o2);
#pragma unroll
                for (int e = 0; e < PR; ++e) o2l[e] = (U)b2l[e] + scale2 * ol[e];
                *reinterpret_cast<UP *>(op2 + (size_t)i * ostride) = o2;
            }
        }
        op += (size_t)B * ostride;
        if constexpr (B2T) op2 += (size_t)B * ostride;
    }
}

// Writes one thread's solved chunk of a y/z line, or of PR x-adjacent lines
// (points j < nv), each point ostride elements after the previous one.
// GENERAL = false: the program's flushes are all plain (out = res), and the
// other forms are not compiled into the kernel.
template <typename T, typename V, int L, bool GENERAL>
__device__ __forceinline__ void flush_yz(const FlushArgs<T> &fa, const V (&res)[L], size_t obase,
                                         size_t ostride, int nv)
{
    if (GENERAL && nv == L && !fa.plain) {
        // du += ...; du += ... with u = u + dt du; pp3 = ... in FP64
        const bool hb = fa.base != nullptr, o2 = fa.out2 != nullptr;
        if (!fa.f64 && hb && !o2) return flush_yz_whole<T, V, T, L, true, false>(fa, res, obase, ostride);
        if (!fa.f64 && hb && o2 && fa.b2s)
            return flush_yz_whole<T, V, T, L, true, true>(fa, res, obase, ostride);
        if (fa.f64 && !hb && !o2) return flush_yz_whole<T, V, double, L, false, false>(fa, res, obase, ostride);
    }
    if (!GENERAL || fa.plain) {
        T *dst = static_cast<T *>(fa.out) + obase;
        if (nv == L) {  // every chunk but a short last one: no per-point test
#pragma unroll
            for (int j = 0; j < L; ++j) {
                *reinterpret_cast<V *>(dst) = res[j];
                dst += ostride;
            }
        } else {
#pragma unroll
            for (int j = 0; j < L; ++j) {
                if (j < nv) *reinterpret_cast<V *>(dst) = res[j];
                dst += ostride;
            }
        }
    } else if constexpr (GENERAL) {
        if (fa.f64) flush_yz_blocked<T, V, double, L>(fa, res, obase, ostride, nv);
        else flush_yz_blocked<T, V, T, L>(fa, res, obase, ostride, nv);
    }
}

// PERSIST: a CTA loops over tiles with two staging slots, issuing the loads
// of tile k+1 before computing tile k; otherwise one CTA per tile.  PR = 2
// (FP32 only): each thread carries the same chunk of two x-adjacent lines in
// packed registers, so every arithmetic instruction, shared-memory load and
// global store serves two lines (x extents must then be even).
//
// A persistent CTA claims its tiles one at a time from a counter (the next
// one claimed as soon as the current one's copies are issued) rather than
// taking every gridDim-th tile.  CTAs that take tiles at a fixed stride
// drift apart over a launch, and then x-adjacent tiles of a plane, whose
// 64-byte row segments make up whole rows only together, are written at
// different times.  Claimed in order, the tiles in flight stay a window of
// consecutive tiles: one read and six writes of 16-column y tiles run at
// 6.4 TB/s that way against 4.6 TB/s at a fixed stride (x3d_roofline_probe
// patterns 5 and 1).  The launcher zeroes the counter before each launch.
//
// TI: the element type of the staged inputs.  TI = double with T = float
// (plain programs, PR = 1, OCC = 1) stages FP64 fields and solves them in FP32: the
// pressure gradient reads the FP64 pressure this way, with no FP32 copy.
//
// OCC > 1: the kernel is compiled for OCC CTAs of at most 256 threads per SM
// (at most 65536 / (256 OCC) registers a thread).  With OCC = 3 the plain
// FP32 16-line, 32-point-chunk kernel fits 80 registers without spilling, so
// an SM holds 24 warps instead of 16 -- the sweep kernels are latency- and
// issue-bound at 16 (issue active about half the cycles).
template <typename T, int W, int L, bool ACC, bool PERSIST, int PR = 1, int OCC = 1, typename TI = T>
__global__ void __launch_bounds__(OCC > 1 ? 256 : kStageThreads<T, L, PR>, OCC)
    ls_stage_yz(const __grid_constant__ StageMaps maps, const __grid_constant__ StageProgram<T> prog, int nx,
                int ny, int dir, int box_n, int nbox, int tma_halo, size_t tile_bytes, long ntiles,
                unsigned long long *claim, int *err)
{
    using V = typename PairOf<T, PR>::type;
    static_assert(std::is_same<TI, T>::value || (PR == 1 && !ACC), "wider staged inputs: plain, unpaired");
    constexpr int WP = W / PR;  // threads across the tile's lines
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bars[2];
    __shared__ long s_tile[2];  // by iteration parity: rewritten only after every thread has read it
    const int n = prog.ops[0].op.n;
    const int C = blockDim.x / WP;
    const int t = threadIdx.x;
    const int l = t % WP, c = t / WP;
    const int tiles_x = (nx + W - 1) / W;
    const size_t slot_bytes = (size_t)prog.ntiles * tile_bytes;
    V *resp_s = reinterpret_cast<V *>(smem_raw + (PERSIST ? 2 : 1) * slot_bytes +
                                      (((size_t)2 * C * W * sizeof(T) + 15) & ~(size_t)15));
    load_resp<V, L>(prog, resp_s);
    if (t == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](long tile, int slot) {
        const int x0 = (int)(tile % tiles_x) * W;
        const int o = (int)(tile / tiles_x);
        uint64_t *bar = &bars[slot];
        mbar_arrive_expect_tx(bar, (uint32_t)((size_t)prog.ntiles * (nbox * box_n + (tma_halo ? 2 * kHalo : 0)) *
                                              W * sizeof(TI)));
        for (int ti = 0; ti < prog.ntiles; ++ti) {
            TI *tp = reinterpret_cast<TI *>(smem_raw + slot * slot_bytes + ti * tile_bytes) + kHalo * W;
            for (int b = 0; b < nbox; ++b) {
                if (dir == DY)
                    tma_load_3d(tp + (size_t)b * box_n * W, &maps.m[ti], bar, x0, b * box_n, o);
                else
                    tma_load_3d(tp + (size_t)b * box_n * W, &maps.m[ti], bar, x0, o, b * box_n);
            }
            if (tma_halo) {  // points n-4 .. n-1 before the line, 0 .. 3 after it
                TI *hb = tp - kHalo * W, *ha = tp + (size_t)n * W;
                if (dir == DY) {
                    tma_load_3d(hb, &maps.hm[ti], bar, x0, n - kHalo, o);
                    tma_load_3d(ha, &maps.hm[ti], bar, x0, 0, o);
                } else {
                    tma_load_3d(hb, &maps.hm[ti], bar, x0, o, n - kHalo);
                    tma_load_3d(ha, &maps.hm[ti], bar, x0, o, 0);
                }
            }
        }
        // the tile's base arrays (read back by the flushes) into L2
        for (int mask = prog.prefetch_mask, k = 0; mask; mask >>= 1, ++k) {
            if (!(mask & 1)) continue;
            for (int b = 0; b < nbox; ++b) {
                if (dir == DY) tma_prefetch_3d(&maps.pm[k], x0, b * box_n, o);
                else tma_prefetch_3d(&maps.pm[k], x0, o, b * box_n);
            }
        }
    };
    const ChunkScratch<V> sc = carve_scratch<V>(smem_raw + (PERSIST ? 2 : 1) * slot_bytes, C, WP);
    const int cs = c * L;
    const int nv = min(L, n - cs);
    const size_t ostride = dir == DY ? (size_t)nx : (size_t)nx * ny;
    long tile = blockIdx.x;
    if (t == 0) {
        if (PERSIST) s_tile[0] = tile = (long)atomicAdd(claim, 1ull);
        if (tile < ntiles) issue(tile, 0);
    }
    __syncthreads();
    if (PERSIST) tile = s_tile[0];
    for (int it = 0; tile < ntiles; ++it) {
        const int slot = PERSIST ? (it & 1) : 0;
        const uint32_t parity = PERSIST ? ((it >> 1) & 1) : 0;
        const bool ok = mbar_wait_bounded(&bars[slot], parity, kChunkWaitNs);
        // this barrier also ends every thread's reads of the other slot (the
        // previous tile), so the next tile's copies may go there now
        if (!__syncthreads_and(ok)) {
            if (t == 0) {
                atomicExch(err, 1);
                mbar_wait_bounded(&bars[slot], parity, kChunkWaitNs);
            }
            return;
        }
        if (PERSIST && t == 0) {
            const long next = (long)atomicAdd(claim, 1ull);
            s_tile[(it + 1) & 1] = next;  // read after this tile's operator barriers
            if (next < ntiles) issue(next, slot ^ 1);
        }
        const int x0 = (int)(tile % tiles_x) * W;
        const int o = (int)(tile / tiles_x);
        unsigned char *base = smem_raw + slot * slot_bytes;
        if (!tma_halo) {
            fill_halos_yz<TI>(base, tile_bytes, prog.ntiles, n, W, kHalo);
            fence_proxy_async_smem();  // the halo rows are refilled by TMA two tiles later
            __syncthreads();
        }
        // window of this chunk: rows kHalo + cs - 4 ...
        auto col = [&](int ti) {
            return reinterpret_cast<const TI *>(base + ti * tile_bytes) + (kHalo + cs - 4) * W + PR * l;
        };
        auto at = [](const TI *p) {
            if constexpr (std::is_same<TI, T>::value) return *reinterpret_cast<const V *>(p);
            else return V(*p);
        };
        auto tile_at = [&](int ti, int j) { return at(col(ti) + (4 + j) * W); };
        auto flush_args = [&](const StageOp<T> &so) {
            if constexpr (std::is_same<TI, T>::value)
                return FlushArgs<T>(so, so.base2_tile >= 0 ? col(so.base2_tile) + 4 * W : nullptr, W);
            else return FlushArgs<T>(so);
        };
        const bool live = x0 + PR * l < nx;
        const size_t obase = (size_t)(x0 + PR * l) + (dir == DY ? (size_t)nx * ny * o : (size_t)nx * o) +
                             (size_t)cs * ostride;
        V r[L];
        V acc[ACC ? L : 1];
        for (int k = 0; k < prog.nops; ++k) {
            const StageOp<T> &so = prog.ops[k];
            const TI *ca = col(so.src_a);
            const TI *cb = so.src_b >= 0 ? col(so.src_b) : nullptr;
            auto load = [&](auto &w, auto j0) {
                constexpr int J0 = decltype(j0)::value;
                constexpr int NW = sizeof(w) / sizeof(V);
                if (cb) {
#pragma unroll
                    for (int j = 0; j < NW; ++j) w[j] = at(ca + (J0 + j) * W) * at(cb + (J0 + j) * W);
                } else {
#pragma unroll
                    for (int j = 0; j < NW; ++j) w[j] = at(ca + (J0 + j) * W);
                }
            };
            constexpr bool trim = !ACC && (OCC == 1 || sizeof(T) == 4);  // FP64 at 80 registers would spill
            chunk_solve_resp<V, L, trim>(so.op, so.kind, resp_s + k * 4 * L, load, r, sc, WP, l, c, C, nv,
                                         c * WP + l, so.keep);
            if constexpr (ACC) {
                accumulate<V, L, 1>(so, acc, r, nv, tile_at);
                if (so.flush && live) flush_yz<T, V, L, true>(flush_args(so), acc, obase, ostride, nv);
            } else {
                if (so.flush && live) flush_yz<T, V, L, false>(flush_args(so), r, obase, ostride, nv);
            }
        }
        if (!PERSIST) break;
        // written by thread 0 before the operator barriers above; rewritten two
        // tiles later, after the next wait barrier, which every thread reaches
        // after reading it here
        tile = s_tile[(it + 1) & 1];
    }
}

// ---------------------------------------------------------------------------
// x-lines.

// General flush of an x chunk (contiguous from element p0) as 16-byte
// vectors of the output type U, in blocks of up to 8 points whose loads
// (base, base2, often the output arrays themselves) all precede their stores.
template <typename T, typename U, int L>
__device__ __forceinline__ void flush_x_blocked(const FlushArgs<T> &fa, const T (&res)[L], size_t p0, int nv)
{
    using UV = typename Vec4<U>::type;
    constexpr int VU = Vec4<U>::N;
    constexpr int B = L < 8 ? L : 8;
    constexpr int NQ = B / VU;
    const U *base = static_cast<const U *>(fa.base);
    const U *base2 = static_cast<const U *>(fa.base2);
    U *out = static_cast<U *>(fa.out);
    U *out2 = static_cast<U *>(fa.out2);
    const U sign = (U)fa.sign, scale2 = (U)fa.scale2;
#pragma unroll
    for (int j0 = 0; j0 < L; j0 += B) {
        UV bq[NQ], b2q[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int j = j0 + q * VU;
            const bool in = j < nv;
            bq[q] = base && in ? *reinterpret_cast<const UV *>(base + p0 + j) : UV{};
            if constexpr (std::is_same<T, U>::value) {
                if (fa.b2s) b2q[q] = *reinterpret_cast<const UV *>(fa.b2s + j);
                else b2q[q] = base2 && in ? *reinterpret_cast<const UV *>(base2 + p0 + j) : UV{};
            } else {
                b2q[q] = base2 && in ? *reinterpret_cast<const UV *>(base2 + p0 + j) : UV{};
            }
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int j = j0 + q * VU;
            if (j < nv) {
                UV o, o2;
                U *ov = reinterpret_cast<U *>(&o);
                U *o2v = reinterpret_cast<U *>(&o2);
                const U *bv = reinterpret_cast<const U *>(&bq[q]);
                const U *b2v = reinterpret_cast<const U *>(&b2q[q]);
#pragma unroll
                for (int e = 0; e < VU; ++e) {
                    ov[e] = bv[e] + sign * (U)res[j + e];
                    o2v[e] = b2v[e] + scale2 * ov[e];
                }
                *reinterpret_cast<UV *>(out + p0 + j) = o;
                if (out2) *reinterpret_cast<UV *>(out2 + p0 + j) = o2;
            }
        }
    }
}

// Writes one thread's solved chunk of an x line (points j < nv) as 16-byte
// vectors starting at element p0.
template <typename T, int L>
__device__ __forceinline__ void flush_x(const FlushArgs<T> &fa, const T (&res)[L], size_t p0, int nv)
{
    using VT = typename Vec4<T>::type;
    constexpr int V = Vec4<T>::N;
    if (fa.plain) {
        T *dst = static_cast<T *>(fa.out) + p0;
#pragma unroll
        for (int j = 0; j < L; j += V) {
            if (j < nv) {
                VT q;
                T *e = reinterpret_cast<T *>(&q);
#pragma unroll
                for (int v = 0; v < V; ++v) e[v] = res[j + v];
                *reinterpret_cast<VT *>(dst + j) = q;
            }
        }
        return;
    }
    if (fa.f64) flush_x_blocked<T, double, L>(fa, res, p0, nv);
    else flush_x_blocked<T, T, L>(fa, res, p0, nv);
}

// The general flush of a tile of x lines from its staging rows: the CTA's
// threads sweep the rows as 16-byte vectors, consecutive threads on
// consecutive vectors of a row, so the loads of base and base2 and the
// stores of out and out2 are coalesced across each warp (each thread's own
// chunk would touch a different line per vector).  A thread's vectors go in
// blocks of NB (2: the accumulator stays live across the flush, so more
// would spill) whose loads all precede their stores: base2 is often out2
// itself (u = u - p in place), so a load after a store could not move ahead
// of it and each vector would wait for memory in turn.  U = double writes
// FP64 outputs.
template <typename T, typename U>
__device__ __forceinline__ void flush_x_rows(const FlushArgs<T> &fa, const T *out_s, long l0, int rows,
                                             int pitch, int n)
{
    using VT = typename Vec4<T>::type;
    constexpr int V = Vec4<T>::N;
    using UV = typename Vec4<U>::type;
    constexpr int NU = V / Vec4<U>::N;  // U vectors per T vector
    constexpr int NB = 2;
    const U *base = static_cast<const U *>(fa.base);
    const U *base2 = static_cast<const U *>(fa.base2);
    U *out = static_cast<U *>(fa.out);
    U *out2 = static_cast<U *>(fa.out2);
    const U sign = (U)fa.sign, scale2 = (U)fa.scale2;
    // this thread's vectors: (row r0 + i * G, vector q) for i = 0, 1, ...
    const int per_row = n / V, nt = blockDim.x, t = threadIdx.x;
    int G, r0, q, qs;  // rows step, first row, vector, vector step
    if (nt >= per_row) {
        G = nt / per_row;
        r0 = t / per_row;
        q = t - r0 * per_row;
        qs = per_row;  // one vector per row
        if (r0 >= G) return;
    } else {
        G = 1;
        r0 = 0;
        q = t;
        qs = nt;
    }
    for (int rr0 = r0; rr0 < rows; rr0 += NB * G) {
        for (int q0 = q; q0 < per_row; q0 += qs) {
            UV b[NB][NU], b2[NB][NU];
#pragma unroll
            for (int i = 0; i < NB; ++i) {
                const int rr = rr0 + i * G;
                const size_t g = (size_t)(l0 + rr) * n + (size_t)q0 * V;
#pragma unroll
                for (int u = 0; u < NU; ++u) {
                    b[i][u] = base && rr < rows ? *reinterpret_cast<const UV *>(base + g + u * (V / NU)) : UV{};
                    b2[i][u] = base2 && rr < rows ? *reinterpret_cast<const UV *>(base2 + g + u * (V / NU)) : UV{};
                }
            }
#pragma unroll
            for (int i = 0; i < NB; ++i) {
                const int rr = rr0 + i * G;
                if (rr >= rows) break;
                const size_t g = (size_t)(l0 + rr) * n + (size_t)q0 * V;
                const VT v = *reinterpret_cast<const VT *>(out_s + (size_t)rr * pitch + (size_t)q0 * V);
                const T *vl = reinterpret_cast<const T *>(&v);
                const U *bl = reinterpret_cast<const U *>(b[i]);
                const U *b2l = reinterpret_cast<const U *>(b2[i]);
                UV o[NU], o2[NU];
                U *ol = reinterpret_cast<U *>(o);
                U *o2l = reinterpret_cast<U *>(o2);
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    ol[e] = bl[e] + sign * (U)vl[e];
                    o2l[e] = b2l[e] + scale2 * ol[e];
                }
#pragma unroll
                for (int u = 0; u < NU; ++u) {
                    *reinterpret_cast<UV *>(out + g + u * (V / NU)) = o[u];
                    if (out2) *reinterpret_cast<UV *>(out2 + g + u * (V / NU)) = o2[u];
                }
            }
        }
    }
}

// Flush of one operator for a tile of x lines.  Every thread first writes
// its chunk into the tile's staging rows (odd 16-byte granules per row, so
// the vector stores do not conflict).  A plain output then leaves as one
// bulk copy per row; any other (base, base2, FP64) is written by the whole
// CTA row by row (flush_x_rows).  A base2 that is a staged input (read from
// the tile, per thread) keeps the direct per-chunk flush.  The caller waits
// for the copies' reads before the staging rows are reused.  fa.plain and
// fa.b2s are the same for the whole CTA, so the barrier is uniform.
// GENERAL = false: the program's flushes are all plain, and the other forms
// are not compiled into the kernel.
template <typename T, int L, bool GENERAL>
__device__ __forceinline__ void flush_x_staged(const FlushArgs<T> &fa, const T (&res)[L], T *out_s, int l,
                                               long l0, int rows, int pitch, int n, int cs, int nv)
{
    using VT = typename Vec4<T>::type;
    constexpr int V = Vec4<T>::N;
    if constexpr (GENERAL) {
        if (fa.b2s) {
            if (l < rows) flush_x<T, L>(fa, res, (size_t)(l0 + l) * n + cs, nv);
            return;
        }
    }
    if (l < rows) {
        // the staging row is the tile's own: a short last chunk may write
        // past the line's end there (room for the last window), and the
        // row pass sends only the line's n points
        T *dst = out_s + (size_t)l * pitch + cs;
#pragma unroll
        for (int j = 0; j < L; j += V) {
            VT q;
            T *e = reinterpret_cast<T *>(&q);
#pragma unroll
            for (int v = 0; v < V; ++v) e[v] = res[j + v];
            *reinterpret_cast<VT *>(dst + j) = q;
        }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if constexpr (GENERAL) {
        if (!fa.plain) {
            if (fa.f64) flush_x_rows<T, double>(fa, out_s, l0, rows, pitch, n);
            else flush_x_rows<T, T>(fa, out_s, l0, rows, pitch, n);
            return;
        }
    }
    const int t = threadIdx.x;
    if (t < rows) {
        bulk_store(static_cast<T *>(fa.out) + (size_t)(l0 + t) * n, out_s + (size_t)t * pitch,
                   (uint32_t)(n * sizeof(T)));
        bulk_commit();
    }
}

// Fills the halos of ntiles staged x tiles of `rows` padded rows whose
// point i sits at element kHalo + i: elements 0 .. 3 from points n-4 .. n-1,
// elements n+4 .. n+7 from points 0 .. 3, moved as 16-byte vectors.
template <typename T>
__device__ __forceinline__ void fill_halos_x(unsigned char *base, size_t tile_bytes, int ntiles, int rows,
                                             int pitch, int n)
{
    using VT = typename Vec4<T>::type;
    constexpr int V = Vec4<T>::N;
    constexpr int per_row = 8 / V;
    const int per = rows * per_row;
    for (int i = threadIdx.x; i < per * ntiles; i += blockDim.x) {
        const int ti = i / per, r = i - ti * per;
        const int rr = r / per_row, h = (r - rr * per_row) * V;
        T *row = reinterpret_cast<T *>(base + ti * tile_bytes) + (size_t)rr * pitch;
        const int dst = h < 4 ? h : n + h;
        const int src = h < 4 ? n + h : h;
        *reinterpret_cast<VT *>(row + dst) = *reinterpret_cast<const VT *>(row + src);
    }
}

template <typename T, int W, int L, bool ACC, bool PERSIST, int OCC = 1>
__global__ void __launch_bounds__(OCC > 1 ? 256 : 512, OCC)
    ls_stage_x(const __grid_constant__ StageProgram<T> prog, long nlines, int pitch, size_t tile_bytes,
               long ntiles, unsigned long long *claim, int *err)
{
    using VT = typename Vec4<T>::type;
    constexpr int V = Vec4<T>::N;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bars[2];
    __shared__ long s_tile[2];  // persistent: tiles claimed in order, as ls_stage_yz does
    const int n = prog.ops[0].op.n;
    const int C = blockDim.x / W;
    const int t = threadIdx.x;
    const int l = t % W, c = t / W;
    const uint32_t row_bytes = (uint32_t)(n * sizeof(T));
    const size_t slot_bytes = (size_t)prog.ntiles * tile_bytes;
    T *resp_s = reinterpret_cast<T *>(smem_raw + (PERSIST ? 2 : 1) * slot_bytes +
                                      (((size_t)2 * C * W * sizeof(T) + 15) & ~(size_t)15));
    load_resp<T, L>(prog, resp_s);
    if (t == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](long tile, int slot) {
        const long l0 = tile * W;
        const int rows = (int)min((long)W, nlines - l0);
        uint64_t *bar = &bars[slot];
        mbar_arrive_expect_tx(bar, row_bytes * (uint32_t)rows * (uint32_t)prog.ntiles);
        for (int ti = 0; ti < prog.ntiles; ++ti) {
            T *tp = reinterpret_cast<T *>(smem_raw + slot * slot_bytes + ti * tile_bytes) + kHalo;
            for (int rr = 0; rr < rows; ++rr)
                bulk_load(tp + (size_t)rr * pitch, prog.in[ti] + (size_t)(l0 + rr) * n, row_bytes, bar);
        }
        // the tile's base rows (read back by the flushes) into L2
        for (int mask = prog.prefetch_mask, k = 0; mask; mask >>= 1, ++k)
            if (mask & 1)
                bulk_prefetch(static_cast<const T *>(prog.ops[k].base ? prog.ops[k].base : prog.ops[k].base2) +
                                  (size_t)l0 * n,
                              row_bytes * (uint32_t)rows);
    };
    const ChunkScratch<T> sc = carve_scratch<T>(smem_raw + (PERSIST ? 2 : 1) * slot_bytes, C, W);
    // staging rows for plain outputs, after the responses (128-byte aligned)
    T *out_s = reinterpret_cast<T *>(
        smem_raw + ((reinterpret_cast<unsigned char *>(resp_s + prog.nops * 4 * L) - smem_raw + 127) & ~(size_t)127));
    const int cs = c * L;
    const int nv = min(L, n - cs);
    long tile = blockIdx.x;
    if (t == 0) {
        if (PERSIST) s_tile[0] = tile = (long)atomicAdd(claim, 1ull);
        if (tile < ntiles) issue(tile, 0);
    }
    __syncthreads();
    if (PERSIST) tile = s_tile[0];
    for (int it = 0; tile < ntiles; ++it) {
        const int slot = PERSIST ? (it & 1) : 0;
        const uint32_t parity = PERSIST ? ((it >> 1) & 1) : 0;
        const bool ok = mbar_wait_bounded(&bars[slot], parity, kChunkWaitNs);
        // this barrier also ends every thread's reads of the other slot (the
        // previous tile), so the next tile's copies may go there now
        if (!__syncthreads_and(ok)) {
            if (t == 0) {
                atomicExch(err, 1);
                mbar_wait_bounded(&bars[slot], parity, kChunkWaitNs);
            }
            if (t < W) bulk_wait_all();
            return;
        }
        if (PERSIST && t == 0) {
            const long next = (long)atomicAdd(claim, 1ull);
            s_tile[(it + 1) & 1] = next;  // read after this tile's barriers
            if (next < ntiles) issue(next, slot ^ 1);
        }
        const long l0 = tile * W;
        const int rows = (int)min((long)W, nlines - l0);
        const int lr = l < rows ? l : 0;  // rows past the end compute on row 0 and store nothing
        unsigned char *base = smem_raw + slot * slot_bytes;
        fill_halos_x<T>(base, tile_bytes, prog.ntiles, rows, pitch, n);
        fence_proxy_async_smem();  // halo elements are refilled by bulk copies two tiles later
        __syncthreads();
        // window of this chunk: elements cs .. cs+L+7 (points cs-4 .. cs+L+3)
        auto row = [&](int ti) {
            return reinterpret_cast<const T *>(base + ti * tile_bytes) + (size_t)lr * pitch + cs;
        };
        auto tile_at = [&](int ti, int j) { return *reinterpret_cast<const VT *>(row(ti) + kHalo + j); };
        auto flush_args = [&](const StageOp<T> &so) {
            return FlushArgs<T>(so, so.base2_tile >= 0 ? row(so.base2_tile) + kHalo : nullptr, 1);
        };
        T r[L];
        T acc[ACC ? L : 1];
        for (int k = 0; k < prog.nops; ++k) {
            const StageOp<T> &so = prog.ops[k];
            const T *ra = row(so.src_a);
            const T *rb = so.src_b >= 0 ? row(so.src_b) : nullptr;
            auto load = [&](auto &w, auto j0) {
                constexpr int J0 = decltype(j0)::value;
                constexpr int NW = sizeof(w) / sizeof(T);
                if (rb) {
#pragma unroll
                    for (int j = 0; j < NW; j += V) {
                        const VT qa = *reinterpret_cast<const VT *>(ra + J0 + j);
                        const VT qb = *reinterpret_cast<const VT *>(rb + J0 + j);
                        const T *ea = reinterpret_cast<const T *>(&qa);
                        const T *eb = reinterpret_cast<const T *>(&qb);
#pragma unroll
                        for (int v = 0; v < V; ++v) w[j + v] = ea[v] * eb[v];
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < NW; j += V) {
                        const VT qa = *reinterpret_cast<const VT *>(ra + J0 + j);
                        const T *ea = reinterpret_cast<const T *>(&qa);
#pragma unroll
                        for (int v = 0; v < V; ++v) w[j + v] = ea[v];
                    }
                }
            };
            // the previous operator's row copies must have read the staging
            // rows before anyone writes them again (after this solve's barriers)
            if (t < W) bulk_wait_read_all();
            chunk_solve_resp<T, L, !ACC>(so.op, so.kind, resp_s + k * 4 * L, load, r, sc, W, l, c, C, nv, c * W + l,
                                         so.keep);
            if constexpr (ACC) {
                accumulate<T, L, V>(so, acc, r, nv, tile_at);
                if (so.flush) flush_x_staged<T, L, true>(flush_args(so), acc, out_s, l, l0, rows, pitch, n, cs, nv);
            } else {
                if (so.flush) flush_x_staged<T, L, false>(flush_args(so), r, out_s, l, l0, rows, pitch, n, cs, nv);
            }
        }
        if (!PERSIST) break;
        tile = s_tile[(it + 1) & 1];  // as in ls_stage_yz
    }
    if (t < W) bulk_wait_all();
}

// ---------------------------------------------------------------------------
// Host side.

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled()
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

struct StageOpView {
    short flush, accumulate, mul_tile;
};

static size_t scratch_bytes(int C, int W, size_t es) { return ((size_t)2 * C * W * es + 15) & ~(size_t)15; }

static bool al16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }
static bool al8(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 7) == 0; }

static bool plain(const StageOpView &v) { return v.flush && !v.accumulate && v.mul_tile < 0; }

template <typename Kern>
static unsigned persistent_grid(x3d_ctx_s *ctx, Kern kern, int threads, size_t smem, long ntiles)
{
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    const long g = (long)ctx->num_sms * (per_sm < 1 ? 1 : per_sm);
    return (unsigned)(g < ntiles ? g : ntiles);
}

// Carry responses of chunk_solve_resp for chunk length L on lines of n
// points: h_j = rho^(j+1) sum_{i < len-j} rho^(2i) and g_j = rho^(len-j),
// len = L (resp[0..1]) and len = the last chunk's length (resp[2..3]).
// Returns chunk_solve_resp's keep for full chunks: nh | ng << 8, the counts
// of leading h and trailing g entries above 2^-32 (FP32) or 2^-62 (FP64) of
// the largest, rounded up to whole blocks of 8.
template <typename T>
static int fill_op_resp(T (&resp)[4][kChunkLong<T>], double al, int L, int n)
{
    const int C = (n + L - 1) / L, last = n - (C - 1) * L;
    const double rho = al == 0.0 ? 0.0 : -2.0 * al / (1.0 + std::sqrt(1.0 - 4.0 * al * al));
    double pw[kChunkLong<T>];
    double q = 1.0;
    for (int j = 0; j < kChunkLong<T>; ++j) pw[j] = (q *= rho);  // rho^(j+1)
    auto fill = [&](T *h, T *g, int len) {
        double S = 0.0, G = 1.0;
        for (int j = kChunkLong<T> - 1; j >= 0; --j) {
            if (j >= len) {
                h[j] = g[j] = T(0);
                continue;
            }
            S = 1.0 + rho * rho * S;
            G *= rho;
            h[j] = (T)(pw[j] * S);
            g[j] = (T)G;
        }
    };
    fill(resp[0], resp[1], L);
    fill(resp[2], resp[3], last);
    const double thr = sizeof(T) == 4 ? std::ldexp(1.0, -32) : std::ldexp(1.0, -62);
    double hmax = 0.0, gmax = 0.0;
    for (int j = 0; j < L; ++j) {
        hmax = std::max(hmax, std::fabs((double)resp[0][j]));
        gmax = std::max(gmax, std::fabs((double)resp[1][j]));
    }
    int nh = 0, ng = 0;
    for (int j = 0; j < L; ++j)
        if (std::fabs((double)resp[0][j]) > thr * hmax) nh = j + 1;
    for (int j = L - 1; j >= 0; --j)
        if (std::fabs((double)resp[1][j]) > thr * gmax) ng = L - j;
    const int b = L < 8 ? L : 8;
    nh = std::min(L, (nh + b - 1) / b * b);
    ng = std::min(L, (ng + b - 1) / b * b);
    return nh | ng << 8;
}

template <typename T>
static void fill_resp(StageProgram<T> &p, int L, int n)
{
    for (int k = 0; k < p.nops; ++k) p.ops[k].keep = fill_op_resp(p.ops[k].resp, p.ops[k].op.alfa, L, n);
}

// PR = 2: the paired y/z kernel (FP32 only).  OCC > 1: the y/z kernel built
// for OCC CTAs per SM (plain programs, at most 256 threads).  Persistent
// kernels claim their tiles from the context's counter, zeroed here before
// each launch.
template <typename T, int W, int L, bool PERSIST, int PR = 1, int OCC = 1>
static int launch_stage_cfg(x3d_ctx_s *ctx, const StageProgram<T> &prog_in, int dir, int nx, int ny,
                            int nz)
{
    if constexpr (PR == 2 && !std::is_same<T, float>::value) {
        return X3D_EUNSUPPORTED;
    } else {
        StageProgram<T> prog = prog_in;
        fill_resp(prog, L, prog.ops[0].op.n);
        // base2 that is a staged input comes from shared memory; T-typed bases
        // are prefetched into L2 with the tile's inputs
        for (int k = 0; k < prog.nops; ++k) {
            StageOp<T> &so = prog.ops[k];
            so.base2_tile = -1;
            for (int ti = 0; ti < prog.ntiles; ++ti)
                if (!so.out_f64 && so.base2 && so.base2 == prog.in[ti]) so.base2_tile = (short)ti;
            so.prefetch_base = (so.flush && !so.out_f64 && (so.base || (so.base2 && so.base2_tile < 0))) ? 1 : 0;
        }
        prog.prefetch_mask = 0;
        for (int k = 0; k < prog.nops; ++k)
            if (prog.ops[k].prefetch_base) prog.prefetch_mask |= 1 << k;
        // the ACC kernels carry the accumulator and every flush form; the
        // others only plain operators (out = the solve)
        bool acc = false;
        for (int k = 0; k < prog.nops; ++k) {
            const StageOp<T> &so = prog.ops[k];
            acc = acc || !plain(StageOpView{so.flush, so.accumulate, so.mul_tile}) ||
                  (so.flush && (so.base || so.out2 || so.out_f64 || so.sign != 1.0));
        }
        const int n = prog.ops[0].op.n;
        for (int k = 0; k < prog.nops; ++k)
            if (!prog.ops[k].op.circ || prog.ops[k].op.n != n) return X3D_EUNSUPPORTED;
        const size_t es = sizeof(T);
        const int C = (n + L - 1) / L;
        const int threads = C * W / PR;
        if (threads > kStageThreads<T, L, PR> || threads % 32) return X3D_EUNSUPPORTED;
        if (OCC > 1 && (acc || threads > 256)) return X3D_EUNSUPPORTED;
        // FP64 inputs of an FP32 program: staged as FP64 by the plain,
        // unpaired y/z kernels only
        const bool in64 = prog.in_f64 != 0;
        if (in64 && (!std::is_same<T, float>::value || PR != 1 || OCC != 1 || acc || dir == DX))
            return X3D_EUNSUPPORTED;
        const size_t resp_bytes = (size_t)prog.nops * 4 * L * es * PR;
        for (int ti = 0; ti < prog.ntiles; ++ti)
            if (!al16(prog.in[ti])) return X3D_EUNSUPPORTED;
        cudaStream_t st = ctx->stream;
        if constexpr (PR == 2) {
            // paired y/z lines: even x extent, 8-byte aligned pair stores
            if (dir == DX || nx % 2) return X3D_EUNSUPPORTED;
            for (int k = 0; k < prog.nops; ++k) {
                const StageOp<T> &so = prog.ops[k];
                if (so.flush && (!al8(so.out) || !al8(so.base) || !al8(so.out2) || !al8(so.base2)))
                    return X3D_EUNSUPPORTED;
            }
        } else if (dir == DX) {
            constexpr int V = Vec4<T>::N;
            if (n % V) return X3D_EUNSUPPORTED;
            for (int k = 0; k < prog.nops; ++k) {
                const StageOp<T> &so = prog.ops[k];
                if (so.flush && (!al16(so.out) || !al16(so.base) || !al16(so.out2) || !al16(so.base2)))
                    return X3D_EUNSUPPORTED;
            }
            // row: kHalo halo elements, the line, and room for the last chunk's window
            int pitch = C * L + 2 * kHalo;
            while (((size_t)pitch * es / 16) % 2 == 0) pitch += V;
            const size_t tile = ((size_t)W * pitch * es + 127) & ~(size_t)127;
            // + staging rows for plain outputs (W rows of the same pitch, 128-byte aligned)
            const size_t smem = (((PERSIST ? 2 : 1) * prog.ntiles * tile + scratch_bytes(C, W, es) + resp_bytes + 127) &
                                 ~(size_t)127) +
                                (size_t)W * pitch * es;
            if (smem + 1024 > ctx->smem_optin) return X3D_EUNSUPPORTED;
            auto kern = ls_stage_x<T, W, L, false, PERSIST, OCC>;
            if constexpr (OCC == 1)  // the OCC > 1 kernels take plain programs only
                if (acc) kern = ls_stage_x<T, W, L, true, PERSIST>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            const long nlines = (long)ny * nz;
            const long ntiles = (nlines + W - 1) / W;
            const unsigned grid = PERSIST ? persistent_grid(ctx, kern, threads, smem, ntiles) : (unsigned)ntiles;
            if (PERSIST) {
                const int rc = cuda_check(ctx, cudaMemsetAsync(ctx->d_claim, 0, sizeof(*ctx->d_claim), st),
                                          "tile counter reset");
                if (rc) return rc;
            }
            ++ctx->launches;
            kern<<<grid, threads, smem, st>>>(prog, nlines, pitch, tile, ntiles, ctx->d_claim, ctx->d_err);
            return cuda_check(ctx, cudaGetLastError(), "ls_stage_x launch");
        }
        auto enc = encode_tiled();
        const size_t esi = in64 ? sizeof(double) : es;  // staged element bytes
        if (!enc || ((size_t)nx * esi) % 16) return X3D_EUNSUPPORTED;
        const int nb = (n + 255) / 256;
        int box_n = (n + nb - 1) / nb;
        const int align_rows = (int)(128 / (W * esi) > 0 ? 128 / (W * esi) : 1);
        box_n = (box_n + align_rows - 1) / align_rows * align_rows;
        if (box_n > 256) return X3D_EUNSUPPORTED;
        // rows: kHalo halo rows (kHalo * W * esi is a multiple of 128 bytes, so the
        // boxes land 128-byte aligned), the boxes, and room for the last window
        const int rows = kHalo + std::max(nb * box_n, C * L + kHalo);
        const size_t tile = ((size_t)rows * W * esi + 127) & ~(size_t)127;
        const size_t smem = (PERSIST ? 2 : 1) * prog.ntiles * tile + scratch_bytes(C, W, es) + resp_bytes;
        if (smem + 1024 > ctx->smem_optin) return X3D_EUNSUPPORTED;
        StageMaps maps;
        std::memset(&maps, 0, sizeof(maps));
        auto encode = [&](CUtensorMap *m, const void *ptr, int rows_in_box, size_t eb) {
            cuuint64_t gdim[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
            cuuint64_t gstride[2] = {(cuuint64_t)nx * eb, (cuuint64_t)nx * ny * eb};
            cuuint32_t box[3] = {(cuuint32_t)W, 1, 1};
            box[dir == DY ? 1 : 2] = (cuuint32_t)rows_in_box;
            cuuint32_t estr[3] = {1, 1, 1};
            return enc(m, eb == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                       const_cast<void *>(ptr), gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                       CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
        };
        for (int ti = 0; ti < prog.ntiles; ++ti)
            if (!encode(&maps.m[ti], prog.in[ti], box_n, esi)) return X3D_EUNSUPPORTED;
        // the periodic halos come by TMA too where the boxes end exactly at the
        // line's end (a box running past it would fill the rows after the line
        // with zeros); otherwise the kernel copies them in shared memory
        int tma_halo = nb * box_n == n ? 1 : 0;
        for (int ti = 0; ti < prog.ntiles && tma_halo; ++ti)
            if (!encode(&maps.hm[ti], prog.in[ti], kHalo, esi)) tma_halo = 0;
        for (int k = 0; k < prog.nops; ++k)
            if (prog.ops[k].prefetch_base &&
                !encode(&maps.pm[k], prog.ops[k].base ? prog.ops[k].base : prog.ops[k].base2, box_n, es))
                prog.ops[k].prefetch_base = 0;
        prog.prefetch_mask = 0;
        for (int k = 0; k < prog.nops; ++k)
            if (prog.ops[k].prefetch_base) prog.prefetch_mask |= 1 << k;
        auto kern = ls_stage_yz<T, W, L, false, PERSIST, PR, OCC>;
        if constexpr (OCC == 1)  // the OCC > 1 kernels take plain programs only
            if (acc) kern = ls_stage_yz<T, W, L, true, PERSIST, PR, OCC>;
        if constexpr (std::is_same<T, float>::value && PR == 1 && OCC == 1)
            if (in64) kern = ls_stage_yz<T, W, L, false, PERSIST, PR, OCC, double>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        const long tiles_x = (nx + W - 1) / W;
        const long ntiles = tiles_x * (dir == DY ? nz : ny);
        const unsigned grid = PERSIST ? persistent_grid(ctx, kern, threads, smem, ntiles) : (unsigned)ntiles;
        if (PERSIST) {
            const int rc = cuda_check(ctx, cudaMemsetAsync(ctx->d_claim, 0, sizeof(*ctx->d_claim), st),
                                      "tile counter reset");
            if (rc) return rc;
        }
        ++ctx->launches;
        kern<<<grid, threads, smem, st>>>(maps, prog, nx, ny, dir, box_n, nb, tma_halo, tile, ntiles, ctx->d_claim,
                                          ctx->d_err);
        return cuda_check(ctx, cudaGetLastError(), "ls_stage_yz launch");

    }
}

template <typename T>
static int launch_stage_sel(x3d_ctx_s *ctx, const StageProgram<T> &prog, int dir, int nx, int ny, int nz, int cfg);

template <typename T>
int launch_stage(x3d_ctx_s *ctx, const StageProgram<T> &prog, int dir, int nx, int ny, int nz, int cfg)
{
    const int rc = launch_stage_sel<T>(ctx, prog, dir, nx, ny, nz, cfg);
    if (rc == X3D_OK) ctx->last_cfg = cfg;
    return rc;
}

template <typename T>
static int launch_stage_sel(x3d_ctx_s *ctx, const StageProgram<T> &prog, int dir, int nx, int ny, int nz, int cfg)
{
    if (prog.nops < 1 || prog.nops > kMaxStageOps || prog.ntiles < 1 || prog.ntiles > kMaxStageTiles)
        return X3D_EINVAL;
    // cfg selects (lines per CTA, chunk length).
    constexpr int Lbig = sizeof(T) == 4 ? 32 : 16;
    constexpr int Lsmall = sizeof(T) == 4 ? 16 : 8;
    // 0-5: one CTA per tile; 6-11: the same shapes, persistent with two slots
    switch (cfg) {
    case 0: return launch_stage_cfg<T, 16, Lbig, false>(ctx, prog, dir, nx, ny, nz);
    case 1: return launch_stage_cfg<T, 32, Lbig, false>(ctx, prog, dir, nx, ny, nz);
    case 2: return launch_stage_cfg<T, 16, Lsmall, false>(ctx, prog, dir, nx, ny, nz);
    case 3: return launch_stage_cfg<T, 8, Lbig, false>(ctx, prog, dir, nx, ny, nz);
    case 4: return launch_stage_cfg<T, 32, Lsmall, false>(ctx, prog, dir, nx, ny, nz);
    case 5: return launch_stage_cfg<T, 8, Lsmall, false>(ctx, prog, dir, nx, ny, nz);
    case 6: return launch_stage_cfg<T, 16, Lbig, true>(ctx, prog, dir, nx, ny, nz);
    case 7: return launch_stage_cfg<T, 32, Lbig, true>(ctx, prog, dir, nx, ny, nz);
    case 8: return launch_stage_cfg<T, 16, Lsmall, true>(ctx, prog, dir, nx, ny, nz);
    case 9: return launch_stage_cfg<T, 8, Lbig, true>(ctx, prog, dir, nx, ny, nz);
    case 10: return launch_stage_cfg<T, 32, Lsmall, true>(ctx, prog, dir, nx, ny, nz);
    case 11: return launch_stage_cfg<T, 8, Lsmall, true>(ctx, prog, dir, nx, ny, nz);
    // 12-15: y/z lines in packed pairs (FP32, even nx)
    case 12: return launch_stage_cfg<T, 32, Lsmall, true, 2>(ctx, prog, dir, nx, ny, nz);
    case 13: return launch_stage_cfg<T, 16, Lsmall, true, 2>(ctx, prog, dir, nx, ny, nz);
    case 14: return launch_stage_cfg<T, 32, Lsmall, false, 2>(ctx, prog, dir, nx, ny, nz);
    case 15: return launch_stage_cfg<T, 32, Lbig, true, 2>(ctx, prog, dir, nx, ny, nz);
    // 17: configuration 6 (y/z) compiled for three CTAs per SM (plain programs)
    case 17: return launch_stage_cfg<T, 16, Lbig, true, 1, 3>(ctx, prog, dir, nx, ny, nz);
    // 18: configuration 9 (8 lines, long chunks, y/z) built for three CTAs per SM
    case 18: return launch_stage_cfg<T, 8, Lbig, true, 1, 3>(ctx, prog, dir, nx, ny, nz);
    // 19: configuration 3 (8 lines, long chunks, one CTA per tile) built for
    // three CTAs per SM: with one staging slot the FP64 x tiles fit three
    case 19: return launch_stage_cfg<T, 8, Lbig, false, 1, 3>(ctx, prog, dir, nx, ny, nz);
    // 20: configuration 0 (16 lines, long chunks, one CTA per tile) built for
    // three CTAs per SM
    case 20: return launch_stage_cfg<T, 16, Lbig, false, 1, 3>(ctx, prog, dir, nx, ny, nz);
    default: return X3D_EUNSUPPORTED;
    }
}

template <typename T>
StageProgram<T> plain_program(const T *in, const LineOp<T> *const *ops, const int *kinds,
                              void *const *outs, int nops)
{
    StageProgram<T> p{};
    p.nops = nops;
    p.ntiles = 1;
    p.in[0] = in;
    for (int k = 0; k < nops; ++k) {
        StageOp<T> &so = p.ops[k];
        so.op = *ops[k];
        so.kind = kinds[k];
        so.src_a = 0;
        so.src_b = -1;
        so.mul_tile = -1;
        so.accumulate = 0;
        so.flush = 1;
        so.out = outs[k];
        so.base = nullptr;
        so.out2 = nullptr;
        so.base2 = nullptr;
        so.sign = 1.0;
        so.scale2 = 0.0;
        so.out_f64 = 0;
    }
    return p;
}

// ---------------------------------------------------------------------------
// Batches of uneven boxes: one persistent launch applies the operator groups
// of every (box, field, direction) job.  CTAs pull tiles from a global
// counter, so boxes of different sizes balance across the SMs; each tile
// uses its job's lines per tile (W), chunk count (C), tensor map or padded
// rows.  Threads beyond W*C of a job idle through its barriers.
// Carry scratch, then the carry responses of the item's operators.
template <typename T>
constexpr size_t batch_scratch_bytes_c()
{
    return (((size_t)2 * kBatchThreads * sizeof(T) + 15) & ~(size_t)15) +
           (size_t)kMaxStageOps * 4 * kChunkLong<T> * sizeof(T);
}

// Byte offset of the x staging rows: after the two slots, the scratch and
// the responses, 128-byte aligned.
template <typename T>
__host__ __device__ constexpr size_t batch_out_offset(size_t tile_cap)
{
    return (2 * tile_cap + batch_scratch_bytes_c<T>() + 127) & ~(size_t)127;
}

// One work item of the batch kernel with chunk length L (the job's): the
// operators of the job solved over the staged tile and written out.  y/z
// outputs go straight to global memory, coalesced across the tile's lines;
// x outputs either go straight out as each thread's 16-byte vectors or, for
// jobs with xstage set, are staged in shared-memory rows (out_s, the tile's
// pitch) and leave as one bulk copy per row, as in ls_stage_x.
template <typename T, int L, bool XS>
__device__ __forceinline__ void batch_item(const BatchJob<T> &J, const T *tile, T *out_s, const T *resp_s,
                                           const ChunkScratch<T> &scf, int t, long l0, int rows, int x0, int o)
{
    using VT = typename Vec4<T>::type;
    constexpr int V = Vec4<T>::N;
    const int W = J.W, C = J.C, n = J.n;
    const int dir = J.dir;
    const bool active = t < W * C;
    const int l = active ? t % W : 0, c = active ? t / W : 0;
    const int q = t;  // scratch slot: active threads use c*W + l == t
    ChunkScratch<T> sc = scf;
    const int cs = c * L;
    const int nv = min(L, n - cs);
    T r[L];
    if (dir == DX) {
        const int lr = l < rows ? l : 0;
        const T *row = tile + (size_t)lr * J.pitch + cs;  // points cs-4 .. cs+L+3
        auto load = [&](auto &w, auto j0) {
            constexpr int J0 = decltype(j0)::value;
            constexpr int NW = sizeof(w) / sizeof(T);
#pragma unroll
            for (int j = 0; j < NW; j += V) {
                const VT qa = *reinterpret_cast<const VT *>(row + J0 + j);
                const T *ea = reinterpret_cast<const T *>(&qa);
#pragma unroll
                for (int v = 0; v < V; ++v) w[j + v] = ea[v];
            }
        };
        for (int k = 0; k < J.nops; ++k) {
            // the previous operator's row copies have read the staging
            // rows before anyone writes them again (after this solve's barriers)
            if (XS) bulk_wait_read_all();
            chunk_solve_resp<T, L, true>(J.op[k], J.kind[k], resp_s + k * 4 * L, load, r, sc, W, l, c, C, nv,
                                         q, J.keep[k]);
            if (!XS || !J.xstage) {  // each thread's chunk straight out, 16 bytes at a time
                if (active && l < rows) {
                    T *dst = J.out[k] + (size_t)(l0 + l) * n + cs;
#pragma unroll
                    for (int j = 0; j < L; j += V) {
                        if (j < nv) {
                            VT qv;
                            T *e = reinterpret_cast<T *>(&qv);
#pragma unroll
                            for (int v = 0; v < V; ++v) e[v] = r[j + v];
                            *reinterpret_cast<VT *>(dst + j) = qv;
                        }
                    }
                }
                continue;
            }
            if (active && l < rows) {
                T *dst = out_s + (size_t)l * J.pitch + cs;  // room for the last window past n
#pragma unroll
                for (int j = 0; j < L; j += V) {
                    VT qv;
                    T *e = reinterpret_cast<T *>(&qv);
#pragma unroll
                    for (int v = 0; v < V; ++v) e[v] = r[j + v];
                    *reinterpret_cast<VT *>(dst + j) = qv;
                }
            }
            fence_proxy_async_smem();
            __syncthreads();
            if (t < rows) {
                bulk_store(J.out[k] + (size_t)(l0 + t) * n, out_s + (size_t)t * J.pitch,
                           (uint32_t)(n * sizeof(T)));
                bulk_commit();
            }
        }
    } else {
        const T *col = tile + (size_t)(J.halo + cs - 4) * W + l;  // points cs-4 .. cs+L+3
        auto load = [&](auto &w, auto j0) {
            constexpr int J0 = decltype(j0)::value;
            constexpr int NW = sizeof(w) / sizeof(T);
#pragma unroll
            for (int j = 0; j < NW; ++j) w[j] = col[(J0 + j) * W];
        };
        const bool live = active && x0 + l < J.nx;
        const size_t ostride = dir == DY ? (size_t)J.nx : (size_t)J.nx * J.ny;
        const size_t obase = (size_t)(x0 + l) +
                             (dir == DY ? (size_t)J.nx * J.ny * o : (size_t)J.nx * o) +
                             (size_t)cs * ostride;
        for (int k = 0; k < J.nops; ++k) {
            chunk_solve_resp<T, L, true>(J.op[k], J.kind[k], resp_s + k * 4 * L, load, r, sc, W, l, c, C, nv,
                                         q, J.keep[k]);
            if (live) {
                T *dst = J.out[k] + obase;
                if (nv == L) {  // every chunk but a short last one: no per-point test
#pragma unroll
                    for (int j = 0; j < L; ++j) {
                        *dst = r[j];
                        dst += ostride;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < L; ++j) {
                        if (j < nv) *dst = r[j];
                        dst += ostride;
                    }
                }
            }
        }
    }
}

// VAR (BatchVariant): kBatchLong runs every job with the long chunk and
// its x outputs straight out; kBatchMixed takes each job's chunk length;
// kBatchStaged also stages the x outputs of jobs with xstage set.  The
// narrower variants carry less code and no staging rows.
// Bytes of a job's header (every field before its responses), in 16-byte units.
template <typename T>
constexpr int kBatchHdrVecs = (int)((offsetof(BatchJob<T>, resp) + 15) / 16);

template <typename T, int VAR>
__global__ void __launch_bounds__(kBatchThreads, 2)
    ls_batch(const BatchJob<T> *__restrict__ jobs, int njobs, long total,
             unsigned long long *counter, size_t tile_cap, int *err)
{
    static_assert(kBatchHdrVecs<T> <= kBatchThreads, "one 16-byte copy per thread");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bars[2];
    __shared__ long s_item;
    __shared__ int s_job;  // the job of s_item
    // the headers of the current and the next item's jobs, by iteration parity
    __shared__ __align__(64) uint4 s_hdr[2][kBatchHdrVecs<T>];
    const int t = threadIdx.x;
    // two staging slots of tile_cap bytes, then the carry scratch and the
    // carry responses of the item's operators
    const ChunkScratch<T> scf = carve_scratch<T>(smem_raw + 2 * tile_cap, kBatchThreads / 1, 1);
    T *resp_s = reinterpret_cast<T *>(smem_raw + 2 * tile_cap +
                                      (((size_t)2 * kBatchThreads * sizeof(T) + 15) & ~(size_t)15));
    // staging rows of x outputs (one tile's worth), after the responses
    T *out_s = reinterpret_cast<T *>(smem_raw + batch_out_offset<T>(tile_cap));
    auto job_of = [&](long item) {
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].tile0 <= item) lo = mid;
            else hi = mid - 1;
        }
        return lo;
    };
    // The copies of one work item of job jb into staging slot `slot` (one thread).
    auto issue = [&](long item, int jb, int slot) {
        const BatchJob<T> &J = jobs[jb];
        const long tl = item - J.tile0;
        T *tile = reinterpret_cast<T *>(smem_raw + slot * tile_cap);
        uint64_t *bar = &bars[slot];
        if (J.dir == DX) {
            const long l0 = tl * J.W;
            const int rows = (int)min((long)J.W, J.span - l0);
            const uint32_t row_bytes = (uint32_t)(J.n * sizeof(T));
            mbar_arrive_expect_tx(bar, row_bytes * (uint32_t)rows);
            for (int rr = 0; rr < rows; ++rr)
                bulk_load(tile + (size_t)rr * J.pitch + kHalo, J.in + (size_t)(l0 + rr) * J.n, row_bytes, bar);
        } else {
            const int x0 = (int)(tl % J.span) * J.W, o = (int)(tl / J.span);
            fence_tensormap_acquire(&J.tmap);
            mbar_arrive_expect_tx(bar, (uint32_t)((size_t)J.nbox * J.box_n * J.W * sizeof(T)));
            T *dst = tile + (size_t)J.halo * J.W;
            for (int b = 0; b < J.nbox; ++b) {
                if (J.dir == DY)
                    tma_load_3d(dst + (size_t)b * J.box_n * J.W, &J.tmap, bar, x0, b * J.box_n, o);
                else
                    tma_load_3d(dst + (size_t)b * J.box_n * J.W, &J.tmap, bar, x0, o, b * J.box_n);
            }
        }
    };
    // every thread copies at most one 16-byte piece of job jb's header
    auto copy_header = [&](int jb, int hs) {
        if (t < kBatchHdrVecs<T>) s_hdr[hs][t] = reinterpret_cast<const uint4 *>(jobs + jb)[t];
    };
    if (t == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
        s_item = (long)atomicAdd(counter, 1ull);
        if (s_item < total) {
            s_job = job_of(s_item);
            issue(s_item, s_job, 0);
        }
    }
    __syncthreads();
    if (s_item < total) copy_header(s_job, 0);
    uint32_t phases = 0;  // bit s: parity of slot s's next completion
    int resp_have = -1;   // the response class in resp_s (the same in every thread)
    for (int it = 0;; ++it) {
        const int slot = it & 1;
        const long item = s_item;  // claimed during the previous item (or above)
        if (item >= total) break;
        const int jb = s_job;
        unsigned char *tbase = smem_raw + slot * tile_cap;
        const T *tile = reinterpret_cast<const T *>(tbase);
        const uint32_t parity = (phases >> slot) & 1u;
        const bool ok = mbar_wait_bounded(&bars[slot], parity, kChunkWaitNs);
        if (!__syncthreads_and(ok)) {
            if (t == 0) atomicExch(err, 1);
            mbar_wait_bounded(&bars[slot], parity, kChunkWaitNs);
            if (VAR == kBatchStaged) bulk_wait_all();
            return;
        }
        phases ^= 1u << slot;
        // The job's header, copied during the previous item (or above) and
        // ordered by the barrier just passed.  Every thread is done with the
        // previous item (its responses are read after its last barrier, its
        // tile and header before): this item's responses go in place, and the
        // next item, claimed now, is copied into the other slot while this
        // one is solved.
        const BatchJob<T> &J = *reinterpret_cast<const BatchJob<T> *>(s_hdr[slot]);
        const long tl = item - J.tile0;
        const int W = J.W, n = J.n;
        const int dir = J.dir;
        long l0 = 0;
        int rows = W, x0 = 0, o = 0;
        if (dir == DX) {
            l0 = tl * W;
            rows = (int)min((long)W, J.span - l0);
        } else {
            x0 = (int)(tl % J.span) * W;
            o = (int)(tl / J.span);
        }
        const int L = VAR == kBatchLong ? kChunkLong<T> : J.L;
        if (J.rclass != resp_have) {  // consecutive items mostly share a job, so this is rare
            const T *resp_g = &jobs[jb].resp[0][0][0];
            for (int i = t; i < J.nops * 4 * L; i += kBatchThreads) {
                const int k = i / (4 * L), rem = i - k * 4 * L, a = rem / L, j = rem - a * L;
                resp_s[i] = resp_g[(k * 4 + a) * kChunkLong<T> + j];
            }
            resp_have = J.rclass;
        }
        if (t == 0) {
            const long next = (long)atomicAdd(counter, 1ull);
            s_item = next;
            if (next < total) {
                const int nj = job_of(next);
                s_job = nj;
                issue(next, nj, slot ^ 1);
            }
        }
        if (dir == DX) fill_halos_x<T>(tbase, 0, 1, rows, J.pitch, n);
        else fill_halos_yz<T>(tbase, 0, 1, n, W, J.halo);
        fence_proxy_async_smem();  // copies into this slot two items later overwrite the halos
        __syncthreads();
        // the next item's header into the other slot, read after the next wait barrier
        if (s_item < total) copy_header(s_job, slot ^ 1);
        constexpr bool XS = VAR == kBatchStaged;
        if (VAR == kBatchLong || J.L == kChunkLong<T>)
            batch_item<T, kChunkLong<T>, XS>(J, tile, out_s, resp_s, scf, t, l0, rows, x0, o);
        else
            batch_item<T, kChunkShort<T>, XS>(J, tile, out_s, resp_s, scf, t, l0, rows, x0, o);
    }
    if (VAR == kBatchStaged) bulk_wait_all();  // x rows in flight (issued by this thread)
}


static int gcd_int(int a, int b) { return b ? gcd_int(b, a % b) : a; }

// Fills the geometry, tiling and staging fields of a job; false when the
// job's box cannot take the chunked batch kernel.
template <typename T>
bool plan_batch_job(BatchJob<T> &J, int L, int w_req, int xstage, size_t *tile_bytes)
{
    const size_t es = sizeof(T);
    const int n = J.n;
    constexpr int V = Vec4<T>::N;
    if (L != kChunkLong<T> && L != kChunkShort<T>) return false;
    for (int k = 0; k < J.nops; ++k)
        if (!J.op[k].circ || J.op[k].n != n) return false;
    for (int k = 0; k < J.nops; ++k) J.keep[k] = fill_op_resp(J.resp[k], J.op[k].alfa, L, n);
    J.L = L;
    J.C = (n + L - 1) / L;
    if (J.C > kBatchThreads) return false;
    int W = kBatchThreads / J.C;
    if (w_req > 0) W = std::min(W, w_req);
    const int wq = (int)(16 / es);  // TMA inner extent: multiple of 16 bytes
    W = std::max(wq, W / wq * wq);
    if (W * J.C > kBatchThreads || W > 256) return false;
    J.W = W;
    if (J.dir == DX) {
        if (n % V || (reinterpret_cast<uintptr_t>(J.in) & 15)) return false;
        // staged outputs leave as bulk row copies: 16-byte aligned rows
        J.xstage = xstage ? 1 : 0;
        for (int k = 0; k < J.nops && J.xstage; ++k)
            if (reinterpret_cast<uintptr_t>(J.out[k]) & 15) J.xstage = 0;
        int pitch = J.C * L + 2 * kHalo;
        while (((size_t)pitch * es / 16) % 2 == 0) pitch += V;
        J.pitch = pitch;
        J.span = (long)J.ny * J.nz;
        J.ntiles = (J.span + W - 1) / W;
        *tile_bytes = ((size_t)W * pitch * es + 127) & ~(size_t)127;
        return true;
    }
    if (((size_t)J.nx * es) % 16) return false;
    const int nb = (n + 255) / 256;
    int box_n = (n + nb - 1) / nb;
    const int align_rows = 128 / gcd_int(128, (int)(W * es));
    box_n = (box_n + align_rows - 1) / align_rows * align_rows;
    if (box_n > 256) return false;
    J.box_n = box_n;
    J.nbox = nb;
    J.span = (J.nx + W - 1) / W;
    J.ntiles = J.span * (J.dir == DY ? J.nz : J.ny);
    // halo rows in front of the boxes: at least kHalo, keeping the boxes
    // 128-byte aligned
    J.halo = kHalo;
    while (((size_t)J.halo * W * es) % 128) ++J.halo;
    const int rows = J.halo + std::max(nb * box_n, J.C * L + kHalo);
    *tile_bytes = ((size_t)rows * W * es + 127) & ~(size_t)127;
    auto enc = encode_tiled();
    if (!enc) return false;
    cuuint64_t gdim[3] = {(cuuint64_t)J.nx, (cuuint64_t)J.ny, (cuuint64_t)J.nz};
    cuuint64_t gstride[2] = {(cuuint64_t)J.nx * es, (cuuint64_t)J.nx * J.ny * es};
    cuuint32_t box[3] = {(cuuint32_t)W, 1, 1};
    box[J.dir == DY ? 1 : 2] = (cuuint32_t)box_n;
    cuuint32_t estr[3] = {1, 1, 1};
    return enc(&J.tmap, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
               const_cast<T *>(J.in), gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Two slots, scratch and responses, then (kBatchStaged) the x staging rows;
// without them more CTAs may fit an SM.
template <typename T>
size_t batch_smem_bytes(size_t tile_cap, int variant)
{
    return variant == kBatchStaged ? batch_out_offset<T>(tile_cap) + tile_cap
                                   : 2 * tile_cap + batch_scratch_bytes_c<T>();
}

template <typename T>
static void (*batch_kernel(int variant))(const BatchJob<T> *, int, long, unsigned long long *, size_t, int *)
{
    if (variant == kBatchStaged) return ls_batch<T, kBatchStaged>;
    if (variant == kBatchMixed) return ls_batch<T, kBatchMixed>;
    return ls_batch<T, kBatchLong>;
}

template <typename T>
int batch_variant(const BatchJob<T> *jobs, int njobs)
{
    int v = kBatchLong;
    for (int i = 0; i < njobs; ++i) {
        if (jobs[i].dir == DX && jobs[i].xstage) return kBatchStaged;
        if (jobs[i].L != kChunkLong<T>) v = kBatchMixed;
    }
    return v;
}

template <typename T>
int prepare_batch(size_t tile_cap, int variant, size_t smem_optin, int num_sms, int *grid)
{
    const size_t smem = batch_smem_bytes<T>(tile_cap, variant);
    if (smem + 1024 > smem_optin) return X3D_EUNSUPPORTED;
    auto kern = batch_kernel<T>(variant);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return X3D_ECUDA;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBatchThreads, smem);
    *grid = num_sms * (per_sm < 1 ? 1 : per_sm);
    return X3D_OK;
}

template <typename T>
int launch_batch(cudaStream_t st, int grid, const BatchJob<T> *d_jobs, int njobs, long total,
                 unsigned long long *d_counter, size_t tile_cap, int variant, int *d_err)
{
    const size_t smem = batch_smem_bytes<T>(tile_cap, variant);
    if (cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), st) != cudaSuccess) return X3D_ECUDA;
    batch_kernel<T>(variant)<<<(unsigned)grid, kBatchThreads, smem, st>>>(d_jobs, njobs, total, d_counter,
                                                                           tile_cap, d_err);
    return cudaGetLastError() == cudaSuccess ? X3D_OK : X3D_ECUDA;
}

template bool plan_batch_job<float>(BatchJob<float> &, int, int, int, size_t *);
template bool plan_batch_job<double>(BatchJob<double> &, int, int, int, size_t *);
template int batch_variant<float>(const BatchJob<float> *, int);
template int batch_variant<double>(const BatchJob<double> *, int);
template int prepare_batch<float>(size_t, int, size_t, int, int *);
template int prepare_batch<double>(size_t, int, size_t, int, int *);
template int launch_batch<float>(cudaStream_t, int, const BatchJob<float> *, int, long, unsigned long long *,
                                 size_t, int, int *);
template int launch_batch<double>(cudaStream_t, int, const BatchJob<double> *, int, long, unsigned long long *,
                                  size_t, int, int *);

template int launch_stage<float>(x3d_ctx_s *, const StageProgram<float> &, int, int, int, int, int);
template int launch_stage<double>(x3d_ctx_s *, const StageProgram<double> &, int, int, int, int, int);
template StageProgram<float> plain_program<float>(const float *, const LineOp<float> *const *,
                                                  const int *, void *const *, int);
template StageProgram<double> plain_program<double>(const double *, const LineOp<double> *const *,
                                                    const int *, void *const *, int);

}  // namespace x3d
