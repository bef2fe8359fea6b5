// Streaming references for the roofline of the sweep launches: one FP32
// read and six FP32 writes per point with no arithmetic, in two orders:
//   flat:  consecutive threads on consecutive 16-byte vectors (the best case
//          of the traffic mix);
//   tile:  the y/z stage kernels' order: a CTA owns W x-adjacent columns of
//          the ny rows of one z plane (or of a block of 128 of them), thread
//          (l, c) moves one to four adjacent columns of 16 or 32 consecutive
//          rows, so each warp touches W-float row segments a row apart.
// bench.py times them next to the sweep to report how close each launch is
// to what its traffic mix and access order allow.
#include "x3d_internal.h"

namespace x3d {

struct Outs6 {
    float *p[6];
};

constexpr int kProbeL = 32;

__global__ void k_probe_flat(const float4 *__restrict__ in, const Outs6 outs, size_t n4)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
        const float4 v = in[i];
#pragma unroll
        for (int k = 0; k < 6; ++k) reinterpret_cast<float4 *>(outs.p[k])[i] = v;
    }
}

template <int V>
struct ProbeVec;
template <>
struct ProbeVec<1> {
    using type = float;
};
template <>
struct ProbeVec<2> {
    using type = float2;
};
template <>
struct ProbeVec<4> {
    using type = float4;
};

// A CTA owns W x-adjacent columns of `rows` consecutive rows (all ny, or a
// block of them) of one z plane; a thread moves V adjacent columns of RT
// rows: all its loads, then its rows of each output in turn.
//   BANDED = false: thread (l, c) takes rows c RT .. c RT + RT - 1 (the stage
//     kernels' chunks), so one store of the CTA touches rows RT apart;
//   BANDED = true: thread (l, r) takes rows r, r + NR, ... (NR = rows / RT),
//     so one store of the CTA touches NR consecutive rows.
// Tiles are numbered row block fastest, then x, then z (ZFIRST: then z,
// then x, so consecutive CTAs work on different z planes).
template <int W, int V, int RT, bool BANDED, bool ZFIRST>
__global__ void k_probe_tile(const float *__restrict__ in, const Outs6 outs, int nx, int ny, int nz, int rows)
{
    using VT = typename ProbeVec<V>::type;
    constexpr int WT = W / V;  // threads across the tile
    const int t = threadIdx.x, l = t % WT, c = t / WT;
    const int nr = rows / RT;
    const int tiles_x = nx / W, nb = ny / rows;
    const size_t r0 = BANDED ? (size_t)c : (size_t)c * RT;
    const size_t rstep = BANDED ? (size_t)nr * nx : (size_t)nx;
    for (long tile = blockIdx.x; tile < (long)tiles_x * nb * nz; tile += gridDim.x) {
        const int rb = (int)(tile % nb);
        const long xo = tile / nb;
        const int x0 = (int)(ZFIRST ? xo / nz : xo % tiles_x) * W;
        const int o = (int)(ZFIRST ? xo % nz : xo / tiles_x);
        const size_t base = (size_t)o * nx * ny + ((size_t)rb * rows + r0) * nx + x0 + V * l;
        VT r[RT];
#pragma unroll
        for (int j = 0; j < RT; ++j) r[j] = *reinterpret_cast<const VT *>(in + base + (size_t)j * rstep);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            float *dst = outs.p[k] + base;
#pragma unroll
            for (int j = 0; j < RT; ++j) *reinterpret_cast<VT *>(dst + (size_t)j * rstep) = r[j];
        }
    }
}

template <int W, int V, int RT, bool BANDED = false, bool ZFIRST = false>
static int probe_tile(x3d_ctx_s *ctx, int per_sm, const float *in, const Outs6 &o, int nx, int ny, int nz, int rows)
{
    const int threads = (W / V) * (rows / RT);
    // at most 512 threads: the 128-column form keeps 64 values per thread
    // in registers (80 registers a thread)
    if (rows % RT || threads > 512 || threads % 32)
        return set_error(ctx, X3D_EINVAL, "tile probe: rows must give a whole number of warps (at most 512 threads)");
    ++ctx->launches;
    k_probe_tile<W, V, RT, BANDED, ZFIRST><<<ctx->num_sms * per_sm, threads, 0, ctx->stream>>>(in, o, nx, ny, nz,
                                                                                               rows);
    return cuda_check(ctx, cudaGetLastError(), "k_probe_tile launch");
}

template <bool BANDED, bool ZFIRST>
static int probe_w(x3d_ctx_s *ctx, int w, int per_sm, const float *in, const Outs6 &o, int nx, int ny, int nz,
                   int rows)
{
    switch (w) {
    case 8: return probe_tile<8, 1, 32, BANDED, ZFIRST>(ctx, per_sm, in, o, nx, ny, nz, rows);
    case 16: return probe_tile<16, 1, 32, BANDED, ZFIRST>(ctx, per_sm, in, o, nx, ny, nz, rows);
    case 32: return probe_tile<32, 1, 32, BANDED, ZFIRST>(ctx, per_sm, in, o, nx, ny, nz, rows);
    case 64: return probe_tile<64, 2, 32, BANDED, ZFIRST>(ctx, per_sm, in, o, nx, ny, nz, rows);
    case 128: return probe_tile<128, 4, 16, BANDED, ZFIRST>(ctx, per_sm, in, o, nx, ny, nz, rows);
    default: return set_error(ctx, X3D_EINVAL, "tile probe: w must be 8, 16, 32, 64 or 128");
    }
}

// Pattern 5: the tile order of pattern 1 with tiles claimed from a counter
// (one atomicAdd per tile) instead of at a fixed stride, as the persistent
// stage kernels take them, so the tiles in flight stay a window of
// consecutive tiles.
// Pattern 6: the same for the z stage kernels' order: tiles of W columns of
// one y row over every z plane (rows nx ny apart), x tiles fastest.
template <int W, bool ZLINES>
__global__ void k_probe_tile_claim(const float *__restrict__ in, const Outs6 outs, int nx, int ny, int nz,
                                   unsigned long long *counter)
{
    constexpr int RT = 32;
    __shared__ long s_tile;
    const int t = threadIdx.x, l = t % W, c = t / W;
    const int tiles_x = nx / W;
    const long ntiles = (long)tiles_x * (ZLINES ? ny : nz);
    const size_t rs = ZLINES ? (size_t)nx * ny : (size_t)nx;  // elements between rows of a tile
    const size_t os = ZLINES ? (size_t)nx : (size_t)nx * ny;  // between tiles' planes (y rows)
    for (;;) {
        if (t == 0) s_tile = (long)atomicAdd(counter, 1ull);
        __syncthreads();
        const long tile = s_tile;
        __syncthreads();
        if (tile >= ntiles) break;
        const int x0 = (int)(tile % tiles_x) * W, o = (int)(tile / tiles_x);
        const size_t base = (size_t)o * os + (size_t)c * RT * rs + x0 + l;
        float r[RT];
#pragma unroll
        for (int j = 0; j < RT; ++j) r[j] = in[base + (size_t)j * rs];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            float *dst = outs.p[k] + base;
#pragma unroll
            for (int j = 0; j < RT; ++j) dst[(size_t)j * rs] = r[j];
        }
    }
}

int launch_roofline_probe(x3d_ctx_s *ctx, int pattern, int w, int ctas_per_sm, const float *in, float *const *outs,
                          int nx, int ny, int nz)
{
    const int per_sm = ctas_per_sm > 0 ? ctas_per_sm : 2;
    Outs6 o;
    for (int k = 0; k < 6; ++k) o.p[k] = outs[k];
    const size_t n = (size_t)nx * ny * nz;
    if (pattern == 0) {
        if (n % 4) return set_error(ctx, X3D_EINVAL, "flat probe needs a multiple of 4 points");
        ++ctx->launches;
        k_probe_flat<<<ctx->num_sms * per_sm * 4, 256, 0, ctx->stream>>>(reinterpret_cast<const float4 *>(in), o,
                                                                          n / 4);
        return cuda_check(ctx, cudaGetLastError(), "k_probe_flat launch");
    }
    // 1: whole columns (rows = ny); 2: blocks of 128 rows; 3: whole
    // columns, banded rows; 4: whole columns, tiles z plane first
    const int rows = pattern == 2 ? 128 : ny;
    if (nx % w || ny % rows || pattern > 6)
        return set_error(ctx, X3D_EINVAL, "tile probe needs nx % w == 0 and ny % rows == 0");
    if (pattern == 5 || pattern == 6) {
        const int rows = pattern == 5 ? ny : nz;
        const int threads = w * (rows / 32);
        if ((w != 8 && w != 16 && w != 32) || nx % w || rows % 32 || threads > 512 || threads % 32)
            return set_error(ctx, X3D_EINVAL, "tile probe patterns 5, 6: w 8, 16 or 32, line length % 32 == 0");
        auto *counter = ctx->d_claim;
        if (cudaMemsetAsync(counter, 0, sizeof(*counter), ctx->stream) != cudaSuccess)
            return set_error(ctx, X3D_ECUDA, "probe counter reset");
        const unsigned grid = (unsigned)(ctx->num_sms * per_sm);
        auto go = [&](auto kern) {
            ++ctx->launches;
            kern<<<grid, threads, 0, ctx->stream>>>(in, o, nx, ny, nz, counter);
            return cuda_check(ctx, cudaGetLastError(), "k_probe_tile_claim launch");
        };
        if (pattern == 5)
            return w == 8 ? go(k_probe_tile_claim<8, false>)
                          : (w == 16 ? go(k_probe_tile_claim<16, false>) : go(k_probe_tile_claim<32, false>));
        return w == 8 ? go(k_probe_tile_claim<8, true>)
                      : (w == 16 ? go(k_probe_tile_claim<16, true>) : go(k_probe_tile_claim<32, true>));
    }
    if (pattern == 3) return probe_w<true, false>(ctx, w, per_sm, in, o, nx, ny, nz, rows);
    if (pattern == 4) return probe_w<false, true>(ctx, w, per_sm, in, o, nx, ny, nz, rows);
    return probe_w<false, false>(ctx, w, per_sm, in, o, nx, ny, nz, rows);
}

}  // namespace x3d
