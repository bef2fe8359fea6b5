// Streaming references for the roofline of the sweep launches: one FP32
// read and six FP32 writes per point with no arithmetic, in two orders:
//   flat:  consecutive threads on consecutive 16-byte vectors (the best case
//          of the traffic mix);
//   tile:  the y/z stage kernels' order: a CTA owns W x-adjacent columns of
//          the ny rows of one z plane, thread (l, c) moves column l, rows
//          c L .. c L + L - 1, so each warp touches W-float row segments
//          ny-row strides apart.
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

template <int W>
__global__ void k_probe_tile(const float *__restrict__ in, const Outs6 outs, int nx, int ny, int nz)
{
    const int t = threadIdx.x, l = t % W, c = t / W;
    const int tiles_x = nx / W;
    for (long tile = blockIdx.x; tile < (long)tiles_x * nz; tile += gridDim.x) {
        const int x0 = (int)(tile % tiles_x) * W, o = (int)(tile / tiles_x);
        const size_t base = (size_t)o * nx * ny + (size_t)c * kProbeL * nx + x0 + l;
        float r[kProbeL];
#pragma unroll
        for (int j = 0; j < kProbeL; ++j) r[j] = in[base + (size_t)j * nx];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            float *dst = outs.p[k] + base;
#pragma unroll
            for (int j = 0; j < kProbeL; ++j) dst[(size_t)j * nx] = r[j];
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
    if (nx % w || ny % kProbeL || (w != 8 && w != 16 && w != 32) || (ny / kProbeL) * w > 1024)
        return set_error(ctx, X3D_EINVAL, "tile probe needs nx % w == 0, ny % 32 == 0, w in {8, 16, 32}");
    const int threads = w * (ny / kProbeL);
    const int grid = ctx->num_sms * per_sm;
    ++ctx->launches;
    if (w == 8) k_probe_tile<8><<<grid, threads, 0, ctx->stream>>>(in, o, nx, ny, nz);
    else if (w == 16) k_probe_tile<16><<<grid, threads, 0, ctx->stream>>>(in, o, nx, ny, nz);
    else k_probe_tile<32><<<grid, threads, 0, ctx->stream>>>(in, o, nx, ny, nz);
    return cuda_check(ctx, cudaGetLastError(), "k_probe_tile launch");
}

}  // namespace x3d
