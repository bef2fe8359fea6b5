// Elementwise field kernels, the initial field, and the reductions behind the
// reference's test-mode checks.  All are single-pass, grid-stride, and sized
// to a multiple of the SM count.
#include <cmath>

#include "ptx.cuh"
#include "x3d_internal.h"

namespace x3d {

static unsigned grid_for(const x3d_ctx_s *ctx, size_t n, int bs)
{
    size_t want = (n + bs - 1) / bs;
    size_t cap = (size_t)ctx->num_sms * 8;
    return (unsigned)(want < cap ? (want ? want : 1) : cap);
}

template <typename T>
__global__ void k_axpy3(T *u, T *v, T *w, const T *du, const T *dv, const T *dw, T alpha, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        u[i] = alpha * du[i] + u[i];
        v[i] = alpha * dv[i] + v[i];
        w[i] = alpha * dw[i] + w[i];
    }
}

template <typename T>
__global__ void k_sub3(T *u, T *v, T *w, const T *a, const T *b, const T *c, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        u[i] = u[i] - a[i];
        v[i] = v[i] - b[i];
        w[i] = w[i] - c[i];
    }
}

template <typename T>
__global__ void k_mul(T *o, const T *a, const T *b, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        o[i] = a[i] * b[i];
}

template <typename T>
__global__ void k_fma_acc(T *o, const T *base, const T *a, const T *b, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        o[i] = base[i] + a[i] * b[i];
}

template <typename T>
__global__ void k_add(T *o, const T *a, const T *b, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        o[i] = a[i] + b[i];
}

template <typename D, typename S>
__global__ void k_convert(D *o, const S *a, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        o[i] = (D)a[i];
}

// vel (src/mom.f90:46-53): x = (i-1)*dx etc. on a single rank.
template <typename T>
__global__ void k_vel(T *u, T *v, T *w, int nx, int ny, int nz, double xlx, double yly, double zlz)
{
    const double twopi = 2.0 * 3.14159265358979323846;
    const double dx = xlx / nx, dy = yly / ny, dz = zlz / nz;
    const size_t n = (size_t)nx * ny * nz;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(p % nx);
        const int j = (int)((p / nx) % ny);
        const int k = (int)(p / ((size_t)nx * ny));
        const double x = i * dx, y = j * dy, z = k * dz;
        const double sx = sin(twopi * (x / xlx)), cx = cos(twopi * (x / xlx));
        const double sy = sin(twopi * (y / yly)), cy = cos(twopi * (y / yly));
        const double sz = sin(twopi * (z / zlz)), cz = cos(twopi * (z / zlz));
        u[p] = (T)(sx * cy * cz);
        v[p] = (T)(cx * sy * cz);
        w[p] = (T)(-2.0 * cx * cy * sz);
    }
}

// Sum of squared errors against the analytic derivative (test_du/dv/dw).
template <typename T>
__global__ void k_test_sq(const T *du, int which, int nx, int ny, int nz, double xlx, double yly,
                          double zlz, double *out)
{
    const double twopi = 2.0 * 3.14159265358979323846;
    const double dx = xlx / nx, dy = yly / ny, dz = zlz / nz;
    const size_t n = (size_t)nx * ny * nz;
    double acc = 0.0;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(p % nx);
        const int j = (int)((p / nx) % ny);
        const int k = (int)(p / ((size_t)nx * ny));
        const double x = i * dx, y = j * dy, z = k * dz;
        double ana = cos(twopi * (x / xlx)) * cos(twopi * (y / yly)) * cos(twopi * (z / zlz));
        if (which == 0) ana = twopi * ana / xlx;
        else if (which == 1) ana = twopi * ana / yly;
        else ana = twopi * (-2.0 * ana) / zlz;
        const double e = (double)du[p] - ana;
        acc += e * e;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += part[q];
        atomicAdd(out, s);
    }
}

__global__ void k_absmax_sum(const double *p, size_t n, double *out)
{
    double mx = 0.0, sm = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double a = fabs(p[i]);
        mx = fmax(mx, a);
        sm += a;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        sm += __shfl_down_sync(0xffffffffu, sm, o);
    }
    __shared__ double pm[32], ps[32];
    if ((threadIdx.x & 31) == 0) {
        pm[threadIdx.x >> 5] = mx;
        ps[threadIdx.x >> 5] = sm;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
            a = fmax(a, pm[q]);
            b += ps[q];
        }
        // max of non-negative doubles: their bit patterns order like integers
        atomicMax(reinterpret_cast<unsigned long long *>(out), __double_as_longlong(a));
        atomicAdd(out + 1, b);
    }
}

// t(i,j,k) *= ppy(j): the stretching multiply of dery_00, deryvp and derypv
// when istret /= 0 (src/x3d_derive.f90:331-337, src/x3d_staggered.f90:629-635,
// 875-881).  Grid-stride over the field; j from the flat index.
template <typename T>
__global__ void k_scale_y(T *t, const double *ppy, int nx, int ny, size_t n)
{
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        t[p] = (T)((double)t[p] * ppy[(p / (size_t)nx) % (size_t)ny]);
}

#define X3D_LAUNCH(kern, n, ...)                                                          \
    do {                                                                                  \
        const int bs_ = 256;                                                              \
        ++ctx->launches;                                                                  \
        kern<<<grid_for(ctx, (n), bs_), bs_, 0, ctx->stream>>>(__VA_ARGS__);              \
        return cuda_check(ctx, cudaGetLastError(), #kern);                                \
    } while (0)

int launch_copy(x3d_ctx_s *ctx, void *dst, const void *src, size_t bytes)
{
    if (dst == src) return X3D_OK;
    return cuda_check(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream),
                      "device copy");
}

int launch_axpy3(x3d_ctx_s *ctx, bool fp32, void *u, void *v, void *w, const void *du,
                 const void *dv, const void *dw, double alpha, size_t n)
{
    if (fp32)
        X3D_LAUNCH(k_axpy3<float>, n, (float *)u, (float *)v, (float *)w, (const float *)du,
                   (const float *)dv, (const float *)dw, (float)alpha, n);
    X3D_LAUNCH(k_axpy3<double>, n, (double *)u, (double *)v, (double *)w, (const double *)du,
               (const double *)dv, (const double *)dw, alpha, n);
}

int launch_sub3(x3d_ctx_s *ctx, bool fp32, void *u, void *v, void *w, const void *a, const void *b,
                const void *c, size_t n)
{
    if (fp32)
        X3D_LAUNCH(k_sub3<float>, n, (float *)u, (float *)v, (float *)w, (const float *)a,
                   (const float *)b, (const float *)c, n);
    X3D_LAUNCH(k_sub3<double>, n, (double *)u, (double *)v, (double *)w, (const double *)a,
               (const double *)b, (const double *)c, n);
}

// A bounded wait that nothing can complete: the mbarrier expects one arrival
// and none comes, and no copy is in flight.  The wait gives up after
// limit_ns and records the failure in the error flag, as every bounded wait
// of the stage and batch kernels does, so the whole path (device flag, host
// status, context still usable) can be checked without a GPU fault.
__global__ void k_wait_selftest(int *err, uint64_t limit_ns)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0, limit_ns);
    if (!__syncthreads_and(ok) && threadIdx.x == 0) atomicExch(err, 2);
}

int launch_wait_selftest(x3d_ctx_s *ctx, uint64_t limit_ns)
{
    ++ctx->launches;
    k_wait_selftest<<<1, 32, 0, ctx->stream>>>(ctx->d_err, limit_ns);
    return cuda_check(ctx, cudaGetLastError(), "k_wait_selftest launch");
}

int launch_scale_y(x3d_ctx_s *ctx, bool fp32, void *t, const double *ppy, int nx, int ny, int nz)
{
    const size_t n = (size_t)nx * ny * nz;
    if (fp32) X3D_LAUNCH(k_scale_y<float>, n, (float *)t, ppy, nx, ny, n);
    X3D_LAUNCH(k_scale_y<double>, n, (double *)t, ppy, nx, ny, n);
}

int launch_mul(x3d_ctx_s *ctx, bool fp32, void *out, const void *a, const void *b, size_t n)
{
    if (fp32) X3D_LAUNCH(k_mul<float>, n, (float *)out, (const float *)a, (const float *)b, n);
    X3D_LAUNCH(k_mul<double>, n, (double *)out, (const double *)a, (const double *)b, n);
}

int launch_fma_acc(x3d_ctx_s *ctx, bool fp32, void *out, const void *base, const void *a,
                   const void *b, size_t n)
{
    if (fp32)
        X3D_LAUNCH(k_fma_acc<float>, n, (float *)out, (const float *)base, (const float *)a,
                   (const float *)b, n);
    X3D_LAUNCH(k_fma_acc<double>, n, (double *)out, (const double *)base, (const double *)a,
               (const double *)b, n);
}

int launch_add(x3d_ctx_s *ctx, bool fp32, void *out, const void *a, const void *b, size_t n)
{
    if (fp32) X3D_LAUNCH(k_add<float>, n, (float *)out, (const float *)a, (const float *)b, n);
    X3D_LAUNCH(k_add<double>, n, (double *)out, (const double *)a, (const double *)b, n);
}

int launch_convert(x3d_ctx_s *ctx, void *dst, bool dst_fp32, const void *src, bool src_fp32, size_t n)
{
    if (dst_fp32 == src_fp32) return launch_copy(ctx, dst, src, n * (dst_fp32 ? 4 : 8));
    if (dst_fp32) X3D_LAUNCH((k_convert<float, double>), n, (float *)dst, (const double *)src, n);
    X3D_LAUNCH((k_convert<double, float>), n, (double *)dst, (const float *)src, n);
}

int launch_vel(x3d_ctx_s *ctx, bool fp32, void *u, void *v, void *w)
{
    const size_t n = ctx->npts();
    if (fp32)
        X3D_LAUNCH(k_vel<float>, n, (float *)u, (float *)v, (float *)w, ctx->nx, ctx->ny, ctx->nz,
                   ctx->xlx, ctx->yly, ctx->zlz);
    X3D_LAUNCH(k_vel<double>, n, (double *)u, (double *)v, (double *)w, ctx->nx, ctx->ny, ctx->nz,
               ctx->xlx, ctx->yly, ctx->zlz);
}

int reduce_test_rms(x3d_ctx_s *ctx, bool fp32, int which, const void *du, double *rms)
{
    const size_t n = ctx->npts();
    int rc = cuda_check(ctx, cudaMemsetAsync(ctx->d_red, 0, 2 * sizeof(double), ctx->stream), "memset");
    if (rc) return rc;
    const int bs = 256;
    ++ctx->launches;
    if (fp32)
        k_test_sq<float><<<grid_for(ctx, n, bs), bs, 0, ctx->stream>>>(
            (const float *)du, which, ctx->nx, ctx->ny, ctx->nz, ctx->xlx, ctx->yly, ctx->zlz, ctx->d_red);
    else
        k_test_sq<double><<<grid_for(ctx, n, bs), bs, 0, ctx->stream>>>(
            (const double *)du, which, ctx->nx, ctx->ny, ctx->nz, ctx->xlx, ctx->yly, ctx->zlz, ctx->d_red);
    rc = cuda_check(ctx, cudaGetLastError(), "k_test_sq");
    if (rc) return rc;
    double s = 0.0;
    rc = cuda_check(ctx, cudaMemcpyAsync(&s, ctx->d_red, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "d2h");
    if (rc) return rc;
    rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (rc) return rc;
    *rms = std::sqrt(s / ctx->nx / ctx->ny / ctx->nz);
    return X3D_OK;
}

int reduce_absmax_mean(x3d_ctx_s *ctx, const double *p, size_t n, double *out)
{
    int rc = cuda_check(ctx, cudaMemsetAsync(ctx->d_red, 0, 2 * sizeof(double), ctx->stream), "memset");
    if (rc) return rc;
    const int bs = 256;
    ++ctx->launches;
    k_absmax_sum<<<grid_for(ctx, n, bs), bs, 0, ctx->stream>>>(p, n, ctx->d_red);
    rc = cuda_check(ctx, cudaGetLastError(), "k_absmax_sum");
    if (rc) return rc;
    double h[2];
    rc = cuda_check(ctx, cudaMemcpyAsync(h, ctx->d_red, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "d2h");
    if (rc) return rc;
    rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (rc) return rc;
    out[0] = h[0];
    out[1] = h[1] / (double)n;
    return X3D_OK;
}

}  // namespace x3d
