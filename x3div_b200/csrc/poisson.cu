// Spectral Poisson solve for a fully periodic box: poisson_000
// (src/poisson.f90:276-419) with the modified wavenumbers of waves()
// (:483-767) and the phase tables of abxyz (:421-479).
//
// The reference transforms with 2decomp's PHYSICAL_IN_Z r2c (z halved),
// then per mode: scales by 1/ntot, applies phase factors e^{-i theta_z},
// e^{-i theta_y} (negated past ny/2+1) and e^{-i theta_x} (negated past
// nx/2+1), divides real and imaginary parts by -K (zero when K < 1e-16),
// and applies the conjugating inverse factors.  Composed, those factors
// cancel exactly for every mode (forward: c e^{-i sum} s_x s_y; backward
// conj(conj(c') e^{-i tz} e^{-i ty} s_y) e^{+i tx} s_x = c'), so the mode
// update is  c <- -c / (K ntot)  with the same K and the same mask.
//
// Here cuFFT's D2Z/Z2D on the (nz, ny, nx) row-major array halves x instead
// of z.  K is even in each index separately (the 1-D tables are mirrored,
// waves :534-538, :568-572), so every mode of the x-halved spectrum gets
// bit-for-bit the K value the reference uses for the same or the conjugate
// mode, and the mask makes the same decisions.
#include <cmath>
#include <vector>

#include "x3d_internal.h"

namespace x3d {

// The 1-D factors of kxyz for one direction (bc = 0), computed on the host in
// FP64 with libm exactly as waves() does:
//   k2[i] = (n wp / L)^2, wp = (acix6 2 d sin(w/2) + bcix6 2 d sin(3w/2)) / (1 + 2 alcaix6 cos w)
//   t[i]  = (2 aicix6 cos(r/2) + 2 (bicix6 cos(1.5r) + cicix6 cos(2.5r) + dicix6 cos(3.5r)))
//           / (1 + 2 ailcaix6 cos r),  r = exs(i) d
static void waves_tables(int n, double len, std::vector<double> &k2, std::vector<double> &t)
{
    const double twopi = 2.0 * std::acos(-1.0);
    const double d = len / n;
    double alcai, aci, bci, c_, d_;
    rhs_scalars(DERVP, d, &alcai, &aci, &bci, &c_, &d_);
    double ailcai, aici, bici, cici, dici;
    rhs_scalars(INTVP, d, &ailcai, &aici, &bici, &cici, &dici);
    std::vector<double> es(n);
    k2.assign(n, 0.0);
    t.assign(n, 0.0);
    for (int i = 0; i < n / 2 + 1; ++i) {
        const double w = twopi * i / n;
        double wp = aci * 2.0 * d * std::sin(w * 0.5) + bci * 2.0 * d * std::sin(3.0 * 0.5 * w);
        wp = wp / (1.0 + 2.0 * alcai * std::cos(w));
        es[i] = n * w / len;
        const double q = n * wp / len;
        k2[i] = q * q;
    }
    for (int i = n / 2 + 1; i < n; ++i) {
        k2[i] = k2[n - i];
        es[i] = es[n - i];
    }
    for (int i = 0; i < n; ++i) {
        const double r = es[i] * d;
        const double tt = 2.0 * (bici * std::cos(r * 1.5) + cici * std::cos(r * 2.5) + dici * std::cos(r * 3.5));
        const double tt1 = 2.0 * aici * std::cos(r * 0.5);
        const double t1 = 1.0 + 2.0 * ailcai * std::cos(r);
        t[i] = (tt1 + tt) / t1;
    }
}

// c(i,j,k) <- -c / (K ntot), K = k2x Ty^2 Tz^2 + k2y Tx^2 Tz^2 + k2z Tx^2 Ty^2
// (waves :690-694: xk2(i) * ((Ty*Tz)**2) etc.), zero where K < 1e-16.
// One division per mode (the reference divides Re and Im by ntot and then by
// -K; the product form differs from it by a few ulp).  Indices are 32-bit:
// the spectrum of any grid that fits one GPU has fewer than 2^32 modes.
__global__ void k_spectral_divide(double2 *c, unsigned nxh, unsigned ny, unsigned n, const double *k2x,
                                  const double *tx, const double *k2y, const double *ty,
                                  const double *k2z, const double *tz, double ntot)
{
    for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const unsigned row = p / nxh;
        const unsigned i = p - row * nxh;
        const unsigned k = row / ny;
        const unsigned j = row - k * ny;
        const double txi = __ldg(tx + i), tyj = __ldg(ty + j), tzk = __ldg(tz + k);
        const double tyz = tyj * tzk, txz = txi * tzk, txy = txi * tyj;
        const double kk = __ldg(k2x + i) * (tyz * tyz) + __ldg(k2y + j) * (txz * txz) +
                          __ldg(k2z + k) * (txy * txy);
        double2 v = c[p];
        const double f = kk < 1.e-16 ? 0.0 : -1.0 / (kk * ntot);
        v.x *= f;
        v.y *= f;
        c[p] = v;
    }
}

int poisson_setup(x3d_ctx_s *ctx)
{
    if (ctx->plans_ready) return X3D_OK;
    const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    std::vector<double> k2x, tx, k2y, ty, k2z, tz;
    waves_tables(nx, ctx->xlx, k2x, tx);
    waves_tables(ny, ctx->yly, k2y, ty);
    waves_tables(nz, ctx->zlz, k2z, tz);
    double *tab = nullptr;
    const size_t tot = 2 * ((size_t)nx + ny + nz);
    if (cudaMalloc(&tab, tot * sizeof(double)) != cudaSuccess) return set_error(ctx, X3D_ENOMEM, "poisson tables");
    std::vector<double> h;
    h.reserve(tot);
    h.insert(h.end(), k2x.begin(), k2x.end());
    h.insert(h.end(), tx.begin(), tx.end());
    h.insert(h.end(), k2y.begin(), k2y.end());
    h.insert(h.end(), ty.begin(), ty.end());
    h.insert(h.end(), k2z.begin(), k2z.end());
    h.insert(h.end(), tz.begin(), tz.end());
    cudaMemcpy(tab, h.data(), tot * sizeof(double), cudaMemcpyHostToDevice);
    ctx->d_k2x = tab;
    ctx->d_tx = tab + nx;
    ctx->d_k2y = tab + 2 * nx;
    ctx->d_ty = tab + 2 * nx + ny;
    ctx->d_k2z = tab + 2 * nx + 2 * ny;
    ctx->d_tz = tab + 2 * nx + 2 * ny + nz;
    const size_t spec = (size_t)nz * ny * (nx / 2 + 1) * sizeof(double2);
    if (cudaMalloc(&ctx->spectrum, spec) != cudaSuccess) return set_error(ctx, X3D_ENOMEM, "poisson spectrum");
    if (cufftPlan3d(&ctx->plan_d2z, nz, ny, nx, CUFFT_D2Z) != CUFFT_SUCCESS ||
        cufftPlan3d(&ctx->plan_z2d, nz, ny, nx, CUFFT_Z2D) != CUFFT_SUCCESS)
        return set_error(ctx, X3D_ECUDA, "cufftPlan3d failed");
    ctx->plans_ready = true;
    return X3D_OK;
}

int poisson_solve(x3d_ctx_s *ctx, double *rhs)
{
    int rc = poisson_setup(ctx);
    if (rc) return rc;
    cufftSetStream(ctx->plan_d2z, ctx->stream);
    cufftSetStream(ctx->plan_z2d, ctx->stream);
    if (cufftExecD2Z(ctx->plan_d2z, rhs, (cufftDoubleComplex *)ctx->spectrum) != CUFFT_SUCCESS)
        return set_error(ctx, X3D_ECUDA, "cufftExecD2Z failed");
    const int nxh = ctx->nx / 2 + 1;
    const size_t n = (size_t)nxh * ctx->ny * ctx->nz;
    if (n >= (1ull << 31)) return set_error(ctx, X3D_EUNSUPPORTED, "spectrum above 2^31 modes");
    const int bs = 256;
    size_t g = (n + bs - 1) / bs;
    const size_t cap = (size_t)ctx->num_sms * 8;
    if (g > cap) g = cap;
    const double ntot = (double)ctx->nx * (double)ctx->ny * (double)ctx->nz;
    ++ctx->launches;
    k_spectral_divide<<<(unsigned)g, bs, 0, ctx->stream>>>((double2 *)ctx->spectrum, (unsigned)nxh,
                                                           (unsigned)ctx->ny, (unsigned)n, ctx->d_k2x,
                                                           ctx->d_tx, ctx->d_k2y, ctx->d_ty, ctx->d_k2z,
                                                           ctx->d_tz, ntot);
    rc = cuda_check(ctx, cudaGetLastError(), "k_spectral_divide");
    if (rc) return rc;
    if (cufftExecZ2D(ctx->plan_z2d, (cufftDoubleComplex *)ctx->spectrum, rhs) != CUFFT_SUCCESS)
        return set_error(ctx, X3D_ECUDA, "cufftExecZ2D failed");
    return X3D_OK;
}

void poisson_free(x3d_ctx_s *ctx)
{
    if (ctx->plans_ready) {
        cufftDestroy(ctx->plan_d2z);
        cufftDestroy(ctx->plan_z2d);
    }
    ctx->plans_ready = false;
    if (ctx->spectrum) cudaFree(ctx->spectrum);
    ctx->spectrum = nullptr;
    if (ctx->d_k2x) cudaFree(ctx->d_k2x);
    ctx->d_k2x = nullptr;
}

}  // namespace x3d
