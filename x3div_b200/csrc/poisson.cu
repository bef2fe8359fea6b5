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
#include <algorithm>
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
// -K; the product form differs from it by a few ulp).  The block c holds
// x modes i0 .. i0 + nxl - 1 and y rows j0 .. j0 + nyl - 1 of every z mode
// ((nz, nyl, nxl), x fastest; the whole spectrum with i0 = j0 = 0).
// Indices are 32-bit: the spectrum of any grid that fits one GPU has fewer
// than 2^32 modes.
__global__ void k_spectral_divide(double2 *c, unsigned nxl, unsigned nyl, unsigned n, unsigned i0, unsigned j0,
                                  const double *k2x, const double *tx, const double *k2y, const double *ty,
                                  const double *k2z, const double *tz, double ntot)
{
    for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const unsigned row = p / nxl;
        const unsigned i = i0 + (p - row * nxl);
        const unsigned k = row / nyl;
        const unsigned j = j0 + (row - k * nyl);
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

// ---------------------------------------------------------------------------
// z transforms fused with the mode division.  The 3-D transform of the
// (nz, ny, nx) field separates into 1-D transforms along x, y and z: the
// library's own real x transforms (below) and batched 1-D cuFFT transforms
// along y, or cuFFT's 2-D (x, y) transforms of each z plane, then the z
// lines of the half spectrum.  One kernel takes a tile of W lane-adjacent z
// lines into shared memory, transforms them forward along z, divides each
// mode, and transforms them back, so the spectrum crosses HBM once for all
// three steps (cuFFT's z passes and a separate division kernel cross it
// three times).
//
// The z transforms are mixed-radix Stockham autosort FFTs (radix 8, 4, 2,
// then 3), the formulation of Govindaraju et al., "High performance discrete
// Fourier transforms on graphics processors" (SC 2008): a stage of radix R
// over sub-transforms of size Ns reads element j + q n/R (q < R) of each
// line, multiplies it by W_n^(q (j mod Ns) n/(Ns R)), takes the length-R DFT
// in registers and writes the results to (j div Ns) Ns R + (j mod Ns) + q Ns.
// Each stage reads all its inputs before a barrier and writes after it, so
// one shared-memory buffer suffices.  Twiddles come from a table of the
// roots of unity computed on the host in FP64: a butterfly reads the first
// of its R - 1 and makes the others as its powers (the recurrence of Van
// Loan, "Computational Frameworks for the FFT", 1.4), so a stage reads one
// table entry a butterfly rather than R - 1.

constexpr int kZftThreads = 512;
constexpr int kZftVals = 8;    // values a thread holds in one stage

// Lines per tile for a transform of length N (W N <= kZftThreads kZftVals).
// (8 lines and 1024 threads for N = 768 timed 3.62 ms against 3.52 for these
// 4 lines and 512 threads, 768^3.)
template <int N>
constexpr int kZftW = N <= 256 ? 16 : (N <= 512 ? 8 : 4);

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// a times -i (forward transform) or +i (inverse)
template <bool INV>
__device__ __forceinline__ double2 cmi(double2 a)
{
    return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// Length-R DFT of v in place, exponent sign - (forward) or + (INV).
template <int R, bool INV>
__device__ __forceinline__ void dft(double2 (&v)[R])
{
    if constexpr (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        const double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        const double2 t2 = cadd(v[1], v[3]), t3 = cmi<INV>(csub(v[1], v[3]));
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    } else if constexpr (R == 8) {
        // two length-4 DFTs of the even and odd points, joined by W_8^k
        double2 e[4] = {v[0], v[2], v[4], v[6]};
        double2 o[4] = {v[1], v[3], v[5], v[7]};
        dft<4, INV>(e);
        dft<4, INV>(o);
        const double c = 0.70710678118654752440;  // sqrt(1/2)
        const double sg = INV ? 1.0 : -1.0;
        const double2 w1 = make_double2(c, sg * c), w3 = make_double2(-c, sg * c);
        const double2 o1 = cmul(o[1], w1), o2 = cmi<INV>(o[2]), o3 = cmul(o[3], w3);
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    } else {  // R == 3
        const double s3 = 0.86602540378443864676;  // sqrt(3)/2
        const double2 t = cadd(v[1], v[2]);
        const double2 m = cmi<INV>(csub(v[1], v[2]));
        const double2 h = make_double2(v[0].x - 0.5 * t.x, v[0].y - 0.5 * t.y);
        v[0] = cadd(v[0], t);
        v[1] = make_double2(h.x + s3 * m.x, h.y + s3 * m.y);
        v[2] = make_double2(h.x - s3 * m.x, h.y - s3 * m.y);
    }
}

// Where a stage reads and writes: the tile in shared memory, or (first
// forward stage) the spectrum's z lines in global memory and (last inverse
// stage) back to them; the last forward stage also divides each mode.
struct ZLines {
    double2 *base;   // the tile's first line at k = 0
    size_t zstride;  // elements between consecutive k
    size_t lstride;  // elements between consecutive lines
    int lines;       // lines of the tile inside the array (<= W)
    double tyj, k2yj, ntot;
    const double2 *xtab;  // shared: (t, k2) of the tile's W lanes
    const double2 *ztab;  // shared: (tz, k2z) of the N z modes
    // c <- -c / (K ntot), zero where K < 1e-16: the K and mask of
    // k_spectral_divide for mode (lane l, row, k)
    __device__ __forceinline__ double2 divide(double2 v, int k, int l) const
    {
        const double2 x = xtab[l], z = ztab[k];
        const double txi = x.x, tzk = z.x;
        const double tyz = tyj * tzk, txz = txi * tzk, txy = txi * tyj;
        const double kk = x.y * (tyz * tyz) + k2yj * (txz * txz) + z.y * (txy * txy);
        const double f = kk < 1.e-16 ? 0.0 : -1.0 / (kk * ntot);
        return make_double2(v.x * f, v.y * f);
    }
};

// One Stockham stage of radix R over sub-transforms of size NS, for the W
// lines of the tile (element e of line l at buf[e W + l]).  SRC_G: read the
// lines from global memory; DST_G: write them to global memory.  FUSE (the
// forward transform's last stage, NS = N / R): divide each mode, then run
// the inverse transform's first stage in registers -- with the inverse's
// radices in reverse order that stage has the same radix, reads exactly the
// values this thread holds (positions j + q N / R) with unit twiddles, and
// writes positions j R + q -- so the modes make one shared-memory pass
// fewer.
template <int N, int R, int NS, int W, bool INV, bool SRC_G, bool DST_G, bool FUSE, int NT = kZftThreads>
__device__ __forceinline__ void zft_stage(double2 *buf, const double2 *tw, const ZLines &zl)
{
    constexpr int MB = kZftVals / R;
    constexpr int NB = W * (N / R);
    constexpr int STRIDE = N / (NS * R);
    static_assert(NB <= MB * NT, "tile too large for one pass of the stage");
    double2 v[MB][R];
    int dk[MB], dl[MB];
#pragma unroll
    for (int s = 0; s < MB; ++s) {
        const int b = threadIdx.x + s * NT;
        if (b < NB) {
            const int l = b % W, j = b / W;
            const int jm = j % NS;
            // the twiddles W_n^(q jm n / (NS R)), q < R, as powers of w1 (q = 1):
            // one table read a butterfly, each power one product from the last
            // (a few ulp of W_n after R - 1 products)
            double2 w1 = make_double2(1.0, 0.0);
            if constexpr (NS > 1) {
                w1 = tw[jm * STRIDE];
                if (INV) w1.y = -w1.y;
            }
            double2 wq = w1;
#pragma unroll
            for (int q = 0; q < R; ++q) {
                const int k = j + q * (N / R);
                double2 x;
                if constexpr (SRC_G)
                    x = l < zl.lines ? zl.base[(size_t)k * zl.zstride + (size_t)l * zl.lstride]
                                     : make_double2(0.0, 0.0);
                else
                    x = buf[k * W + l];
                if (q == 0 || NS == 1) {  // the first stage's twiddles are all 1
                    v[s][q] = x;
                } else {
                    v[s][q] = cmul(x, wq);
                    wq = cmul(wq, w1);
                }
            }
            dft<R, INV>(v[s]);
            dk[s] = (j / NS) * NS * R + jm;
            dl[s] = l;
            if constexpr (FUSE) {
                static_assert(NS * R == N, "the fused stage is the forward transform's last");
#pragma unroll
                for (int q = 0; q < R; ++q) v[s][q] = zl.divide(v[s][q], dk[s] + q * NS, l);
                dft<R, true>(v[s]);
                dk[s] = j * R;  // the inverse's first stage (sub-transforms of size 1) writes j R + q
            }
        }
    }
    if constexpr (!SRC_G && !DST_G) __syncthreads();  // in place in shared memory
#pragma unroll
    for (int s = 0; s < MB; ++s) {
        const int b = threadIdx.x + s * NT;
        if (b < NB) {
#pragma unroll
            for (int q = 0; q < R; ++q) {
                const int k = dk[s] + q * (FUSE ? 1 : NS), l = dl[s];
                if constexpr (DST_G) {
                    if (l < zl.lines) zl.base[(size_t)k * zl.zstride + (size_t)l * zl.lstride] = v[s][q];
                } else {
                    buf[k * W + l] = v[s][q];
                }
            }
        }
    }
    if constexpr (!DST_G) __syncthreads();
}

// Radices of a length-N transform: 8s, 4, 2, then 3s (the inverse
// transform takes them in reverse order: a Stockham sequence may run its
// radices in any order).
struct RadixSeq {
    int count;
    int r[10];
};
constexpr RadixSeq radix_seq(int n, bool reversed = false)
{
    RadixSeq s{0, {}};
    int m = n;
    while (m % 8 == 0 && m > 1) s.r[s.count++] = 8, m /= 8;
    while (m % 4 == 0) s.r[s.count++] = 4, m /= 4;
    while (m % 2 == 0) s.r[s.count++] = 2, m /= 2;
    while (m % 3 == 0) s.r[s.count++] = 3, m /= 3;
    if (reversed)
        for (int a = 0, b = s.count - 1; a < b; ++a, --b) {
            const int t = s.r[a];
            s.r[a] = s.r[b];
            s.r[b] = t;
        }
    return s;
}

// The z transform, division and inverse of a tile (SOLVE).  The forward
// transform reads the lines from global memory in its first stage; its last
// stage divides the modes and runs the inverse's first stage in registers
// (the inverse takes the radices in reverse order); the inverse writes the
// lines back to global memory in its last stage, which is that fused stage
// itself when the length has a single radix.  Without SOLVE: the forward
// transform alone (!INV: lines from global memory, the transform left in
// buf in natural order) or the inverse alone (INV: from buf to global
// memory).
// Stages ST .. END - 1 only where END >= 0 (a stage before the sequence's
// last then writes shared memory and ends with a barrier).
template <int N, int W, bool INV, bool SOLVE = true, int NT = kZftThreads, int ST = 0, int NS = 1, int END = -1>
__device__ __forceinline__ void zft(double2 *buf, const double2 *tw, const ZLines &zl)
{
    constexpr RadixSeq seq = radix_seq(N, INV);
    if constexpr (ST < (END < 0 ? seq.count : END)) {
        constexpr int R = seq.r[ST];
        constexpr bool last = ST + 1 == seq.count;
        if constexpr (SOLVE && !INV && last) {
            zft_stage<N, R, NS, W, false, ST == 0, seq.count == 1, true, NT>(buf, tw, zl);
            zft<N, W, true, true, NT, 1, R>(buf, tw, zl);  // the inverse from its second stage
        } else {
            zft_stage<N, R, NS, W, INV, !INV && ST == 0, INV && last, false, NT>(buf, tw, zl);
            zft<N, W, INV, SOLVE, NT, ST + 1, NS * R, END>(buf, tw, zl);
        }
    }
}


// One CTA per (j, tile of W x-modes): z transform, c <- -c / (K ntot) with the
// K and mask of k_spectral_divide, inverse z transform.  The tile's modes go
// from global memory straight into the first stage's registers and leave
// the last inverse stage straight to global memory; the twiddles and the
// wavenumber tables the division reads are copied into shared memory first
// (read through L1 instead, the z kernel at 512^3 took 790 us against 720).
// The spectrum is (nz, ny, nxl) with x fastest:
// x modes ig0 .. ig0 + nxl - 1 of the nxh = nx/2 + 1 and y rows j0 .. j0 +
// ny - 1 of the box (a Z pencil of the half spectrum).  K is symmetric in
// the x and y factors, so the same kernel solves a spectrum stored (nz,
// nxh, ny) with y fastest when given the y tables as (k2x, tx), the x tables
// as (k2y, ty) and ny as nxl and nxh, nxh as ny.
template <int N>
__global__ void __launch_bounds__(kZftThreads, 2)
    k_poisson_z(double2 *__restrict__ c, int nxl, int ny, int ig0, int j0, int nxh,
                const double2 *__restrict__ tw, const double *__restrict__ k2x, const double *__restrict__ tx,
                const double *__restrict__ k2y, const double *__restrict__ ty, double ntot)
{
    constexpr int W = kZftW<N>;
    extern __shared__ __align__(16) double2 zbuf[];
    double2 *const tws = zbuf + N * W;  // twiddles, then (tz, k2z), then the lanes' (t, k2)
    double2 *const xtab = tws + 2 * N;
    const int tiles_i = (nxl + W - 1) / W;
    const int j = blockIdx.x / tiles_i;
    const int i0 = (blockIdx.x - j * tiles_i) * W;
    ZLines zl;
    zl.base = c + (size_t)j * nxl + i0;
    zl.zstride = (size_t)ny * nxl;
    zl.lstride = 1;
    zl.lines = min(W, nxl - i0);
    zl.tyj = __ldg(ty + j0 + j);  // j0: global index of the spectrum's first row
    zl.k2yj = __ldg(k2y + j0 + j);
    zl.ntot = ntot;
    zl.xtab = xtab;
    zl.ztab = tws + N;
    for (int t = threadIdx.x; t < 2 * N; t += kZftThreads) tws[t] = __ldg(tw + t);
    if (threadIdx.x < W) {  // ig0 + i0: global index of the tile's first lane
        const int i = min(ig0 + i0 + (int)threadIdx.x, nxh - 1);
        xtab[threadIdx.x] = make_double2(__ldg(tx + i), __ldg(k2x + i));
    }
    __syncthreads();
    zft<N, W, false>(zbuf, tws, zl);  // and the inverse, from its fused first stage
}

// The z lengths with a fused kernel.
#define X3D_ZFT_SIZES(X) X(8) X(12) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024)

static bool zft_supported(int n)
{
#define X3D_ZFT_CASE(N) \
    if (n == N) return true;
    X3D_ZFT_SIZES(X3D_ZFT_CASE)
#undef X3D_ZFT_CASE
    return false;
}

// ---------------------------------------------------------------------------
// Own x transforms: a real line of n = 2M points as the complex line z[m] =
// f[2m] + i f[2m+1] of M points (the same memory), transformed by the
// Stockham stages above, then split into the n/2 + 1 modes of the real
// transform -- the half-length method for real sequences (Brigham, "The
// Fast Fourier Transform", ch. 10; Press et al., Numerical Recipes, 12.3):
// with Z = DFT_M(z), A = Z[k], B = conj(Z[M - k]) (indices mod M),
//   F[k] = (A + B) / 2 - i e^{-2 pi i k / n} (A - B) / 2,   k = 0 .. M.
// The inverse runs it backwards: from G[0 .. M] (a Hermitian half spectrum)
//   Z[k] = (G[k] + conj(G[M - k])) + i e^{+2 pi i k / n} (G[k] - conj(G[M - k])),
// k < M, and the unnormalised inverse DFT_M of Z is f[2m] + i f[2m+1], the
// unnormalised c2r transform of G (cuFFT's Z2D convention).  Tiles are W
// consecutive y rows of one z plane; the spectrum is stored (nz, M + 1, ny)
// with y fastest, so a mode of the tile's rows is one run of W elements.

// Rows per tile of the x kernels: 4, so that a warp's first-stage loads
// take 4 rows x 8 consecutive points (128 bytes of each row), and threads
// enough for the tile's values in one pass of every stage (8 a thread; 6
// where a radix-3 stage takes two triples a thread), at least one warp.
constexpr int kXftW = 4;
template <int M>
constexpr int kXftThreads = (((M % 3 ? kXftW * M / 8 : kXftW * M / 6) + 31) / 32) * 32;

// The last radix R of a length-M forward transform (the first of the
// inverse).  Where R <= 4 and M / R is even, the split runs inside the last
// forward stage and the merge inside the first inverse one: the partner M - k
// of a mode k = j + q M/R (0 < j < M/R) is mode (M/R - j) + (R - 1 - q) M/R,
// an output of butterfly M/R - j, and butterfly 0 holds its own partners
// (q -> R - q); so one thread takes butterflies j and M/R - j (0 and M/(2R)
// together) and splits or merges in registers, one shared-memory pass fewer
// each way.  Radix-8 last stages keep the separate pass (16 complex values a
// thread do not fit the 64 registers).
template <int M>
constexpr int kXftLastR = radix_seq(M).r[radix_seq(M).count - 1];
template <int M>
constexpr bool kXftPaired = kXftLastR<M> <= 4 && (M / kXftLastR<M>) % 2 == 0;

// F[k] = (A + B) / 2 - i w (A - B) / 2 with B = conj(zp), w = e^{-2 pi i k / n}
__device__ __forceinline__ double2 split_mode(double2 a, double2 zp, double2 w)
{
    const double2 e = make_double2(0.5 * (a.x + zp.x), 0.5 * (a.y - zp.y));
    const double2 d = make_double2(0.5 * (a.x - zp.x), 0.5 * (a.y + zp.y));
    const double2 wd = cmul(w, d);
    return make_double2(e.x + wd.y, e.y - wd.x);
}

// Z[k] = (G[k] + conj(gp)) + i conj(w) (G[k] - conj(gp)), gp = G[M - k]
__device__ __forceinline__ double2 merge_mode(double2 g, double2 gp, double2 w)
{
    const double2 e = make_double2(g.x + gp.x, g.y - gp.y);
    const double2 d = make_double2(g.x - gp.x, g.y + gp.y);
    const double2 od = cmul(make_double2(w.x, -w.y), d);
    return make_double2(e.x - od.y, e.y + od.x);
}

// e^{-i pi q / R}, q < R: the factor between e^{-2 pi i j / n} and
// e^{-2 pi i (j + q M/R) / n} (n = 2M), so a butterfly's split or merge
// reads one table entry and scales it (q is a constant once unrolled).
template <int R>
__device__ __forceinline__ double2 half_turn(int q)
{
    constexpr double s2 = 0.70710678118654752440;  // sqrt(1/2)
    constexpr double s3 = 0.86602540378443864676;  // sqrt(3)/2
    if (q == 0) return make_double2(1.0, 0.0);
    if constexpr (R == 2) return make_double2(0.0, -1.0);
    if constexpr (R == 3) return q == 1 ? make_double2(0.5, -s3) : make_double2(-0.5, -s3);
    return q == 1 ? make_double2(s2, -s2) : (q == 2 ? make_double2(0.0, -1.0) : make_double2(-s2, -s2));
}

// Butterfly j of the last forward stage (sub-transforms of M/R, twiddle
// stride 1) for line l: y[q] = Z[j + q M/R].
template <int M, int R, int W>
__device__ __forceinline__ void last_butterfly(const double2 *buf, const double2 *tw, int j, int l, double2 (&y)[R])
{
    constexpr int NSL = M / R;
    const double2 w1 = tw[j];
    double2 wq = w1;
#pragma unroll
    for (int q = 0; q < R; ++q) {
        const double2 x = buf[(j + q * NSL) * W + l];
        if (q == 0) {
            y[q] = x;
        } else {
            y[q] = cmul(x, wq);
            wq = cmul(wq, w1);
        }
    }
    dft<R, false>(y);
}

template <int M>
__global__ void __launch_bounds__(kXftThreads<M>, 1024 / kXftThreads<M>)
    k_rfft_x(const double *__restrict__ f, double2 *__restrict__ spec, int ny, const double2 *__restrict__ tw)
{
    constexpr int W = kXftW;
    constexpr int NT = kXftThreads<M>;
    extern __shared__ __align__(16) double2 zbuf[];
    const double2 *const wx = tw + M;  // the tables are read through L1
    const int tiles_j = (ny + W - 1) / W;
    const int kz = blockIdx.x / tiles_j;
    const int j0 = (blockIdx.x - kz * tiles_j) * W;
    ZLines zl;
    zl.base = const_cast<double2 *>(reinterpret_cast<const double2 *>(f)) + ((size_t)kz * ny + j0) * M;
    zl.zstride = 1;
    zl.lstride = M;
    zl.lines = min(W, ny - j0);
    double2 *const out = spec + (size_t)kz * (M + 1) * ny + j0;
    if constexpr (kXftPaired<M>) {
        constexpr RadixSeq seq = radix_seq(M);
        constexpr int R = kXftLastR<M>, NSL = M / R;
        zft<M, W, false, false, NT, 0, 1, seq.count - 1>(zbuf, tw, zl);  // every stage but the last
        for (int it = threadIdx.x; it < W * (NSL / 2); it += NT) {
            const int l = it % W, i = it / W;
            if (l >= zl.lines) continue;
            const int a = i, b = i > 0 ? NSL - i : NSL / 2;  // butterflies a and b, partners of each other
            double2 ya[R], yb[R];
            last_butterfly<M, R, W>(zbuf, tw, a, l, ya);
            last_butterfly<M, R, W>(zbuf, tw, b, l, yb);
            const double2 wa = __ldg(wx + a), wb = __ldg(wx + b);
#pragma unroll
            for (int q = 0; q < R; ++q) {
                // Z[M - k] of k = a + q M/R and of k = b + q M/R
                const double2 pa = i > 0 ? yb[R - 1 - q] : ya[(R - q) % R];
                const double2 pb = i > 0 ? ya[R - 1 - q] : yb[R - 1 - q];
                const double2 h = half_turn<R>(q);
                out[(size_t)(a + q * NSL) * ny + l] = split_mode(ya[q], pa, q ? cmul(wa, h) : wa);
                out[(size_t)(b + q * NSL) * ny + l] = split_mode(yb[q], pb, q ? cmul(wb, h) : wb);
            }
            if (i == 0) out[(size_t)M * ny + l] = split_mode(ya[0], ya[0], make_double2(-1.0, 0.0));
        }
        return;
    }
    zft<M, W, false, false, NT>(zbuf, tw, zl);  // Z of each row, natural order, in zbuf
    for (int b = threadIdx.x; b < (M / 2 + 1) * W; b += NT) {
        const int l = b % W, p = b / W, q = (M - p) % M;  // modes p and M - p from Z[p] and Z[q]
        if (l >= zl.lines) continue;
        const double2 zp = zbuf[p * W + l], zq = zbuf[q * W + l];
        const double2 wp = __ldg(wx + p), wq = __ldg(wx + M - p);
        // F[p]: A = Z[p], B = conj(Z[q]);  F[M - p]: A = Z[q], B = conj(Z[p])
        const double2 e = make_double2(0.5 * (zp.x + zq.x), 0.5 * (zp.y - zq.y));  // (A + B) / 2 of F[p]
        const double2 d = make_double2(0.5 * (zp.x - zq.x), 0.5 * (zp.y + zq.y));  // (A - B) / 2 of F[p]
        const double2 wd = cmul(wp, d);
        out[(size_t)p * ny + l] = make_double2(e.x + wd.y, e.y - wd.x);
        if (M - p != p) {  // F[M - p]: (A + B) / 2 = conj(e), (A - B) / 2 = -conj(d)
            const double2 wd2 = cmul(wq, make_double2(-d.x, d.y));
            out[(size_t)(M - p) * ny + l] = make_double2(e.x + wd2.y, -e.y - wd2.x);
        }
    }
}

template <int M>
__global__ void __launch_bounds__(kXftThreads<M>, 1024 / kXftThreads<M>)
    k_irfft_x(const double2 *__restrict__ spec, double *__restrict__ f, int ny, const double2 *__restrict__ tw)
{
    constexpr int W = kXftW;
    constexpr int NT = kXftThreads<M>;
    extern __shared__ __align__(16) double2 zbuf[];
    const double2 *const wx = tw + M;  // the tables are read through L1
    const int tiles_j = (ny + W - 1) / W;
    const int kz = blockIdx.x / tiles_j;
    const int j0 = (blockIdx.x - kz * tiles_j) * W;
    const int lines = min(W, ny - j0);
    const double2 *const in = spec + (size_t)kz * (M + 1) * ny + j0;
    ZLines zl;
    zl.base = reinterpret_cast<double2 *>(f) + ((size_t)kz * ny + j0) * M;
    zl.zstride = 1;
    zl.lstride = M;
    zl.lines = lines;
    if constexpr (kXftPaired<M>) {
        constexpr int R = kXftLastR<M>, NSL = M / R;  // the inverse's first radix
        static_assert(radix_seq(M, true).r[0] == R, "the inverse takes the radices in reverse order");
        for (int it = threadIdx.x; it < W * (NSL / 2); it += NT) {
            const int l = it % W, i = it / W;
            const int a = i, b = i > 0 ? NSL - i : NSL / 2;
            double2 ga[R], gb[R], gm = make_double2(0.0, 0.0);
#pragma unroll
            for (int q = 0; q < R; ++q) ga[q] = gb[q] = gm;
            if (l < lines) {
#pragma unroll
                for (int q = 0; q < R; ++q) {
                    ga[q] = in[(size_t)(a + q * NSL) * ny + l];
                    gb[q] = in[(size_t)(b + q * NSL) * ny + l];
                }
                if (i == 0) gm = in[(size_t)M * ny + l];
            }
            // merged in place, a mode and its partner together; the table
            // entry of mode j + q M/R is wx[j] times half_turn(q)
            const double2 wa = __ldg(wx + a), wb = __ldg(wx + b);
            auto pair = [&](double2 &g1, double2 &g2, double2 w1, double2 w2, bool self) {
                const double2 x1 = g1, x2 = g2;
                g1 = merge_mode(x1, x2, w1);
                if (!self) g2 = merge_mode(x2, x1, w2);
            };
            auto scaled = [](double2 w, int q, double2 h) { return q ? cmul(w, h) : w; };
            if (i > 0) {  // partner of a + q M/R is b + (R - 1 - q) M/R
#pragma unroll
                for (int q = 0; q < R; ++q)
                    pair(ga[q], gb[R - 1 - q], scaled(wa, q, half_turn<R>(q)),
                         scaled(wb, R - 1 - q, half_turn<R>(R - 1 - q)), false);
            } else {  // butterfly 0: q M/R and (R - q) M/R, and 0 with M; butterfly M/(2R) as above
                const double2 g0 = merge_mode(ga[0], gm, make_double2(1.0, 0.0));
#pragma unroll
                for (int q = 1; 2 * q <= R; ++q)
                    pair(ga[q], ga[R - q], half_turn<R>(q), half_turn<R>(R - q), 2 * q == R);
                ga[0] = g0;
#pragma unroll
                for (int q = 0; 2 * q < R; ++q)
                    pair(gb[q], gb[R - 1 - q], scaled(wb, q, half_turn<R>(q)),
                         scaled(wb, R - 1 - q, half_turn<R>(R - 1 - q)), 2 * q == R - 1);
            }
            dft<R, true>(ga);  // the inverse's first stage: sub-transforms of size 1, no twiddles
            dft<R, true>(gb);
#pragma unroll
            for (int q = 0; q < R; ++q) {
                zbuf[(a * R + q) * W + l] = ga[q];
                zbuf[(b * R + q) * W + l] = gb[q];
            }
        }
        __syncthreads();
        zft<M, W, true, false, NT, 1, R>(zbuf, tw, zl);  // the inverse from its second stage
        return;
    }
    for (int b = threadIdx.x; b < (M / 2 + 1) * W; b += NT) {
        const int l = b % W, p = b / W, q = M - p;  // Z[p] and Z[q] (q < M) from G[p] and G[q]
        double2 gp = make_double2(0.0, 0.0), gq = gp;
        if (l < lines) {
            gp = in[(size_t)p * ny + l];
            gq = in[(size_t)q * ny + l];
        }
        // Z[p] = (G[p] + conj(G[q])) + i conj(wx[p]) (G[p] - conj(G[q]))
        const double2 e = make_double2(gp.x + gq.x, gp.y - gq.y);
        const double2 d = make_double2(gp.x - gq.x, gp.y + gq.y);
        const double2 w = __ldg(wx + p);
        const double2 od = cmul(make_double2(w.x, -w.y), d);
        zbuf[p * W + l] = make_double2(e.x - od.y, e.y + od.x);
        if (q != p && q < M) {  // Z[q] = (G[q] + conj(G[p])) + i conj(wx[q]) (G[q] - conj(G[p]))
            const double2 w2 = __ldg(wx + q);
            const double2 od2 = cmul(make_double2(w2.x, -w2.y), make_double2(-d.x, d.y));
            zbuf[q * W + l] = make_double2(e.x - od2.y, -e.y + od2.x);
        }
    }
    __syncthreads();
    zft<M, W, true, false, NT>(zbuf, tw, zl);  // the inverse, its last stage to the rows
}

// The 1-D modified-wavenumber tables and, where a fused z kernel exists for
// nz, its twiddles: all that the z part of the solve reads.
static int poisson_tables(x3d_ctx_s *ctx)
{
    if (ctx->d_k2x) return X3D_OK;
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
    if (cudaMemcpy(tab, h.data(), tot * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(tab);
        return set_error(ctx, X3D_ECUDA, "poisson tables upload");
    }
    ctx->d_k2x = tab;
    ctx->d_tx = tab + nx;
    ctx->d_k2y = tab + 2 * nx;
    ctx->d_ty = tab + 2 * nx + ny;
    ctx->d_k2z = tab + 2 * nx + 2 * ny;
    ctx->d_tz = tab + 2 * nx + 2 * ny + nz;
    if (zft_supported(nz)) {  // the twiddles, then (tz, k2z) of each z mode
        std::vector<double> tw(4 * (size_t)nz);
        const double twopi = 2.0 * std::acos(-1.0);
        for (int t = 0; t < nz; ++t) {
            tw[2 * t] = std::cos(twopi * t / nz);
            tw[2 * t + 1] = -std::sin(twopi * t / nz);
            tw[2 * ((size_t)nz + t)] = tz[t];
            tw[2 * ((size_t)nz + t) + 1] = k2z[t];
        }
        if (cudaMalloc(&ctx->d_zft_tw, tw.size() * sizeof(double)) != cudaSuccess)
            return set_error(ctx, X3D_ENOMEM, "poisson twiddles");
        if (cudaMemcpy(ctx->d_zft_tw, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
            cudaFree(ctx->d_zft_tw);
            ctx->d_zft_tw = nullptr;
            return set_error(ctx, X3D_ECUDA, "poisson twiddles upload");
        }
    }
    if (nx % 2 == 0 && zft_supported(nx / 2)) {
        const int m = nx / 2;
        const double twopi = 2.0 * std::acos(-1.0);
        std::vector<double> tw(2 * (size_t)(2 * m + 1));
        for (int t = 0; t < m; ++t) {
            tw[2 * t] = std::cos(twopi * t / m);
            tw[2 * t + 1] = -std::sin(twopi * t / m);
        }
        for (int k = 0; k <= m; ++k) {
            tw[2 * (m + k)] = std::cos(twopi * k / nx);
            tw[2 * (m + k) + 1] = -std::sin(twopi * k / nx);
        }
        if (cudaMalloc(&ctx->d_xft_tw, tw.size() * sizeof(double)) != cudaSuccess) {
            ctx->d_xft_tw = nullptr;
            return set_error(ctx, X3D_ENOMEM, "poisson x twiddles");
        }
        if (cudaMemcpy(ctx->d_xft_tw, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
            cudaFree(ctx->d_xft_tw);
            ctx->d_xft_tw = nullptr;
            return set_error(ctx, X3D_ECUDA, "poisson x twiddles upload");
        }
    }
    return X3D_OK;
}

// Whether a solve on this context takes the own x transforms: the fused z
// kernel and a fused length nx / 2, unless the stage choice "poisson_x" is 0.
static bool poisson_own_x(const x3d_ctx_s *ctx)
{
    const auto it = ctx->stage_tuned.find("poisson_x");
    return ctx->zfused && ctx->d_xft_tw && (it == ctx->stage_tuned.end() || it->second != 0);
}

int poisson_setup(x3d_ctx_s *ctx)
{
    if (!ctx->spectrum) {
        int rc = poisson_tables(ctx);
        if (rc) return rc;
        const size_t spec = (size_t)ctx->nz * ctx->ny * (ctx->nx / 2 + 1) * sizeof(double2);
        if (cudaMalloc(&ctx->spectrum, spec) != cudaSuccess) {
            ctx->spectrum = nullptr;
            return set_error(ctx, X3D_ENOMEM, "poisson spectrum");
        }
        ctx->zfused = ctx->d_zft_tw && ctx->zfuse_allowed;
    }
    const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    if (poisson_own_x(ctx)) {
        if (ctx->plan_y_ready) return X3D_OK;
        int n = ny;
        if (cufftPlanMany(&ctx->plan_y, 1, &n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2Z, nz * (nx / 2 + 1)) !=
            CUFFT_SUCCESS)
            return set_error(ctx, X3D_ECUDA, "cufftPlanMany (y lines) failed");
        ctx->plan_y_ready = true;
        return X3D_OK;
    }
    if (ctx->plans_ready) return X3D_OK;
    if (ctx->zfused) {
        int dims[2] = {ny, nx};
        if (cufftPlanMany(&ctx->plan_d2z, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, nz) != CUFFT_SUCCESS ||
            cufftPlanMany(&ctx->plan_z2d, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, nz) != CUFFT_SUCCESS)
            return set_error(ctx, X3D_ECUDA, "cufftPlanMany failed");
    } else if (cufftPlan3d(&ctx->plan_d2z, nz, ny, nx, CUFFT_D2Z) != CUFFT_SUCCESS ||
               cufftPlan3d(&ctx->plan_z2d, nz, ny, nx, CUFFT_Z2D) != CUFFT_SUCCESS) {
        return set_error(ctx, X3D_ECUDA, "cufftPlan3d failed");
    }
    ctx->plans_ready = true;
    return X3D_OK;
}

// The fused z kernel over a spectrum of nxl lanes (the fastest index)
// starting at global index i0, ny_loc rows starting at global row j0 and nz
// planes; lanes and rows are x modes and y rows ((nz, ny_loc, nxl)) unless
// yfast, where they are y rows and x modes ((nz, nxh, ny)).
static int launch_poisson_z(x3d_ctx_s *ctx, double2 *spec, int nxl, int i0, int ny_loc, int j0, bool yfast = false)
{
    const int nxh = ctx->nx / 2 + 1;
    const double ntot = (double)ctx->nx * (double)ctx->ny * (double)ctx->nz;
    const double *lk2 = yfast ? ctx->d_k2y : ctx->d_k2x, *lt = yfast ? ctx->d_ty : ctx->d_tx;
    const double *rk2 = yfast ? ctx->d_k2x : ctx->d_k2y, *rt = yfast ? ctx->d_tx : ctx->d_ty;
    const int lane_end = yfast ? ctx->ny : nxh;
    const auto *ztw = reinterpret_cast<const double2 *>(ctx->d_zft_tw);
    auto go = [&](auto kern, int W, int NT) {
        const unsigned grid = (unsigned)(((nxl + W - 1) / W) * ny_loc);
        // tile, twiddles, z and lane wavenumber tables
        const size_t smem = ((size_t)ctx->nz * W + 2 * (size_t)ctx->nz + W) * sizeof(double2);
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        ++ctx->launches;
        kern<<<grid, NT, smem, ctx->stream>>>(spec, nxl, ny_loc, i0, j0, lane_end, ztw, lk2, lt, rk2, rt, ntot);
        return cuda_check(ctx, cudaGetLastError(), "k_poisson_z");
    };
    switch (ctx->nz) {
#define X3D_ZFT_LAUNCH(N) \
    case N: return go(k_poisson_z<N>, kZftW<N>, kZftThreads);
        X3D_ZFT_SIZES(X3D_ZFT_LAUNCH)
#undef X3D_ZFT_LAUNCH
    default: return set_error(ctx, X3D_EUNSUPPORTED, "no fused z transform for this nz");
    }
}

// k_rfft_x (forward) or k_irfft_x over the whole box: real (nz, ny, nx) and
// the spectrum (nz, nx/2 + 1, ny).
static int launch_xft(x3d_ctx_s *ctx, double *f, double2 *spec, bool forward)
{
    auto go = [&](auto fwd, auto inv, int M, int NT) {
        const int W = kXftW;
        const unsigned grid = (unsigned)(((ctx->ny + W - 1) / W) * ctx->nz);
        const size_t smem = (size_t)M * W * sizeof(double2);  // the tile
        const auto *tw = reinterpret_cast<const double2 *>(ctx->d_xft_tw);
        ++ctx->launches;
        if (forward) {
            cudaFuncSetAttribute(fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            fwd<<<grid, NT, smem, ctx->stream>>>(f, spec, ctx->ny, tw);
        } else {
            cudaFuncSetAttribute(inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            inv<<<grid, NT, smem, ctx->stream>>>(spec, f, ctx->ny, tw);
        }
        return cuda_check(ctx, cudaGetLastError(), forward ? "k_rfft_x" : "k_irfft_x");
    };
    switch (ctx->nx / 2) {
#define X3D_XFT_LAUNCH(N) \
    case N: return go(k_rfft_x<N>, k_irfft_x<N>, N, kXftThreads<N>);
        X3D_ZFT_SIZES(X3D_XFT_LAUNCH)
#undef X3D_XFT_LAUNCH
    default: return set_error(ctx, X3D_EUNSUPPORTED, "no own x transform for this nx");
    }
}

// k_spectral_divide over n modes of a block (see there), grid-strided.
static int launch_divide(x3d_ctx_s *ctx, double2 *c, int nxl, int nyl, size_t n, int i0, int j0)
{
    if (n >= (1ull << 31)) return set_error(ctx, X3D_EUNSUPPORTED, "spectrum above 2^31 modes");
    const int bs = 256;
    size_t g = (n + bs - 1) / bs;
    const size_t cap = (size_t)ctx->num_sms * 8;
    if (g > cap) g = cap;
    const double ntot = (double)ctx->nx * (double)ctx->ny * (double)ctx->nz;
    ++ctx->launches;
    k_spectral_divide<<<(unsigned)g, bs, 0, ctx->stream>>>(c, (unsigned)nxl, (unsigned)nyl, (unsigned)n,
                                                           (unsigned)i0, (unsigned)j0, ctx->d_k2x, ctx->d_tx,
                                                           ctx->d_k2y, ctx->d_ty, ctx->d_k2z, ctx->d_tz, ntot);
    return cuda_check(ctx, cudaGetLastError(), "k_spectral_divide");
}

int poisson_solve(x3d_ctx_s *ctx, double *rhs)
{
    const TraceRange trace("poisson");
    int rc = poisson_setup(ctx);
    if (rc) return rc;
    if (poisson_own_x(ctx)) {
        // x transforms (spectrum y fastest), y transforms, z solve, and back
        auto *spec = static_cast<double2 *>(ctx->spectrum);
        auto *cs = reinterpret_cast<cufftDoubleComplex *>(spec);
        cufftSetStream(ctx->plan_y, ctx->stream);
        rc = launch_xft(ctx, rhs, spec, true);
        if (rc) return rc;
        if (cufftExecZ2Z(ctx->plan_y, cs, cs, CUFFT_FORWARD) != CUFFT_SUCCESS)
            return set_error(ctx, X3D_ECUDA, "cufftExecZ2Z (y lines, forward) failed");
        rc = launch_poisson_z(ctx, spec, ctx->ny, 0, ctx->nx / 2 + 1, 0, true);
        if (rc) return rc;
        if (cufftExecZ2Z(ctx->plan_y, cs, cs, CUFFT_INVERSE) != CUFFT_SUCCESS)
            return set_error(ctx, X3D_ECUDA, "cufftExecZ2Z (y lines, inverse) failed");
        return launch_xft(ctx, rhs, spec, false);
    }
    cufftSetStream(ctx->plan_d2z, ctx->stream);
    cufftSetStream(ctx->plan_z2d, ctx->stream);
    if (cufftExecD2Z(ctx->plan_d2z, rhs, (cufftDoubleComplex *)ctx->spectrum) != CUFFT_SUCCESS)
        return set_error(ctx, X3D_ECUDA, "cufftExecD2Z failed");
    if (ctx->zfused) {
        rc = launch_poisson_z(ctx, (double2 *)ctx->spectrum, ctx->nx / 2 + 1, 0, ctx->ny, 0);
        if (rc) return rc;
        if (cufftExecZ2D(ctx->plan_z2d, (cufftDoubleComplex *)ctx->spectrum, rhs) != CUFFT_SUCCESS)
            return set_error(ctx, X3D_ECUDA, "cufftExecZ2D failed");
        return X3D_OK;
    }
    const int nxh = ctx->nx / 2 + 1;
    rc = launch_divide(ctx, (double2 *)ctx->spectrum, nxh, ctx->ny, (size_t)nxh * ctx->ny * ctx->nz, 0, 0);
    if (rc) return rc;
    if (cufftExecZ2D(ctx->plan_z2d, (cufftDoubleComplex *)ctx->spectrum, rhs) != CUFFT_SUCCESS)
        return set_error(ctx, X3D_ECUDA, "cufftExecZ2D failed");
    return X3D_OK;
}

// The z part of the spectral solve on a block of x modes and y rows of the
// x-y transformed spectrum, for a box spread over ranks.  Needs only the
// wavenumber tables and twiddles: no plans or spectrum of the whole box.
// z lengths without a fused kernel take batched 1-D cuFFT transforms along
// z (one plan per block shape, kept), k_spectral_divide on the block and
// the inverse transforms.
int poisson_zpencil(x3d_ctx_s *ctx, void *spec, int nxl, int i0, int ny_loc, int j0)
{
    int rc = poisson_tables(ctx);
    if (rc) return rc;
    if (ny_loc < 1 || j0 < 0 || j0 + ny_loc > ctx->ny) return set_error(ctx, X3D_EINVAL, "bad block of y rows");
    if (nxl < 1 || i0 < 0 || i0 + nxl > ctx->nx / 2 + 1) return set_error(ctx, X3D_EINVAL, "bad block of x modes");
    double2 *c = static_cast<double2 *>(spec);
    if (ctx->d_zft_tw) return launch_poisson_z(ctx, c, nxl, i0, ny_loc, j0);
    if (!ctx->zblk_ready || ctx->zblk_nxl != nxl || ctx->zblk_nyl != ny_loc) {
        if (ctx->zblk_ready) cufftDestroy(ctx->plan_zblk);
        ctx->zblk_ready = false;
        int n = ctx->nz, emb = ctx->nz;
        const int lines = nxl * ny_loc;
        if (cufftPlanMany(&ctx->plan_zblk, 1, &n, &emb, lines, 1, &emb, lines, 1, CUFFT_Z2Z, lines) !=
            CUFFT_SUCCESS)
            return set_error(ctx, X3D_ECUDA, "cufftPlanMany (z lines of a block) failed");
        ctx->zblk_ready = true;
        ctx->zblk_nxl = nxl;
        ctx->zblk_nyl = ny_loc;
    }
    cufftSetStream(ctx->plan_zblk, ctx->stream);
    auto *cz = reinterpret_cast<cufftDoubleComplex *>(c);
    if (cufftExecZ2Z(ctx->plan_zblk, cz, cz, CUFFT_FORWARD) != CUFFT_SUCCESS)
        return set_error(ctx, X3D_ECUDA, "cufftExecZ2Z (forward z) failed");
    rc = launch_divide(ctx, c, nxl, ny_loc, (size_t)nxl * ny_loc * ctx->nz, i0, j0);
    if (rc) return rc;
    if (cufftExecZ2Z(ctx->plan_zblk, cz, cz, CUFFT_INVERSE) != CUFFT_SUCCESS)
        return set_error(ctx, X3D_ECUDA, "cufftExecZ2Z (inverse z) failed");
    return X3D_OK;
}

// ---- non-periodic directions ------------------------------------------------
//
// decomp_2d_poisson_init gives the pressure bc = 1 along every non-periodic
// direction (src/poisson.f90:85-99, m = n - 1 pressure points,
// :114-117) and tabulates that case in waves() (:539-553, :573-588,
// :603-613): the cosine modes i = 0 .. m of w = pi i / m, i.e. homogeneous
// Neumann conditions at the walls, half a cell beyond the first and last
// pressure points.  x3div stops there (:104-108).  Here the solve is the
// periodic one on the box mirrored about both walls of each such direction
// (2 m points over twice the length): the mirrored field is even about the
// walls, so it holds exactly those cosine modes, whose modified wavenumbers
// on the doubled grid (w = 2 pi i / 2m, spacing 2L / 2m) are waves()'s bc = 1
// values, and the periodic solution is even too; its first m points are
// the solution.  The periodic solve is the library's (cuFFT 2-D transforms
// and the fused z kernel); mirroring and cutting back are one pass each.

// ext (Mx, My, Mz) from p (mx, my, mz): M = 2m along a mirrored direction,
// M = m otherwise.
__global__ void k_mirror_extend(double *__restrict__ ext, const double *__restrict__ p, int mx, int my, int mz,
                                int Mx, int My, int Mz)
{
    const size_t total = (size_t)Mx * My * Mz;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int X = (int)(e % Mx);
        const size_t t = e / Mx;
        const int Y = (int)(t % My), Z = (int)(t / My);
        const int i = X < mx ? X : 2 * mx - 1 - X;
        const int j = Y < my ? Y : 2 * my - 1 - Y;
        const int k = Z < mz ? Z : 2 * mz - 1 - Z;
        ext[e] = p[(size_t)i + (size_t)mx * ((size_t)j + (size_t)my * k)];
    }
}

// p (mx, my, mz) = the first m points of ext along each direction.
__global__ void k_mirror_restrict(double *__restrict__ p, const double *__restrict__ ext, int mx, int my, int mz,
                                  int Mx, int My)
{
    const size_t total = (size_t)mx * my * mz;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % mx);
        const size_t t = e / mx;
        const int j = (int)(t % my), k = (int)(t / my);
        p[e] = ext[(size_t)i + (size_t)Mx * ((size_t)j + (size_t)My * k)];
    }
}

int poisson_solve_mirror(x3d_ctx_s *ctx, double *rhs)
{
    const TraceRange trace("poisson (mirrored)");
    int m[3], M[3];
    double len[3] = {ctx->xlx, ctx->yly, ctx->zlz};
    for (int d = 0; d < 3; ++d) {
        m[d] = ctx->pdim(d);
        const bool per = ctx->ncl[2 * d] == 0 && ctx->ncl[2 * d + 1] == 0;
        M[d] = per ? m[d] : 2 * m[d];
        if (!per) len[d] *= 2.0;
    }
    if (!ctx->mirror) {
        x3d_ctx_s *mc = nullptr;
        const int rc = x3d_ctx_create(&mc, M[0], M[1], M[2], len[0], len[1], len[2], X3D_F64, ctx->device);
        if (rc) return set_error(ctx, rc, "the mirrored box's periodic context could not be made (mirrored "
                                          "lengths must be at least 8 points)");
        ctx->mirror = mc;
    }
    if (!ctx->mirror_rhs &&
        cudaMalloc(&ctx->mirror_rhs, sizeof(double) * (size_t)M[0] * M[1] * M[2]) != cudaSuccess) {
        ctx->mirror_rhs = nullptr;
        return set_error(ctx, X3D_ENOMEM, "mirrored right-hand side allocation failed");
    }
    x3d_ctx_s *mc = ctx->mirror;
    mc->stream = ctx->stream;  // the mirrored solve runs in order with the caller's work
    const size_t total = (size_t)M[0] * M[1] * M[2];
    const unsigned grid = (unsigned)std::min<size_t>((total + 255) / 256, (size_t)ctx->num_sms * 8);
    ++ctx->launches;
    k_mirror_extend<<<grid, 256, 0, ctx->stream>>>(ctx->mirror_rhs, rhs, m[0], m[1], m[2], M[0], M[1], M[2]);
    int rc = cuda_check(ctx, cudaGetLastError(), "k_mirror_extend");
    if (rc) return rc;
    const unsigned long long l0 = mc->launches;
    rc = poisson_solve(mc, ctx->mirror_rhs);
    ctx->launches += mc->launches - l0;
    if (rc) return set_error(ctx, rc, mc->last_error);
    ++ctx->launches;
    k_mirror_restrict<<<grid, 256, 0, ctx->stream>>>(rhs, ctx->mirror_rhs, m[0], m[1], m[2], M[0], M[1]);
    return cuda_check(ctx, cudaGetLastError(), "k_mirror_restrict");
}

void poisson_free(x3d_ctx_s *ctx)
{
    if (ctx->mirror) x3d_ctx_destroy(ctx->mirror);
    ctx->mirror = nullptr;
    if (ctx->mirror_rhs) cudaFree(ctx->mirror_rhs);
    ctx->mirror_rhs = nullptr;
    if (ctx->plans_ready) {
        cufftDestroy(ctx->plan_d2z);
        cufftDestroy(ctx->plan_z2d);
    }
    ctx->plans_ready = false;
    if (ctx->spectrum) cudaFree(ctx->spectrum);
    ctx->spectrum = nullptr;
    if (ctx->d_k2x) cudaFree(ctx->d_k2x);
    ctx->d_k2x = nullptr;
    if (ctx->d_zft_tw) cudaFree(ctx->d_zft_tw);
    ctx->d_zft_tw = nullptr;
    if (ctx->d_xft_tw) cudaFree(ctx->d_xft_tw);
    ctx->d_xft_tw = nullptr;
    if (ctx->plan_y_ready) cufftDestroy(ctx->plan_y);
    ctx->plan_y_ready = false;
    ctx->zfused = false;
    if (ctx->zblk_ready) cufftDestroy(ctx->plan_zblk);
    ctx->zblk_ready = false;
}

}  // namespace x3d
