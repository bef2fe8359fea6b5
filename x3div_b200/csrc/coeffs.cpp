// FP64 operator precompute, done once per context on the host: the
// x3d_operator_1d_init path of the reference (src/x3d_operator_1d.f90:59-195)
// for fully periodic boundaries, plus the two vectors the single-pass GPU
// sweep needs (g = first row of M^-1 and the Sherman-Morrison denominator).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "x3d_internal.h"

namespace x3d {

// Explicit RHS scalars (the module globals of x3d_operator_{x,y,z}_data).
//  DER:   first_deriv_exp_ with ifirstder = 4 (src/x3d_operator_1d.f90:350-353)
//  DERVP, DERPV: interpol_exp_ staggered derivative (:510-512)
//  INTVP, INTPV: interpol_exp_ with ipinter = 3 (:539-544)
//  DER2:  Lele (1992) sixth-order compact second derivative (alpha = 2/11,
//         a = 12/11, b = 3/11 in Lele's notation, i.e. asix = (12/11)/d^2 and
//         bsix = (3/44)/d^2 on the (u(i+2) - 2u(i) + u(i-2)) difference).
//         The reference declares its scalars (alsaix, asix, bsix) and arrays
//         (sfx, ssx, swx) but never fills them.
void rhs_scalars(int kind, double d, double *alfa, double *a, double *b, double *c, double *dd)
{
    *alfa = *a = *b = *c = *dd = 0.0;
    switch (kind) {
    case DER:
        *alfa = 1.0 / 3.0;
        *a = (7.0 / 9.0) / d;
        *b = (1.0 / 36.0) / d;
        break;
    case DERVP:
    case DERPV:
        *alfa = 9.0 / 62.0;
        *a = (63.0 / 62.0) / d;
        *b = (17.0 / 62.0) / 3.0 / d;
        break;
    case INTVP:
    case INTPV: {
        const double al = 0.49;
        *alfa = al;
        *a = 1.0 / 128.0 * (75.0 + 70.0 * al);
        *b = 1.0 / 256.0 * (126.0 * al - 25.0);
        *c = 1.0 / 256.0 * (-10.0 * al + 3.0);
        *dd = 0.0;
        break;
    }
    case DER2:
        *alfa = 2.0 / 11.0;
        *a = (12.0 / 11.0) / (d * d);
        *b = (3.0 / 44.0) / (d * d);
        break;
    default:
        break;
    }
}

// Thomas LU of the tridiagonal (b, c, f): prepare (src/x3d_operator_1d.f90:301-323).
static void lu_prepare(const std::vector<double> &b, const std::vector<double> &c,
                       const std::vector<double> &f, std::vector<double> &s, std::vector<double> &w)
{
    const int n = (int)c.size();
    s.assign(n, 0.0);
    w = c;
    for (int i = 1; i < n; ++i) {
        s[i] = b[i - 1] / w[i - 1];
        w[i] = w[i] - f[i - 1] * s[i];
    }
    for (int i = 0; i < n; ++i) w[i] = 1.0 / w[i];
}

// In-place Thomas solve with the prepared factors (thomas1d, src/thomas.f90:200-218).
static void lu_solve(std::vector<double> &t, const std::vector<double> &f,
                     const std::vector<double> &s, const std::vector<double> &w)
{
    const int n = (int)t.size();
    for (int k = 1; k < n; ++k) t[k] -= t[k - 1] * s[k];
    t[n - 1] *= w[n - 1];
    for (int k = n - 2; k >= 0; --k) t[k] = (t[k] - f[k] * t[k + 1]) * w[k];
}

// Periodic operator: every family shares the reference's periodic matrix
// pattern (first_deriv_imp_ :414-445,467-471; interpol_imp_ :576-599 and
// :622-645): off-diagonals alpha, corner rows folded by Sherman-Morrison so
// that c(1) = 2, c(n) = 1 + alpha^2, f(n) = b(n) = 0.  The "p" copies
// (ffxp, cifxp6) equal these when periodic (:473-486, :667-676).
static void periodic_lu(int n, double al, std::vector<double> &f, std::vector<double> &s,
                        std::vector<double> &w, std::vector<double> &per)
{
    std::vector<double> fb(n, 0.0), fc(n, 0.0), ff(n, 0.0);
    ff[0] = al; ff[1] = al;
    fc[0] = 2.0; fc[1] = 1.0;
    fb[0] = al; fb[1] = al;
    ff[n - 3] = al; ff[n - 2] = al; ff[n - 1] = 0.0;
    fc[n - 3] = 1.0; fc[n - 2] = 1.0; fc[n - 1] = 1.0 + al * al;
    fb[n - 3] = al; fb[n - 2] = al; fb[n - 1] = 0.0;
    for (int i = 2; i < n - 3; ++i) {
        ff[i] = al;
        fc[i] = 1.0;
        fb[i] = al;
    }
    f = ff;
    lu_prepare(fb, fc, ff, s, w);
    // init(): periodic = M^-1 (-1, 0, ..., 0, alfa)  (:260-264)
    per.assign(n, 0.0);
    per[0] = -1.0;
    per[n - 1] = al;
    lu_solve(per, f, s, w);
}

int build_periodic_op(int kind, int dir, int n, double d, OpHost &op)
{
    if (n < 8) return X3D_EUNSUPPORTED;
    op.kind = kind;
    op.dir = dir;
    op.n = n;
    op.periodic = 1;
    op.npaire = (kind == DER || kind == DER2 || kind == DERPV) ? 0 : 1;
    rhs_scalars(kind, d, &op.alfa, &op.a, &op.b, &op.c, &op.d);
    periodic_lu(n, op.alfa, op.f, op.s, op.w, op.per);
    finish_op(op);
    return X3D_OK;
}

// Non-periodic sixth-order compact first derivative, ifirstder = 4
// (first_deriv_exp_ and first_deriv_imp_, src/x3d_operator_1d.f90:325-488):
// interior rows (alfa, 1, alfa); free-slip ends (ncl = 1) fold the symmetric
// ghost points into the first/last rows; Dirichlet ends (ncl = 2) use the
// third-order one-sided rows (alfa1 = 2, alfa2 = 1/4 and their mirror).
// The operator of parity npaire = 1 (derxp) uses the "p" factors, prepared
// from ff with ffp(1) = 0 at a free-slip start and fb(n-1) = 0 at a free-slip
// end (:477-486).
int build_nonperiodic_der(int dir, int n, double d, int ncl1, int ncln, int npaire, OpHost &op)
{
    if (n < 8 || ncl1 < 1 || ncl1 > 2 || ncln < 1 || ncln > 2) return X3D_EUNSUPPORTED;
    op.kind = DER;
    op.dir = dir;
    op.n = n;
    op.periodic = 0;
    op.npaire = npaire;
    op.ncl1 = ncl1;
    op.ncln = ncln;
    rhs_scalars(DER, d, &op.alfa, &op.a, &op.b, &op.c, &op.d);
    const double al = op.alfa;
    const double alfa1 = 2.0, alfa2 = 0.25, alfan = 2.0, alfam = 0.25;
    // af1, bf1, cf1, af2, afm, afn, bfn, cfn (:375-390)
    const double cl[8] = {-2.5 / d, 2.0 / d, 0.5 / d, 0.75 / d, 0.75 / d, -2.5 / d, 2.0 / d, 0.5 / d};
    for (int i = 0; i < 8; ++i) op.cl[i] = cl[i];
    std::vector<double> fb(n, 0.0), fc(n, 0.0), ff(n, 0.0);
    if (ncl1 == 1) {
        ff[0] = al + al; ff[1] = al;
        fc[0] = 1.0; fc[1] = 1.0;
        fb[0] = al; fb[1] = al;
    } else {
        ff[0] = alfa1; ff[1] = alfa2;
        fc[0] = 1.0; fc[1] = 1.0;
        fb[0] = alfa2; fb[1] = al;
    }
    if (ncln == 1) {
        ff[n - 3] = al; ff[n - 2] = al; ff[n - 1] = 0.0;
        fc[n - 3] = 1.0; fc[n - 2] = 1.0; fc[n - 1] = 1.0;
        fb[n - 3] = al; fb[n - 2] = al + al; fb[n - 1] = 0.0;
    } else {
        ff[n - 3] = al; ff[n - 2] = alfam; ff[n - 1] = 0.0;
        fc[n - 3] = 1.0; fc[n - 2] = 1.0; fc[n - 1] = 1.0;
        fb[n - 3] = alfam; fb[n - 2] = alfan; fb[n - 1] = 0.0;
    }
    for (int i = 2; i < n - 3; ++i) {
        ff[i] = al;
        fc[i] = 1.0;
        fb[i] = al;
    }
    if (npaire == 0) {
        op.f = ff;
        lu_prepare(fb, fc, ff, op.s, op.w);
    } else {
        std::vector<double> ffp = ff;
        if (ncl1 == 1) ffp[0] = 0.0;
        if (ncln == 1) fb[n - 2] = 0.0;
        op.f = ffp;
        lu_prepare(fb, fc, ffp, op.s, op.w);
    }
    op.per.clear();
    finish_op(op);
    return X3D_OK;
}

// Non-periodic staggered operators: the LHS of interpol_imp_
// (src/x3d_operator_1d.f90:549-706) for a direction of n velocity points and
// nm = n - 1 pressure points, with the bindings of x3d_operator_1d_init
// (:152-189).  The operator's n is its output length m.
//   DERVP (m = nm): cbx6, ccx6, cfx6 (:576-599), factored at :677, before the
//     last-end edits;
//   INTVP (m = nm): cibx6, cicx6 and cifxp6 (a copy of cifx6, :667-670),
//     factored after cibx6(nxm) = 0 (:688, :697);
//   DERPV (m = n):  cbi6, cci6 and cfip6 (cfi6 with cfip6(1) = 0, :676),
//     factored after cbi6(nx-1) = 0 (:689, :698);
//   INTPV (m = n):  cibi6, cici6 and cifip6 (a copy of cifi6), factored
//     after cibi6(nx) = 0.  Only cfxp6(1) and cfip6(1) are zeroed (:675-676).
// The first and last diagonal entries of the nm-point matrices are 1 + alfa
// for free slip and Dirichlet ends alike (:579-584, :625-630).
int build_nonperiodic_stag(int kind, int dir, int n, double d, int ncl1, int ncln, int npaire, OpHost &op)
{
    if (n < 9 || ncl1 < 1 || ncl1 > 2 || ncln < 1 || ncln > 2) return X3D_EUNSUPPORTED;
    if (kind != DERVP && kind != INTVP && kind != DERPV && kind != INTPV) return X3D_EINVAL;
    const bool vp = kind == DERVP || kind == INTVP;
    const int m = vp ? n - 1 : n;
    op.kind = kind;
    op.dir = dir;
    op.n = m;
    op.periodic = 0;
    op.npaire = npaire;
    op.ncl1 = ncl1;
    op.ncln = ncln;
    rhs_scalars(kind, d, &op.alfa, &op.a, &op.b, &op.c, &op.d);
    const double al = op.alfa;
    std::vector<double> fb(m, al), fc(m, 1.0), ff(m, al);
    ff[m - 1] = 0.0;
    fb[m - 1] = 0.0;
    if (vp) {
        fc[0] = 1.0 + al;
        fc[m - 1] = 1.0 + al;
    } else {
        ff[0] = kind == DERPV ? 0.0 : al + al;  // cfi6(1) = 2 alfa; cfip6(1) = 0
        fb[m - 2] = kind == DERPV ? 0.0 : al + al;  // cbi6(nx-1) = 2 alfa, zeroed for derxpv
    }
    op.f = ff;
    lu_prepare(fb, fc, ff, op.s, op.w);
    op.per.clear();
    finish_op(op);
    return X3D_OK;
}

// True when an operator's factors are those of the periodic matrix for its
// alfa (to 1e-12 relative), i.e. when it is the circulant (alfa, 1, alfa).
static bool circulant(const OpHost &h)
{
    if (!h.periodic || h.per.size() != (size_t)h.n || h.n < 8) return false;
    if (!(std::fabs(h.alfa) < 0.5)) return false;
    std::vector<double> f, s, w, per;
    periodic_lu(h.n, h.alfa, f, s, w, per);
    auto same = [](const std::vector<double> &a, const std::vector<double> &b) {
        double m = 0.0, e = 0.0;
        for (size_t i = 0; i < a.size(); ++i) {
            m = std::max(m, std::fabs(b[i]));
            e = std::max(e, std::fabs(a[i] - b[i]));
        }
        return e <= 1e-12 * (m > 0 ? m : 1.0);
    };
    return same(h.f, f) && same(h.s, s) && same(h.w, w) && same(h.per, per);
}

// Chunks a carry scan must visit for chunk length L (LineOp::depth).
static int circ_depth(double rho, int L, int n, double thr)
{
    const int C = (n + L - 1) / L;
    const double ar = std::fabs(rho);
    if (std::pow(ar, n) >= thr) return C;
    std::vector<double> m(C, std::pow(ar, L));
    m[C - 1] = std::pow(ar, n - (C - 1) * L);
    int k = 1;
    for (int c = 0; c < C; ++c) {
        double prod = 1.0;
        int d = 0;
        while (prod >= thr && d < C) {
            prod *= m[((c - d) % C + C) % C];
            ++d;
        }
        k = std::max(k, d);
    }
    return std::min(k, C);
}

template <typename T>
static void fill_circ(const OpHost &h, LineOp<T> &lo, double thr)
{
    lo.circ = circulant(h) ? 1 : 0;
    const double al = h.alfa;
    const double rho = al == 0.0 ? 0.0 : -2.0 * al / (1.0 + std::sqrt(1.0 - 4.0 * al * al));
    const double sc = 1.0 + rho * rho;
    lo.ca = (T)(h.a * sc);
    lo.cb = (T)(h.b * sc);
    lo.cc = (T)(h.c * sc);
    lo.cd = (T)(h.d * sc);
    lo.rho = (T)rho;
    const int Ls[2] = {kChunkLong<T>, kChunkShort<T>};
    for (int i = 0; i < 2; ++i) {
        const int L = Ls[i], C = (h.n + L - 1) / L;
        lo.mfull[i] = (T)std::pow(rho, L);
        lo.mlast[i] = (T)std::pow(rho, h.n - (C - 1) * L);
        lo.depth[i] = circ_depth(rho, L, h.n, thr);
    }
    lo.wrap = (T)(1.0 / (1.0 - std::pow(rho, h.n)));
}

// g = M^-T e_1 with M = L U, L unit lower bidiagonal (L(i,i-1) = s_i) and U
// upper bidiagonal (U(i,i) = 1/w_i, U(i,i+1) = f_i).  Then y_0 = g . r for
// y = M^-1 r, which lets the GPU sweep form the Sherman-Morrison scalar
// after the forward pass and emit final values during the backward pass.
void finish_op(OpHost &op)
{
    const int n = op.n;
    std::vector<double> h(n), g(n);
    h[0] = op.w[0];  // U^T h = e_1
    for (int i = 1; i < n; ++i) h[i] = -op.f[i - 1] * h[i - 1] * op.w[i];
    g[n - 1] = h[n - 1];  // L^T g = h
    for (int i = n - 2; i >= 0; --i) g[i] = h[i] - op.s[i + 1] * g[i + 1];
    op.g = g;
    // g decays geometrically from i = 0; terms below 1e-18 |g_0| are below
    // FP64 resolution of y_0 and are dropped.
    op.glen = n;
    const double gcut = 1e-18 * std::fabs(g[0]);
    while (op.glen > 1 && std::fabs(g[op.glen - 1]) <= gcut) --op.glen;
    if (op.periodic && !op.per.empty())
        op.den = 1.0 + op.per[0] - op.alfa * op.per[n - 1];
    else
        op.den = 1.0;
}

// Scan depths for chunk length L: smallest k such that any k consecutive
// chunk multipliers multiply to below 1e-20 (capped at the chunk count).
int upload_op(x3d_op_s *op)
{
    const OpHost &h = op->h;
    const int n = h.n;
    // layout (bytes, each part 256-aligned): float s,w,fw,p | double s,w,fw,p,g
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t o_f = 0, o_d = al(o_f + 4 * n * sizeof(float));
    const size_t total = al(o_d + 5 * n * sizeof(double));
    std::vector<unsigned char> host(total, 0);
    float *hf = reinterpret_cast<float *>(host.data() + o_f);
    double *hd = reinterpret_cast<double *>(host.data() + o_d);
    for (int i = 0; i < n; ++i) {
        const double fw = h.f[i] * h.w[i];
        const double p = h.per.empty() ? 0.0 : h.per[i];
        hf[0 * n + i] = (float)h.s[i];
        hf[1 * n + i] = (float)h.w[i];
        hf[2 * n + i] = (float)fw;
        hf[3 * n + i] = (float)p;
        hd[0 * n + i] = h.s[i];
        hd[1 * n + i] = h.w[i];
        hd[2 * n + i] = fw;
        hd[3 * n + i] = p;
        hd[4 * n + i] = h.g[i];
    }
    if (op->dmem) cudaFree(op->dmem);
    op->dmem = nullptr;
    if (cudaMalloc(&op->dmem, host.size()) != cudaSuccess) return X3D_ENOMEM;
    if (cudaMemcpy(op->dmem, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return X3D_ECUDA;
    const unsigned char *base = static_cast<const unsigned char *>(op->dmem);
    const float *df = reinterpret_cast<const float *>(base + o_f);
    const double *dd = reinterpret_cast<const double *>(base + o_d);
    auto fill = [&](auto &lo, auto *arr) {
        lo.s = arr + 0 * n;
        lo.w = arr + 1 * n;
        lo.fw = arr + 2 * n;
        lo.p = arr + 3 * n;
        lo.g = dd + 4 * n;
        lo.alfa = h.alfa;
        lo.den = h.den;
        lo.n = n;
        lo.periodic = h.periodic;
        lo.glen = h.glen;
    };
    fill(op->opf, df);
    fill(op->opd, dd);
    op->opf.ncl1 = op->opd.ncl1 = h.ncl1;
    op->opf.ncln = op->opd.ncln = h.ncln;
    op->opf.npaire = op->opd.npaire = h.npaire;
    for (int i = 0; i < 8; ++i) {
        op->opf.cl[i] = (float)h.cl[i];
        op->opd.cl[i] = h.cl[i];
    }
    op->opf.a = (float)h.a; op->opf.b = (float)h.b; op->opf.c = (float)h.c; op->opf.d = (float)h.d;
    op->opd.a = h.a; op->opd.b = h.b; op->opd.c = h.c; op->opd.d = h.d;
    fill_circ(h, op->opf, 1e-12);
    fill_circ(h, op->opd, 1e-20);
    return X3D_OK;
}

void free_op(x3d_op_s *op)
{
    if (op && op->dmem) cudaFree(op->dmem);
    if (op) op->dmem = nullptr;
}

}  // namespace x3d
