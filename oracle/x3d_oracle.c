/*
 * x3d_oracle.c -- CPU FP64 restatement of x3div's Euler-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * library in x3div_b200/.  It is compiled into oracle/_build/liboracle.so
 * and may only be loaded by tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py.  Nothing in the product
 * path links or calls it.
 *
 * Parity status: the reference (Fortran 2008 + MPI + the un-vendored
 * 2decomp&FFT library) cannot be compiled in this image (no gfortran, no
 * MPI), and it ships no golden vectors or unit tests.  This restatement is
 * pinned against the reference's own known-answer formulas instead:
 *   - the modified wavenumbers of the staggered first derivative and the
 *     interpolation transfer function from src/poisson.f90:522-533 and
 *     :631-650 (a periodic compact operator applied to a Fourier mode must
 *     reproduce them to round-off),
 *   - the analytic derivatives of the initial field in src/mom.f90:88-113,
 *     151-175, 210-235 (test_du/dv/dw),
 *   - the divergence-free projection (src/navier.f90:98-236 after
 *     src/poisson.f90:276-419) driving div(u) to round-off.
 * The 6th-order compact second derivative is not implemented in the
 * reference (src/x3d_derive.f90:54-59,91-92 declare null pointers only); its
 * restatement here follows the published Lele (1992) interior scheme and is
 * pinned only by its analytic transfer function.
 *
 * Arrays are Fortran-ordered: element (i,j,k) of an (nx,ny,nz) field lives at
 * i + nx*(j + ny*k), with i (x) fastest, exactly as every 2decomp pencil
 * stores data.  Indices in comments are the reference's 1-based ones.
 * The periodic (ncl=0) branches are restated for every operator; of the
 * non-periodic ones, which the reference can only reach without its Poisson
 * solver (it aborts in decomp_2d_poisson_init for them, src/poisson.f90:
 * 104-108), the first derivatives der?_ij (free slip and Dirichlet ends) and
 * the staggered routines' nclx = .false. branches are.  Those are pinned by
 * exactness on cubics (Dirichlet closures) and by the analytic derivatives
 * and interpolants of mirrored cosines (free slip, staggered).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_OK 0
#define ORC_EBADARG -1

enum { ORC_DER = 0, ORC_DER2 = 1, ORC_DERVP = 2, ORC_DERPV = 3, ORC_INTVP = 4, ORC_INTPV = 5 };
enum { ORC_X = 0, ORC_Y = 1, ORC_Z = 2 };

/* ------------------------------------------------------------------------ */
/* Thomas LU preparation: src/x3d_operator_1d.f90:301-323 (prepare).        */
/* b lower, c diagonal, f upper diagonal; outputs s (forward factors) and   */
/* w (inverse pivots).                                                       */
void orc_prepare(const double *b, const double *c, const double *f, double *s, double *w, int n)
{
    for (int i = 0; i < n; ++i) w[i] = c[i];
    s[0] = 0.0; /* s(1) is never set by the reference; its arrays start at zero (x3d_operator_x_data.f90:92-93) */
    for (int i = 1; i < n; ++i) {
        s[i] = b[i - 1] / w[i - 1];
        w[i] = w[i] - f[i - 1] * s[i];
    }
    for (int i = 0; i < n; ++i) w[i] = 1.0 / w[i];
}

/* Single-vector Thomas solve: src/thomas.f90:200-218 (thomas1d). */
void orc_thomas1d(double *t, const double *f, const double *s, const double *w, int n)
{
    for (int k = 1; k < n; ++k) t[k] = t[k] - t[k - 1] * s[k];
    t[n - 1] = t[n - 1] * w[n - 1];
    for (int k = n - 2; k >= 0; --k) t[k] = (t[k] - f[k] * t[k + 1]) * w[k];
}

/* ------------------------------------------------------------------------ */
/* Explicit RHS scalars per operator kind.                                   */
/*  DER   : first_deriv_exp_, ifirstder=4   (x3d_operator_1d.f90:350-353)    */
/*  DERVP/DERPV : interpol_exp_ staggered derivative (:510-512)              */
/*  INTVP/INTPV : interpol_exp_ ipinter=3 interpolation (:539-544)           */
/*  DER2  : Lele (1992) 6th-order compact second derivative, alpha=2/11,     */
/*          a=12/11, b=3/11 (absent from the reference)                      */
/* out: alfa, a, b, c, d                                                     */
void orc_rhs_scalars(int kind, double d, double *out)
{
    const double one = 1.0, two = 2.0, three = 3.0, seven = 7.0, nine = 9.0, ten = 10.0;
    double alfa = 0, a = 0, b = 0, c = 0, dd = 0;
    switch (kind) {
    case ORC_DER:
        alfa = one / three;
        a = (seven / nine) / d;
        b = (one / 36.0) / d;
        break;
    case ORC_DERVP:
    case ORC_DERPV:
        alfa = nine / 62.0;
        a = (63.0 / 62.0) / d;
        b = (17.0 / 62.0) / three / d;
        break;
    case ORC_INTVP:
    case ORC_INTPV: {
        const double ail = 0.49;
        alfa = ail;
        a = one / 128.0 * (75.0 + 70.0 * ail);
        b = one / 256.0 * (126.0 * ail - 25.0);
        c = one / 256.0 * (-ten * ail + three);
        dd = 0.0;
        break;
    }
    case ORC_DER2:
        alfa = two / 11.0;
        a = (12.0 / 11.0) / (d * d);
        b = (3.0 / 44.0) / (d * d);
        break;
    }
    out[0] = alfa; out[1] = a; out[2] = b; out[3] = c; out[4] = dd;
}

/* ------------------------------------------------------------------------ */
/* Periodic LHS assembly for the given kind, then prepare() and the          */
/* Sherman-Morrison vector of init():                                        */
/*   first derivative: first_deriv_imp_ ncl1=ncln=0 (x3d_operator_1d.f90:    */
/*     411-420, 436-445, 467-477)                                            */
/*   staggered derivative: interpol_imp_ cfx6/ccx6/cbx6 (:576-599, 677)      */
/*   interpolation: interpol_imp_ cifx6/cicx6/cibx6 (:622-645, 679); the     */
/*     "p" copies used by x3d_op_intxvp are equal to these when periodic     */
/*     (:667-670 copy, only cfxp6(1)/cfip6(1) are zeroed at :675-676)        */
/*   periodic vector: init() (:260-264): p = M^-1 (-1, 0, ..., 0, alfa)     */
/* The same assembly is used for the second derivative with its alpha.       */
/* f, s, w, per: length n outputs.  Returns alfa.                            */
int orc_build_lhs(int kind, int n, double d, double *f, double *s, double *w, double *per, double *rhs5)
{
    if (n < 8) return ORC_EBADARG;
    orc_rhs_scalars(kind, d, rhs5);
    const double al = rhs5[0];
    double *fb = (double *)calloc((size_t)n, sizeof(double));
    double *fc = (double *)calloc((size_t)n, sizeof(double));
    double *ff = f;
    for (int i = 0; i < n; ++i) ff[i] = 0.0;
    /* boundary rows in the reference's assignment order (1-based → 0-based) */
    ff[0] = al;
    ff[1] = al;
    fc[0] = 2.0;          /* ncl1 == 0: fc(1) = two / ccx6(1) = two */
    fc[1] = 1.0;
    fb[0] = al;
    fb[1] = al;
    ff[n - 3] = al;
    ff[n - 2] = al;
    ff[n - 1] = 0.0;
    fc[n - 3] = 1.0;
    fc[n - 2] = 1.0;
    fc[n - 1] = 1.0 + al * al; /* ncln == 0 */
    fb[n - 3] = al;
    fb[n - 2] = al;
    fb[n - 1] = 0.0;
    for (int i = 2; i < n - 3; ++i) { /* do i = 3, n-3 */
        ff[i] = al;
        fc[i] = 1.0;
        fb[i] = al;
    }
    orc_prepare(fb, fc, ff, s, w, n);
    /* init(): periodic = (/-one, (zero, i=2, n-1), alfa/) ; thomas1d */
    per[0] = -1.0;
    for (int i = 1; i < n - 1; ++i) per[i] = 0.0;
    per[n - 1] = al;
    orc_thomas1d(per, ff, s, w, n);
    free(fb);
    free(fc);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Periodic explicit stencils.  For n >= 8 every boundary row written out in */
/* the reference equals the interior formula with indices taken mod n, e.g.  */
/* derx_00 tx(1) = afix*(ux(2)-ux(nx)) + bfix*(ux(3)-ux(nx-1)).              */
/*  DER   : derx_00 x3d_derive.f90:130-141, dery_00 :302-319, derz_00 :531-548 */
/*  DERVP : derxvp x3d_staggered.f90:44-55, deryvp :568-585, derzvp :916-935  */
/*  DERPV : derxpv :242-253, derypv :816-833, derzpv :1173-1192               */
/*  INTVP : interxvp :131-164, interyvp :430-475, interzvp :1031-1078         */
/*  INTPV : interxpv :310-343, interypv :663-708, interzpv :1263-1310         */
static inline double stencil(int kind, const double *u, int i, int n, long st, const double *c5)
{
#define U(o) u[(long)((((i) + (o)) % n + n) % n) * st]
    const double a = c5[1], b = c5[2], c = c5[3], d = c5[4];
    switch (kind) {
    case ORC_DER:
        return a * (U(1) - U(-1)) + b * (U(2) - U(-2));
    case ORC_DER2: /* differences of differences: exact for neighbouring values (Sterbenz) */
        return a * ((U(1) - U(0)) - (U(0) - U(-1))) + b * ((U(2) - U(0)) - (U(0) - U(-2)));
    case ORC_DERVP:
        return a * (U(1) - U(0)) + b * (U(2) - U(-1));
    case ORC_DERPV:
        return a * (U(0) - U(-1)) + b * (U(1) - U(-2));
    case ORC_INTVP:
        return a * (U(1) + U(0)) + b * (U(2) + U(-1)) + c * (U(3) + U(-2)) + d * (U(4) + U(-3));
    case ORC_INTPV:
        return a * (U(0) + U(-1)) + b * (U(1) + U(-2)) + c * (U(2) + U(-3)) + d * (U(3) + U(-4));
    }
#undef U
    return 0.0;
}

/* Periodic Thomas along one line with Sherman-Morrison correction:        */
/* xthomas_0 / ythomas_0 / zthomas_0 (thomas.f90:34-58, 87-111, 139-163),   */
/* whose inner solve is ?thomas_12 (:61-84, 114-136, 166-188).               */
static void thomas_line_periodic(double *t, long st, int n, const double *f, const double *s,
                                 const double *w, const double *per, double alfa)
{
    for (int i = 1; i < n; ++i) t[i * st] = t[i * st] - t[(i - 1) * st] * s[i];
    t[(n - 1) * st] = t[(n - 1) * st] * w[n - 1];
    for (int i = n - 2; i >= 0; --i) t[i * st] = (t[i * st] - f[i] * t[(i + 1) * st]) * w[i];
    const double ss = (t[0] - alfa * t[(n - 1) * st]) / (1.0 + per[0] - alfa * per[n - 1]);
    for (int i = 0; i < n; ++i) t[i * st] = t[i * st] - ss * per[i];
}

/* Line geometry of an (nx,ny,nz) field along direction dir. */
static void line_geom(int dir, int nx, int ny, int nz, int *n, long *st, long *nlines)
{
    if (dir == ORC_X) { *n = nx; *st = 1; *nlines = (long)ny * nz; }
    else if (dir == ORC_Y) { *n = ny; *st = nx; *nlines = (long)nx * nz; }
    else { *n = nz; *st = (long)nx * ny; *nlines = (long)nx * ny; }
}

static long line_base(int dir, int nx, int ny, long l)
{
    if (dir == ORC_X) return l * nx;                 /* l = j + ny*k */
    if (dir == ORC_Y) { long i = l % nx, k = l / nx; return i + (long)nx * ny * k; }
    return l;                                        /* l = i + nx*j */
}

/* In-place batched periodic Thomas over every line of a pencil:
 * ?thomas_0 generics of thomas.f90:15-28. */
int orc_thomas_periodic(int dir, double *t, int nx, int ny, int nz, const double *f, const double *s,
                        const double *w, const double *per, double alfa)
{
    int n; long st, nl;
    line_geom(dir, nx, ny, nz, &n, &st, &nl);
    if (n < 2) return ORC_EBADARG;
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nl; ++l)
        thomas_line_periodic(t + line_base(dir, nx, ny, l), st, n, f, s, w, per, alfa);
    return ORC_OK;
}

/* Non-periodic batched Thomas (?thomas_12, thomas.f90:61-84 etc.). */
int orc_thomas_plain(int dir, double *t, int nx, int ny, int nz, const double *f, const double *s,
                     const double *w)
{
    int n; long st, nl;
    line_geom(dir, nx, ny, nz, &n, &st, &nl);
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nl; ++l) {
        double *tt = t + line_base(dir, nx, ny, l);
        for (int i = 1; i < n; ++i) tt[i * st] = tt[i * st] - tt[(i - 1) * st] * s[i];
        tt[(n - 1) * st] = tt[(n - 1) * st] * w[n - 1];
        for (int i = n - 2; i >= 0; --i) tt[i * st] = (tt[i * st] - f[i] * tt[(i + 1) * st]) * w[i];
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Non-periodic sixth-order compact first derivative (ifirstder = 4).       */
/* first_deriv_exp_ (x3d_operator_1d.f90:325-393) closure scalars, returned */
/* in cl[8] = {af1, bf1, cf1, af2, afm, afn, bfn, cfn}, and first_deriv_imp_ */
/* (:395-488) factors f, s, w of the operator of parity npaire (0: ff/fs/fw,  */
/* 1: ffp/fsp/fwp).  ncl1, ncln: 1 free slip, 2 Dirichlet.                   */
int orc_build_der_np(int n, double d, int ncl1, int ncln, int npaire, double *f, double *s, double *w,
                     double *cl)
{
    if (n < 8 || ncl1 < 1 || ncl1 > 2 || ncln < 1 || ncln > 2) return ORC_EBADARG;
    const double alfai = 1.0 / 3.0;
    const double alfa1 = 2.0, alfa2 = 0.25, alfan = 2.0, alfam = 0.25;
    cl[0] = -(5.0 / 2.0) / d; cl[1] = 2.0 / d; cl[2] = 0.5 / d;  /* af1 bf1 cf1 :376-378 */
    cl[3] = (3.0 / 4.0) / d;                                   /* af2 :382 */
    cl[4] = (3.0 / 4.0) / d;                                   /* afm :389 */
    cl[5] = -(5.0 / 2.0) / d; cl[6] = 2.0 / d; cl[7] = 0.5 / d;  /* afn bfn cfn :384-386 */
    double *fb = calloc(n, sizeof(double)), *fc = calloc(n, sizeof(double)), *ff = calloc(n, sizeof(double));
    if (ncl1 == 1) {               /* :424-430 */
        ff[0] = alfai + alfai; ff[1] = alfai; fc[0] = 1.0; fc[1] = 1.0; fb[0] = alfai; fb[1] = alfai;
    } else {                       /* :431-437 */
        ff[0] = alfa1; ff[1] = alfa2; fc[0] = 1.0; fc[1] = 1.0; fb[0] = alfa2; fb[1] = alfai;
    }
    if (ncln == 1) {               /* :449-458 */
        ff[n - 3] = alfai; ff[n - 2] = alfai; ff[n - 1] = 0.0;
        fc[n - 3] = 1.0; fc[n - 2] = 1.0; fc[n - 1] = 1.0;
        fb[n - 3] = alfai; fb[n - 2] = alfai + alfai; fb[n - 1] = 0.0;
    } else {                       /* :459-468 */
        ff[n - 3] = alfai; ff[n - 2] = alfam; ff[n - 1] = 0.0;
        fc[n - 3] = 1.0; fc[n - 2] = 1.0; fc[n - 1] = 1.0;
        fb[n - 3] = alfam; fb[n - 2] = alfan; fb[n - 1] = 0.0;
    }
    for (int i = 2; i < n - 3; ++i) { ff[i] = alfai; fc[i] = 1.0; fb[i] = alfai; }  /* :470-474 */
    if (npaire == 1) {             /* :476-486 */
        if (ncl1 == 1) ff[0] = 0.0;
        if (ncln == 1) fb[n - 2] = 0.0;
    }
    for (int i = 0; i < n; ++i) f[i] = ff[i];
    orc_prepare(fb, fc, ff, s, w, n);
    free(fb); free(fc); free(ff);
    return ORC_OK;
}

/* der?_ij (x3d_derive.f90:156-215 and the y/z analogues): RHS with the
 * boundary closures, then the non-periodic Thomas solve.  1-based
 * tx(1), tx(2), tx(nx-1), tx(nx) are rows 0, 1, n-2, n-1 here. */
int orc_apply_der_np(int dir, double *out, const double *in, int nx, int ny, int nz, double d, int ncl1,
                     int ncln, int npaire)
{
    int n; long st, nl;
    line_geom(dir, nx, ny, nz, &n, &st, &nl);
    double *f = malloc(sizeof(double) * n), *s = malloc(sizeof(double) * n), *w = malloc(sizeof(double) * n);
    double cl[8];
    int rc = orc_build_der_np(n, d, ncl1, ncln, npaire, f, s, w, cl);
    if (rc) { free(f); free(s); free(w); return rc; }
    const double a = (7.0 / 9.0) / d, b = (1.0 / 36.0) / d;  /* afix, bfix */
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nl; ++l) {
        const long b0 = line_base(dir, nx, ny, l);
        const double *u = in + b0;
        double *t = out + b0;
#define U(i) u[(long)(i) * st]
#define T(i) t[(long)(i) * st]
        if (ncl1 == 1) {                                       /* :172-181 */
            if (npaire == 1) {
                T(0) = 0.0;
                T(1) = a * (U(2) - U(0)) + b * (U(3) - U(1));
            } else {
                T(0) = a * (U(1) + U(1)) + b * (U(2) + U(2));
                T(1) = a * (U(2) - U(0)) + b * (U(3) + U(1));
            }
        } else {                                               /* :182-185 */
            T(0) = cl[0] * U(0) + cl[1] * U(1) + cl[2] * U(2);
            T(1) = cl[3] * (U(2) - U(0));
        }
        for (int i = 2; i < n - 2; ++i) T(i) = a * (U(i + 1) - U(i - 1)) + b * (U(i + 2) - U(i - 2));
        if (ncln == 1) {                                       /* :191-202 */
            if (npaire == 1) {
                T(n - 2) = a * (U(n - 1) - U(n - 3)) + b * (U(n - 2) - U(n - 4));
                T(n - 1) = 0.0;
            } else {
                T(n - 2) = a * (U(n - 1) - U(n - 3)) + b * ((-U(n - 2)) - U(n - 4));
                T(n - 1) = a * ((-U(n - 2)) - U(n - 2)) + b * ((-U(n - 3)) - U(n - 3));
            }
        } else {                                               /* :203-206 */
            T(n - 2) = cl[4] * (U(n - 1) - U(n - 3));
            T(n - 1) = -cl[5] * U(n - 1) - cl[6] * U(n - 2) - cl[7] * U(n - 3);
        }
        for (int i = 1; i < n; ++i) T(i) = T(i) - T(i - 1) * s[i];          /* thomas.f90:72-80 */
        T(n - 1) = T(n - 1) * w[n - 1];
        for (int i = n - 2; i >= 0; --i) T(i) = (T(i) - f[i] * T(i + 1)) * w[i];
#undef U
#undef T
    }
    free(f); free(s); free(w);
    return ORC_OK;
}

/* Non-periodic staggered LHS (interpol_imp_, x3d_operator_1d.f90:549-706),
 * for a direction of n velocity points, nm = n - 1, with the arrays that
 * x3d_operator_1d_init binds (:152-189).  *m receives the row count.
 *   DERVP: cbx6 ccx6 cfx6 (:576-599), prepared at :677 (before :686-703)
 *   INTVP: cibx6 cicx6 cifxp6 (= cifx6, :667-670), re-prepared at :697
 *   DERPV: cbi6 cci6 cfip6 (cfip6(1) = 0, :676), cbi6(nx-1) = 0, :698
 *   INTPV: cibi6 cici6 cifip6 (= cifi6), re-prepared at :698 */
int orc_build_stag_np(int kind, int n, double d, int ncl1, int ncln, double *f, double *s, double *w, int *m)
{
    if (n < 9 || ncl1 < 1 || ncl1 > 2 || ncln < 1 || ncln > 2) return ORC_EBADARG;
    double sc[5];
    orc_rhs_scalars(kind, d, sc);
    const double al = sc[0];
    const int vp = kind == ORC_DERVP || kind == ORC_INTVP;
    if (!vp && kind != ORC_DERPV && kind != ORC_INTPV) return ORC_EBADARG;
    const int nm = n - 1, r = vp ? nm : n;
    double *b = calloc(r, sizeof(double)), *c = calloc(r, sizeof(double)), *ff = calloc(r, sizeof(double));
    if (vp) {  /* cfx6/ccx6/cbx6 (:576-599), cifx6/cicx6/cibx6 (:622-645) */
        ff[0] = al; ff[1] = al; ff[nm - 3] = al; ff[nm - 2] = al; ff[nm - 1] = 0.0;
        c[0] = 1.0 + al;  /* nclx1 = 1 or 2 */
        c[1] = 1.0; c[nm - 3] = 1.0; c[nm - 2] = 1.0;
        c[nm - 1] = 1.0 + al;  /* nclxn = 1 or 2 */
        b[0] = al; b[1] = al; b[nm - 3] = al; b[nm - 2] = al; b[nm - 1] = 0.0;
        for (int i = 2; i <= nm - 4; ++i) { ff[i] = al; c[i] = 1.0; b[i] = al; }
        if (kind == ORC_INTVP) b[nm - 1] = 0.0;  /* cibx6(nxm) = 0 (:688) */
    } else {   /* cfi6/cci6/cbi6 (:601-620), cifi6/cici6/cibi6 (:646-665) */
        ff[0] = al + al; ff[1] = al; ff[n - 3] = al; ff[n - 2] = al; ff[n - 1] = 0.0;
        c[0] = 1.0; c[1] = 1.0; c[n - 3] = 1.0; c[n - 2] = 1.0; c[n - 1] = 1.0;
        b[0] = al; b[1] = al; b[n - 3] = al; b[n - 2] = al + al; b[n - 1] = 0.0;
        for (int i = 2; i <= n - 4; ++i) { ff[i] = al; c[i] = 1.0; b[i] = al; }
        if (kind == ORC_DERPV) {
            ff[0] = 0.0;      /* cfip6(1) = 0 (:676) */
            b[n - 2] = 0.0;   /* cbi6(nx-1) = 0 (:689) */
        } else {
            b[n - 1] = 0.0;   /* cibi6(nx) = 0 (:691) */
        }
    }
    for (int i = 0; i < r; ++i) f[i] = ff[i];
    orc_prepare(b, c, ff, s, w, r);
    free(b); free(c); free(ff);
    *m = r;
    return ORC_OK;
}

/* Non-periodic branches of the 12 staggered routines, row by row as the
 * reference writes them (1-based comments), then ?thomas_12.  (nx, ny, nz)
 * are the velocity-grid extents; along dir the input has n (vp) or n - 1
 * (pv) points and the output the other.  The branches that exist
 * (x3d_staggered.f90): derxvp/derzvp npaire 1 (:64, :944) and otherwise (the
 * odd closure, :83, :968); deryvp npaire 0 only (:595, the odd closure);
 * the others npaire 1 only.  Returns ORC_EBADARG where there is none. */
int orc_apply_stag_np(int kind, int dir, double *out, const double *in, int nx, int ny, int nz, double d, int ncl1,
                      int ncln, int npaire)
{
    const int n = dir == ORC_X ? nx : (dir == ORC_Y ? ny : nz);
    const int vp = kind == ORC_DERVP || kind == ORC_INTVP;
    int odd = 0;
    if (kind == ORC_DERVP) {
        if (dir == ORC_Y) { if (npaire != 0) return ORC_EBADARG; odd = 1; }
        else odd = npaire != 1;
    } else if (npaire != 1) {
        return ORC_EBADARG;
    }
    double *f = malloc(sizeof(double) * n), *s = malloc(sizeof(double) * n), *w = malloc(sizeof(double) * n);
    int m = 0;
    const int rc = orc_build_stag_np(kind, n, d, ncl1, ncln, f, s, w, &m);
    if (rc) { free(f); free(s); free(w); return rc; }
    const int ni = vp ? n : n - 1, nm = n - 1;
    double sc[5];
    orc_rhs_scalars(kind, d, sc);
    const double a = sc[1], b = sc[2], c = sc[3], dd = sc[4];
    const int o1 = dir == ORC_X ? ny : nx, o2 = dir == ORC_Z ? ny : nz;
    long st = dir == ORC_X ? 1 : (dir == ORC_Y ? nx : (long)nx * ny);
    const long nl = (long)o1 * o2;
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nl; ++l) {
        long bi, bo;
        if (dir == ORC_X) { bi = l * ni; bo = l * m; }
        else if (dir == ORC_Y) { const long i = l % nx, k = l / nx; bi = i + (long)nx * ni * k; bo = i + (long)nx * m * k; }
        else { bi = bo = l; }
        const double *u = in + bi;
        double *t = out + bo;
#define U(i) u[(long)((i) - 1) * st]
#define T(i) t[(long)((i) - 1) * st]
        if (kind == ORC_DERVP) {       /* derxvp :64-101, deryvp :595-622, derzvp :944-988 */
            if (!odd) {
                T(1) = a * (U(2) - U(1)) + b * (U(3) - U(2));
                T(nm) = a * (U(n) - U(nm)) + b * (U(nm) - U(nm - 1));
            } else {
                T(1) = a * (U(2) - U(1)) + b * (U(3) - 2.0 * U(1) + U(2));
                T(nm) = a * (U(n) - U(nm)) + b * (2.0 * U(n) - U(nm) - U(nm - 1));
            }
            T(2) = a * (U(3) - U(2)) + b * (U(4) - U(1));
            for (int i = 3; i <= nm - 2; ++i) T(i) = a * (U(i + 1) - U(i)) + b * (U(i + 2) - U(i - 1));
            T(nm - 1) = a * (U(nm) - U(nm - 1)) + b * (U(n) - U(nm - 2));
        } else if (kind == ORC_INTVP) { /* interxvp :173-206 */
            T(1) = a * (U(2) + U(1)) + b * (U(3) + U(2)) + c * (U(4) + U(3)) + dd * (U(5) + U(4));
            T(2) = a * (U(3) + U(2)) + b * (U(4) + U(1)) + c * (U(5) + U(2)) + dd * (U(6) + U(3));
            T(3) = a * (U(4) + U(3)) + b * (U(5) + U(2)) + c * (U(6) + U(1)) + dd * (U(7) + U(2));
            for (int i = 4; i <= nm - 3; ++i)
                T(i) = a * (U(i + 1) + U(i)) + b * (U(i + 2) + U(i - 1)) + c * (U(i + 3) + U(i - 2)) +
                       dd * (U(i + 4) + U(i - 3));
            T(nm - 2) = a * (U(nm - 1) + U(nm - 2)) + b * (U(nm) + U(nm - 3)) + c * (U(n) + U(nm - 4)) +
                        dd * (U(nm) + U(nm - 5));
            T(nm - 1) = a * (U(nm) + U(nm - 1)) + b * (U(n) + U(nm - 2)) + c * (U(nm) + U(nm - 3)) +
                        dd * (U(nm - 1) + U(nm - 4));
            T(nm) = a * (U(n) + U(nm)) + b * (U(nm) + U(nm - 1)) + c * (U(nm - 1) + U(nm - 2)) +
                    dd * (U(nm - 2) + U(nm - 3));
        } else if (kind == ORC_DERPV) { /* derxpv :262-277 */
            T(1) = 0.0;
            T(2) = a * (U(2) - U(1)) + b * (U(3) - U(1));
            for (int i = 3; i <= n - 2; ++i) T(i) = a * (U(i) - U(i - 1)) + b * (U(i + 1) - U(i - 2));
            T(n - 1) = a * (U(n - 1) - U(n - 2)) + b * (U(n - 1) - U(n - 3));
            T(n) = 0.0;
        } else {                        /* interxpv :352-397 */
            T(1) = a * (U(1) + U(1)) + b * (U(2) + U(2)) + c * (U(3) + U(3)) + dd * (U(4) + U(4));
            T(2) = a * (U(2) + U(1)) + b * (U(3) + U(1)) + c * (U(4) + U(2)) + dd * (U(5) + U(3));
            T(3) = a * (U(3) + U(2)) + b * (U(4) + U(1)) + c * (U(5) + U(1)) + dd * (U(6) + U(2));
            T(4) = a * (U(4) + U(3)) + b * (U(5) + U(2)) + c * (U(6) + U(1)) + dd * (U(7) + U(1));
            for (int i = 5; i <= n - 4; ++i)
                T(i) = a * (U(i) + U(i - 1)) + b * (U(i + 1) + U(i - 2)) + c * (U(i + 2) + U(i - 3)) +
                       dd * (U(i + 3) + U(i - 4));
            T(n - 3) = a * (U(n - 3) + U(n - 4)) + b * (U(n - 2) + U(n - 5)) + c * (U(n - 1) + U(n - 6)) +
                       dd * (U(n - 1) + U(n - 7));
            T(n - 2) = a * (U(n - 2) + U(n - 3)) + b * (U(n - 1) + U(n - 4)) + c * (U(n - 1) + U(n - 5)) +
                       dd * (U(n - 2) + U(n - 6));
            T(n - 1) = a * (U(n - 1) + U(n - 2)) + b * (U(n - 1) + U(n - 3)) + c * (U(n - 2) + U(n - 4)) +
                       dd * (U(n - 3) + U(n - 5));
            T(n) = a * (U(n - 1) + U(n - 1)) + b * (U(n - 2) + U(n - 2)) + c * (U(n - 3) + U(n - 3)) +
                   dd * (U(n - 4) + U(n - 4));
        }
        for (int i = 2; i <= m; ++i) T(i) = T(i) - T(i - 1) * s[i - 1];   /* thomas.f90:72-80 */
        T(m) = T(m) * w[m - 1];
        for (int i = m - 1; i >= 1; --i) T(i) = (T(i) - f[i - 1] * T(i + 1)) * w[i - 1];
#undef U
#undef T
    }
    free(f); free(s); free(w);
    return ORC_OK;
}

/* Operator application: explicit RHS then the periodic Thomas solve, as in
 * derx_00/dery_00/derz_00 and the periodic branches of the 12 staggered
 * routines (nxm = nx when periodic).  out and in must not alias (the
 * reference's t is intent(out), u intent(in)).  The stretching multiply of
 * dery_00/deryvp/derypv is skipped: istret=0 (parameters.f90:117). */
int orc_apply(int kind, int dir, double *out, const double *in, int nx, int ny, int nz, double d)
{
    int n; long st, nl;
    line_geom(dir, nx, ny, nz, &n, &st, &nl);
    if (n < 8 || kind < 0 || kind > 5) return ORC_EBADARG;
    double *f = malloc(sizeof(double) * n), *s = malloc(sizeof(double) * n);
    double *w = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n);
    double c5[5];
    orc_build_lhs(kind, n, d, f, s, w, p, c5);
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nl; ++l) {
        long b0 = line_base(dir, nx, ny, l);
        for (int i = 0; i < n; ++i) out[b0 + i * st] = stencil(kind, in + b0, i, n, st, c5);
        thomas_line_periodic(out + b0, st, n, f, s, w, p, c5[0]);
    }
    free(f); free(s); free(w); free(p);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Spectral Poisson, fully periodic (poisson_000, poisson.f90:276-419).      */
/* Tables: abxyz bc=0 (:436-440, 450-454, 464-468) and waves() bc=0          */
/* (:522-538, 556-572, 591-601, 659-699).  cw is the (nx, ny, nz/2+1)        */
/* complex spectrum with i fastest, interleaved re/im, as produced by an    */
/* unnormalised r2c transform along z followed by c2c along y and x         */
/* (2decomp PHYSICAL_IN_Z).  Modified in place exactly as :338-396.          */
static void waves_1d(int n, double len, double d, double *k2, double *es, double *ttot)
{
    const double pi = acos(-1.0), twopi = 2.0 * acos(-1.0);
    double c5d[5], c5i[5];
    orc_rhs_scalars(ORC_DERVP, d, c5d);
    orc_rhs_scalars(ORC_INTVP, d, c5i);
    const double alcai = c5d[0], aci = c5d[1], bci = c5d[2];
    const double ailcai = c5i[0], aici = c5i[1], bici = c5i[2], cici = c5i[3], dici = c5i[4];
    (void)pi;
    for (int i = 0; i < n / 2 + 1; ++i) {
        double w = twopi * i / n;
        double wp = aci * 2.0 * d * sin(w * 0.5) + bci * 2.0 * d * sin(3.0 * 0.5 * w);
        wp = wp / (1.0 + 2.0 * alcai * cos(w));
        es[i] = n * w / len;
        double t = n * wp / len;
        k2[i] = t * t;
    }
    for (int i = n / 2 + 1; i < n; ++i) { /* do i = nx/2+2, nx: xk2(i) = xk2(nx-i+2) */
        k2[i] = k2[n - i];
        es[i] = es[n - i];
    }
    for (int i = 0; i < n; ++i) {
        double rle = es[i] * d;
        double tt = 2.0 * (bici * cos(rle * 1.5) + cici * cos(rle * 2.5) + dici * cos(rle * 3.5));
        double tt1 = 2.0 * aici * cos(rle * 0.5);
        double t1 = 1.0 + 2.0 * ailcai * cos(rle);
        ttot[i] = (tt1 + tt) / t1;
    }
}

/* Writes the modified wavenumber tables used by the spectral division.
 * k2x,tx: length nx; k2y,ty: ny; k2z,tz: nz.  Exposed for tests. */
void orc_poisson_tables(int nx, int ny, int nz, double xlx, double yly, double zlz,
                        double *k2x, double *tx, double *k2y, double *ty, double *k2z, double *tz)
{
    double *es = malloc(sizeof(double) * (size_t)(nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz)));
    waves_1d(nx, xlx, xlx / nx, k2x, es, tx);
    waves_1d(ny, yly, yly / ny, k2y, es, ty);
    waves_1d(nz, zlz, zlz / nz, k2z, es, tz);
    free(es);
}

/* The non-periodic (bc = 1) branch of waves() for one direction of m = n - 1
 * pressure points (src/poisson.f90:539-553 for x, :573-588 for y): mode
 * i = 0 .. m of the cosine expansion, w = pi i / m, the staggered
 * derivative's modified wavenumber squared k2[i] = (m wp / len)^2 (zero for
 * i = 0) and the interpolation's transfer function tt[i] at rle = es d = w,
 * d = len / m.  The z branch (:603-613) packs modes i and m + 1 - i of the
 * same two functions into the real and imaginary parts of one complex
 * entry, for 2decomp's half-length transform; its values are these. */
void orc_poisson_tables_bc1(int m, double len, double *k2, double *tt)
{
    const double pi = acos(-1.0);
    const double d = len / m;
    double c5d[5], c5i[5];
    orc_rhs_scalars(ORC_DERVP, d, c5d);
    orc_rhs_scalars(ORC_INTVP, d, c5i);
    const double alcai = c5d[0], aci = c5d[1], bci = c5d[2];
    const double ailcai = c5i[0], aici = c5i[1], bici = c5i[2], cici = c5i[3], dici = c5i[4];
    for (int i = 0; i <= m; ++i) {
        const double w = 2.0 * pi * 0.5 * i / m;
        double wp = aci * 2.0 * d * sin(w * 0.5) + bci * 2.0 * d * sin(3.0 * 0.5 * w);
        wp = wp / (1.0 + 2.0 * alcai * cos(w));
        const double t = m * wp / len;
        k2[i] = i == 0 ? 0.0 : t * t;
        const double es = i == 0 ? 0.0 : m * w / len;
        const double rle = es * d;
        const double tt2 = 2.0 * (bici * cos(rle * 1.5) + cici * cos(rle * 2.5) + dici * cos(rle * 3.5));
        const double tt1 = 2.0 * aici * cos(rle * 0.5);
        tt[i] = (tt1 + tt2) / (1.0 + 2.0 * ailcai * cos(rle));
    }
}

int orc_poisson_spectral(double *cw, int nx, int ny, int nz, double xlx, double yly, double zlz)
{
    const double pi = acos(-1.0);
    const double epsilon = 1.e-16;
    const int nz2 = nz / 2 + 1;
    double *k2x = malloc(sizeof(double) * nx), *tx = malloc(sizeof(double) * nx);
    double *k2y = malloc(sizeof(double) * ny), *ty = malloc(sizeof(double) * ny);
    double *k2z = malloc(sizeof(double) * nz), *tz = malloc(sizeof(double) * nz);
    orc_poisson_tables(nx, ny, nz, xlx, yly, zlz, k2x, tx, k2y, ty, k2z, tz);
    double *ax = malloc(sizeof(double) * nx), *bx = malloc(sizeof(double) * nx);
    double *ay = malloc(sizeof(double) * ny), *by = malloc(sizeof(double) * ny);
    double *az = malloc(sizeof(double) * nz), *bz = malloc(sizeof(double) * nz);
    for (int i = 0; i < nx; ++i) { ax[i] = sin((double)i * pi / (double)nx); bx[i] = cos((double)i * pi / (double)nx); }
    for (int j = 0; j < ny; ++j) { ay[j] = sin((double)j * pi / (double)ny); by[j] = cos((double)j * pi / (double)ny); }
    for (int k = 0; k < nz; ++k) { az[k] = sin((double)k * pi / (double)nz); bz[k] = cos((double)k * pi / (double)nz); }
    const double ntot = (double)nx * (double)ny * (double)nz;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz2; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                /* kxyz(i,j,k): waves() :690-695 (both components equal) */
                double tyz = ty[j] * tz[k], txz = tx[i] * tz[k], txy = tx[i] * ty[j];
                double kk = k2x[i] * (tyz * tyz) + k2y[j] * (txz * txz) + k2z[k] * (txy * txy);
                double *c = cw + 2 * ((size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k));
                double re = c[0], im = c[1], t1, t2;
                /* post-processing in z, y, x (:341-359) */
                t1 = re / ntot; t2 = im / ntot;
                re = t1 * bz[k] + t2 * az[k]; im = t2 * bz[k] - t1 * az[k];
                t1 = re; t2 = im;
                re = t1 * by[j] + t2 * ay[j]; im = t2 * by[j] - t1 * ay[j];
                if (j + 1 > ny / 2 + 1) { re = -re; im = -im; }
                t1 = re; t2 = im;
                re = t1 * bx[i] + t2 * ax[i]; im = t2 * bx[i] - t1 * ax[i];
                if (i + 1 > nx / 2 + 1) { re = -re; im = -im; }
                /* solve (:362-370) */
                if (kk < epsilon || kk < epsilon) { re = 0.0; im = 0.0; }
                else { re = re / (-kk); im = im / (-kk); }
                /* backward post-processing in z, y, x (:375-392) */
                t1 = re; t2 = im;
                re = t1 * bz[k] - t2 * az[k]; im = -t2 * bz[k] - t1 * az[k];
                t1 = re; t2 = im;
                re = t1 * by[j] + t2 * ay[j]; im = t2 * by[j] - t1 * ay[j];
                if (j + 1 > ny / 2 + 1) { re = -re; im = -im; }
                t1 = re; t2 = im;
                re = t1 * bx[i] + t2 * ax[i]; im = -t2 * bx[i] + t1 * ax[i];
                if (i + 1 > nx / 2 + 1) { re = -re; im = -im; }
                c[0] = re; c[1] = im;
            }
    free(k2x); free(tx); free(k2y); free(ty); free(k2z); free(tz);
    free(ax); free(bx); free(ay); free(by); free(az); free(bz);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Stage compositions at a 1x1 decomposition, where every 2decomp pencil of */
/* an (nx,ny,nz) field has the same i-fastest layout and each transpose is  */
/* a copy, so the transposes are elided.                                    */

/* divergence (navier.f90:98-236), periodic so nxm=nx etc.  pp3 out. */
int orc_divergence(double *pp3, const double *ux, const double *uy, const double *uz,
                   int nx, int ny, int nz, double dx, double dy, double dz)
{
    size_t N = (size_t)nx * ny * nz;
    double *pp1 = malloc(N * 8), *pgy1 = malloc(N * 8), *pgz1 = malloc(N * 8);
    double *upi2 = malloc(N * 8), *duydypi2 = malloc(N * 8), *po3 = malloc(N * 8);
    int rc = 0;
    rc |= orc_apply(ORC_DERVP, ORC_X, pp1, ux, nx, ny, nz, dx);        /* :166 */
    rc |= orc_apply(ORC_INTVP, ORC_X, pgy1, uy, nx, ny, nz, dx);       /* :168 */
    rc |= orc_apply(ORC_INTVP, ORC_X, pgz1, uz, nx, ny, nz, dx);       /* :169 */
    rc |= orc_apply(ORC_INTVP, ORC_Y, upi2, pp1, nx, ny, nz, dy);      /* :177 */
    rc |= orc_apply(ORC_DERVP, ORC_Y, duydypi2, pgy1, nx, ny, nz, dy); /* :178 */
    for (size_t p = 0; p < N; ++p) duydypi2[p] = duydypi2[p] + upi2[p]; /* :182-184 */
    rc |= orc_apply(ORC_INTVP, ORC_Y, upi2, pgz1, nx, ny, nz, dy);     /* :187 */
    rc |= orc_apply(ORC_INTVP, ORC_Z, pp3, duydypi2, nx, ny, nz, dz);  /* :193 */
    rc |= orc_apply(ORC_DERVP, ORC_Z, po3, upi2, nx, ny, nz, dz);      /* :195 */
    for (size_t p = 0; p < N; ++p) pp3[p] = pp3[p] + po3[p];           /* :200-202 */
    free(pp1); free(pgy1); free(pgz1); free(upi2); free(duydypi2); free(po3);
    return rc;
}

/* gradp (navier.f90:249-359).  px,py,pz out on the velocity grid. */
int orc_gradp(double *px, double *py, double *pz, const double *pp3, int nx, int ny, int nz,
              double dx, double dy, double dz)
{
    size_t N = (size_t)nx * ny * nz;
    double *ppi3 = malloc(N * 8), *pgz3 = malloc(N * 8), *ppi2 = malloc(N * 8);
    double *pgy2 = malloc(N * 8), *pgzi2 = malloc(N * 8);
    int rc = 0;
    rc |= orc_apply(ORC_INTPV, ORC_Z, ppi3, pp3, nx, ny, nz, dz);   /* :273 */
    rc |= orc_apply(ORC_DERPV, ORC_Z, pgz3, pp3, nx, ny, nz, dz);   /* :275 */
    rc |= orc_apply(ORC_INTPV, ORC_Y, ppi2, ppi3, nx, ny, nz, dy);  /* :286 (pp2 = ppi3) */
    rc |= orc_apply(ORC_DERPV, ORC_Y, pgy2, ppi3, nx, ny, nz, dy);  /* :288 */
    rc |= orc_apply(ORC_INTPV, ORC_Y, pgzi2, pgz3, nx, ny, nz, dy); /* :290 (pgz2 = pgz3) */
    rc |= orc_apply(ORC_DERPV, ORC_X, px, ppi2, nx, ny, nz, dx);    /* :302 */
    rc |= orc_apply(ORC_INTPV, ORC_X, py, pgy2, nx, ny, nz, dx);    /* :303 */
    rc |= orc_apply(ORC_INTPV, ORC_X, pz, pgzi2, nx, ny, nz, dx);   /* :304 */
    free(ppi3); free(pgz3); free(ppi2); free(pgy2); free(pgzi2);
    return rc;
}

/* cor_vel (navier.f90:64-91). */
void orc_cor_vel(double *ux, double *uy, double *uz, const double *px, const double *py,
                 const double *pz, long N)
{
#pragma omp parallel for schedule(static)
    for (long p = 0; p < N; ++p) {
        ux[p] = ux[p] - px[p];
        uy[p] = uy[p] - py[p];
        uz[p] = uz[p] - pz[p];
    }
}

/* intt, Euler branch (time_integrators.f90:40-44): var = gdt*dvar + var. */
void orc_intt(double *var, const double *dvar, double gdt, long N)
{
#pragma omp parallel for schedule(static)
    for (long p = 0; p < N; ++p) var[p] = gdt * dvar[p] + var[p];
}

/* momentum_rhs_eq (transeq.f90:44-355).  dux,duy,duz out.  The derx/derxp
 * pair (and y/z) are numerically identical operators when periodic
 * (first_deriv_imp_ :473-486 only changes ffp for free-slip), so both map to
 * the DER kind. */
int orc_momentum_rhs(double *dux, double *duy, double *duz, const double *ux, const double *uy,
                     const double *uz, int nx, int ny, int nz, double dx, double dy, double dz)
{
    size_t N = (size_t)nx * ny * nz;
    double *ta = malloc(N * 8), *td = malloc(N * 8), *tg = malloc(N * 8);
    double *tz_ = malloc(N * 8), *acc = malloc(N * 8);
    const double *u[3] = {ux, uy, uz};
    double *du[3] = {dux, duy, duz};
    int rc = 0;
    for (int c = 0; c < 3; ++c) {
        const double *uc = u[c];
        /* X pencil: ta = ux*uc ; td = derx(ta) ; ta = derx(uc) ; du = td + ux*ta */
        for (size_t p = 0; p < N; ++p) ta[p] = ux[p] * uc[p];
        rc |= orc_apply(ORC_DER, ORC_X, td, ta, nx, ny, nz, dx);
        rc |= orc_apply(ORC_DER, ORC_X, ta, uc, nx, ny, nz, dx);
        for (size_t p = 0; p < N; ++p) du[c][p] = td[p] + ux[p] * ta[p];
        /* Y pencil: td = uc*uy (ux2*uy2, uy2*uy2, uz2*uy2) ; tg = dery(td) ; td = dery(uc) ;
         * tg = tg + uy*td */
        for (size_t p = 0; p < N; ++p) td[p] = (c == 1) ? uy[p] * uy[p] : uc[p] * uy[p];
        rc |= orc_apply(ORC_DER, ORC_Y, tg, td, nx, ny, nz, dy);
        rc |= orc_apply(ORC_DER, ORC_Y, td, uc, nx, ny, nz, dy);
        for (size_t p = 0; p < N; ++p) tg[p] = tg[p] + uy[p] * td[p];
        /* Z pencil: td3 = uc*uz ; tg3 = derz(td3) ; td3 = derz(uc) ; ta3 = tg3 + uz*td3 */
        for (size_t p = 0; p < N; ++p) td[p] = (c == 2) ? uz[p] * uz[p] : uc[p] * uz[p];
        rc |= orc_apply(ORC_DER, ORC_Z, tz_, td, nx, ny, nz, dz);
        rc |= orc_apply(ORC_DER, ORC_Z, td, uc, nx, ny, nz, dz);
        for (size_t p = 0; p < N; ++p) acc[p] = tz_[p] + uz[p] * td[p];
        /* transpose z->y then tg = tg + ta3 ; transpose y->x then du = du + tg */
        for (size_t p = 0; p < N; ++p) tg[p] = tg[p] + acc[p];
        for (size_t p = 0; p < N; ++p) du[c][p] = du[c][p] + tg[p];
    }
    free(ta); free(td); free(tg); free(tz_); free(acc);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Initial field and analytic checks (mom.f90).                              */
/* vel (mom.f90:46-53): x=(i-1)*dx etc. on a single rank (xstart=1).         */
void orc_vel(double *u, double *v, double *w, int nx, int ny, int nz, double xlx, double yly,
             double zlz)
{
    const double twopi = 2.0 * acos(-1.0);
    const double dx = xlx / nx, dy = yly / ny, dz = zlz / nz;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double z = k * dz, y = j * dy, x = i * dx;
                size_t p = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
                u[p] = sin(twopi * (x / xlx)) * cos(twopi * (y / yly)) * cos(twopi * (z / zlz));
                v[p] = cos(twopi * (x / xlx)) * sin(twopi * (y / yly)) * cos(twopi * (z / zlz));
                w[p] = -2.0 * cos(twopi * (x / xlx)) * cos(twopi * (y / yly)) * sin(twopi * (z / zlz));
            }
}

/* test_du / test_dv / test_dw (mom.f90:88-113, 151-175, 210-235): RMS error
 * of a derivative field against the analytic derivative of vel's field.
 * which = 0 (du/dx), 1 (dv/dy), 2 (dw/dz). */
double orc_test_rms(int which, const double *du, int nx, int ny, int nz, double xlx, double yly,
                    double zlz)
{
    const double twopi = 2.0 * acos(-1.0);
    const double dx = xlx / nx, dy = yly / ny, dz = zlz / nz;
    double err = 0.0;
#pragma omp parallel for reduction(+ : err) schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double z = k * dz, y = j * dy, x = i * dx, ana;
                ana = cos(twopi * (x / xlx)) * cos(twopi * (y / yly)) * cos(twopi * (z / zlz));
                if (which == 0) ana = twopi * ana / xlx;
                else if (which == 1) ana = twopi * ana / yly;
                else ana = twopi * (-2.0 * ana) / zlz;
                size_t p = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
                err += (du[p] - ana) * (du[p] - ana);
            }
    return sqrt(err / nx / ny / nz);
}
