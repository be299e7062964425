/*
 * bem_oracle.c -- CPU FP64 restatement of the BEM-MECECCS hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the parity oracle).  Only tests/, the smoke
 * check and the benchmark's CPU-baseline leg may load this library; the
 * product path never does.
 *
 * Each routine follows one reference routine line for line (file:line in
 * giulianobelinassi/BEM-MECECCS src/).  The reference is built with
 * -fdefault-real-8 for the FP64 form, so every REAL here is a double and
 * every COMPLEX a double complex.  Built with -O2 -fno-fast-math so that
 * the oracle is deterministic; OpenMP parallelises over the element
 * column J exactly where the reference does (Ghmatece.for:92,
 * Ghmatecd.for:113, Interec.for:86,188).
 */
#include "bem_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex zc;

#define ORC_OK 0
#define ORC_DEGENERATE 1
#define ORC_SINGULAR 2

int orc_version(void) { return 1; }

static const double kDelta[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

/* Gauleg.for:9-36 with X1=-1, X2=1 (Main.for:114). */
void orc_gauleg(int n, double *x, double *w)
{
    const double eps = 3.0e-14;
    const double x1 = -1.0, x2 = 1.0;
    int m = (n + 1) / 2;
    double xm = 0.50 * (x2 + x1);
    double xl = 0.50 * (x2 - x1);
    for (int i = 1; i <= m; ++i) {
        double z = cos(3.141592654 * (i - 0.25) / (n + 0.5));
        double z1, pp;
        do {
            double p1 = 1.0, p2 = 0.0, p3;
            for (int j = 1; j <= n; ++j) {
                p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            z1 = z;
            z = z1 - p1 / pp;
        } while (fabs(z - z1) > eps);
        x[i - 1] = xm - xl * z;
        x[n - i] = xm + xl * z;
        w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
        w[n - i] = w[i - 1];
    }
}

/* Normvec.for:20-38. */
void orc_normvec(int n, const int *cone, const double *cx, const double *cy,
                 const double *cz, double *etas)
{
    for (int j = 0; j < n; ++j) {
        int n1 = cone[j] - 1, n2 = cone[n + j] - 1, n3 = cone[2 * n + j] - 1;
        double a = (cy[n2] - cy[n1]) * (cz[n3] - cz[n1]) -
                   (cz[n2] - cz[n1]) * (cy[n3] - cy[n1]);
        double b = (cz[n2] - cz[n1]) * (cx[n3] - cx[n1]) -
                   (cx[n2] - cx[n1]) * (cz[n3] - cz[n1]);
        double c = (cx[n2] - cx[n1]) * (cy[n3] - cy[n1]) -
                   (cy[n2] - cy[n1]) * (cx[n3] - cx[n1]);
        double r = sqrt(a * a + b * b + c * c);
        etas[3 * j + 0] = a / r;
        etas[3 * j + 1] = b / r;
        etas[3 * j + 2] = c / r;
    }
}

/* Inputece.for:100-102. */
void orc_centroids(int n, const int *cone, const double *cx, const double *cy,
                   const double *cz, double *cxm, double *cym, double *czm)
{
    for (int i = 0; i < n; ++i) {
        int n1 = cone[i] - 1, n2 = cone[n + i] - 1;
        int n3 = cone[2 * n + i] - 1, n4 = cone[3 * n + i] - 1;
        cxm[i] = (cx[n1] + cx[n2] + cx[n3] + cx[n4]) * 0.250;
        cym[i] = (cy[n1] + cy[n2] + cy[n3] + cy[n4]) * 0.250;
        czm[i] = (cz[n1] + cz[n2] + cz[n3] + cz[n4]) * 0.250;
    }
}

/* Inputecd.for:58-60. */
void orc_material(double ge, double rnu, double dam, double rho, double *zge,
                  double *zcs, double *zcp)
{
    zc g = ge + I * (ge * 2.0 * dam);
    zc s = csqrt(g / rho);
    zc p = s * sqrt((2.0 - 2.0 * rnu) / (1.0 - 2.0 * rnu));
    zge[0] = creal(g); zge[1] = cimag(g);
    zcs[0] = creal(s); zcs[1] = cimag(s);
    zcp[0] = creal(p); zcp[1] = cimag(p);
}

/* Ghmatece.for:55-63 (PI = 4*ATAN(1)). */
void orc_static_consts(double rmu, double rnu, double *c)
{
    double pi = 4.0 * atan(1.0);
    c[0] = 1.0 / (16.0 * pi * rmu * (1.0 - rnu));
    c[1] = 3.0 - (4.0 * rnu);
    c[2] = -1.0 / (8.0 * pi * (1.0 - rnu));
    c[3] = 1.0 - (2.0 * rnu);
}

/* Element corner coordinates CO(4,3) (Ghmatece.for:115-126). */
static void load_co(int n, int j, const int *cone, const double *cx,
                    const double *cy, const double *cz, double co[4][3])
{
    for (int k = 0; k < 4; ++k) {
        int nk = cone[k * n + j] - 1;
        co[k][0] = cx[nk];
        co[k][1] = cy[nk];
        co[k][2] = cz[nk];
    }
}

/* Shape functions, Jacobian and Gauss point: Nonsinge.for:47-106 (the same
 * block appears in Nonsingd.for, Sing_de.for, Singge.for and Sigmaec.for).
 * Returns 0, or ORC_DEGENERATE when DET < 1e-5. */
static int gauss_point(const double co[4][3], double g1, double g2,
                       double *xg, double *yg, double *zg, double *det)
{
    double p[2][4], f[4], xj[2][3];
    double sp = 1.0 + g2, sm = 1.0 - g2;
    p[0][0] = -0.250 * sm;
    p[0][1] = 0.250 * sm;
    p[0][2] = 0.250 * sp;
    p[0][3] = -0.250 * sp;
    double rp = 1.0 + g1, rm = 1.0 - g1;
    f[0] = 0.250 * rm * sm;
    f[1] = 0.250 * rp * sm;
    f[2] = 0.250 * rp * sp;
    f[3] = 0.250 * rm * sp;
    p[1][0] = -0.250 * rm;
    p[1][1] = -0.250 * rp;
    p[1][2] = 0.250 * rp;
    p[1][3] = 0.250 * rm;
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 3; ++j) {
            double temp = 0.0;
            for (int k = 0; k < 4; ++k) temp = temp + p[i][k] * co[k][j];
            xj[i][j] = temp;
        }
    double d1 = xj[0][1] * xj[1][2] - xj[1][1] * xj[0][2];
    double d2 = xj[1][0] * xj[0][2] - xj[0][0] * xj[1][2];
    double d3 = xj[0][0] * xj[1][1] - xj[1][0] * xj[0][1];
    *det = sqrt(d1 * d1 + d2 * d2 + d3 * d3);
    if (*det < 1.0e-5) return ORC_DEGENERATE;
    double x = 0.0, y = 0.0, z = 0.0;
    for (int i = 0; i < 4; ++i) {
        x = x + co[i][0] * f[i];
        y = y + co[i][1] * f[i];
        z = z + co[i][2] * f[i];
    }
    *xg = x; *yg = y; *zg = z;
    return ORC_OK;
}

/* Solfune.for:18-31, accumulated with weight p12 (Nonsinge.for:112-115). */
static void solfune_acc(double t[3][3], double cxp, double cyp, double czp,
                        double cxg, double cyg, double czg, const double *eta,
                        double c3, double c4, double p12)
{
    double r1 = cxg - cxp, r2 = cyg - cyp, r3 = czg - czp;
    double r = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
    double rdn = (r1 * eta[0] + r2 * eta[1] + r3 * eta[2]) / r;
    double rd[3] = {r1 / r, r2 / r, r3 / r};
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double v = (c3 / (r * r)) *
                       (rdn * (c4 * kDelta[i][j] + 3.0 * rd[i] * rd[j]) +
                        c4 * (rd[j] * eta[i] - rd[i] * eta[j]));
            t[j][i] += v * p12; /* t[j][i] == T(I,J) column-major */
        }
}

/* Singge.for:195-198 (SOLFUNE_G), accumulated as in Singge.for:161-163. */
static void solfune_g_acc(double u[3][3], double cxp, double cyp, double czp,
                          double cxg, double cyg, double czg, double c1,
                          double c2, double p12)
{
    double r1 = cxg - cxp, r2 = cyg - cyp, r3 = czg - czp;
    double r = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
    double rd[3] = {r1 / r, r2 / r, r3 / r};
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i)
            u[j][i] += ((c1 / r) * (c2 * kDelta[i][j] + rd[i] * rd[j])) * p12;
}

/* Nonsinge.for:12-121: static T over one element, collocation (xp,yp,zp). */
static int nonsinge(double helem[3][3], const double co[4][3], double xp,
                    double yp, double zp, const double *eta, int npg,
                    const double *gi, const double *ome, double c3, double c4)
{
    memset(helem, 0, 9 * sizeof(double));
    for (int jg = 0; jg < npg; ++jg) {
        double g2 = gi[jg], p2 = ome[jg];
        for (int ig = 0; ig < npg; ++ig) {
            double g1 = gi[ig], p1 = ome[ig];
            double xg, yg, zg, det;
            if (gauss_point(co, g1, g2, &xg, &yg, &zg, &det)) return ORC_DEGENERATE;
            double p12 = p1 * p2 * det;
            solfune_acc(helem, xp, yp, zp, xg, yg, zg, eta, c3, c4, p12);
        }
    }
    return ORC_OK;
}

/* Singge.for:83-173 (NONSINGE_G). */
static int nonsinge_g(double gelem[3][3], const double co[4][3], double xp,
                      double yp, double zp, int npg, const double *gi,
                      const double *ome, double c1, double c2)
{
    memset(gelem, 0, 9 * sizeof(double));
    for (int jg = 0; jg < npg; ++jg) {
        double g2 = gi[jg], p2 = ome[jg];
        for (int ig = 0; ig < npg; ++ig) {
            double g1 = gi[ig], p1 = ome[ig];
            double xg, yg, zg, det;
            if (gauss_point(co, g1, g2, &xg, &yg, &zg, &det)) return ORC_DEGENERATE;
            solfune_g_acc(gelem, xp, yp, zp, xg, yg, zg, c1, c2, p1 * p2 * det);
        }
    }
    return ORC_OK;
}

/* Singge.for:11-81: 4 collapsed triangles (corners 3,4 -> centroid). */
static int singge(double gelem[3][3], double xm, double ym, double zm,
                  const double co_el[4][3], int npg, const double *gi,
                  const double *ome, double c1, double c2)
{
    double co[4][3], gp[3][3];
    co[2][0] = xm; co[2][1] = ym; co[2][2] = zm;
    co[3][0] = xm; co[3][1] = ym; co[3][2] = zm;
    memset(gelem, 0, 9 * sizeof(double));
    for (int it = 0; it < 4; ++it) {
        int a = it, b = (it + 1) % 4; /* edges (1,2),(2,3),(3,4),(4,1) */
        for (int c = 0; c < 3; ++c) {
            co[0][c] = co_el[a][c];
            co[1][c] = co_el[b][c];
        }
        if (nonsinge_g(gp, (const double (*)[3])co, xm, ym, zm, npg, gi, ome, c1, c2))
            return ORC_DEGENERATE;
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) gelem[j][i] = gelem[j][i] + gp[j][i];
    }
    return ORC_OK;
}

int orc_ghmatece(int n, int nbe, int np, int npg, const int *cone,
                 const double *cx, const double *cy, const double *cz,
                 const double *cxm, const double *cym, const double *czm,
                 const double *etas, const double *gi, const double *ome,
                 double rmu, double rnu, double *hestdiag, double *gestdiag,
                 double *hest)
{
    (void)np;
    double c[4];
    orc_static_consts(rmu, rnu, c);
    const int nn = 3 * nbe;
    int status = ORC_OK;
    /* Every 3x3 block of HEST; HESTdiag is summed from them afterwards. */
    double *blocks = malloc((size_t)9 * nbe * n * sizeof(double));
    if (!blocks) return -1;

    /* Ghmatece.for:92-150: OMP DO over J; block (I,J) = NONSINGE, I==J zero. */
#pragma omp parallel for schedule(dynamic, 4) reduction(max : status)
    for (int j = 0; j < n; ++j) {
        double co[4][3];
        load_co(n, j, cone, cx, cy, cz, co);
        for (int i = 0; i < nbe; ++i) {
            double *blk = blocks + 9 * ((size_t)j * nbe + i);
            if (i == j) {
                memset(blk, 0, 9 * sizeof(double));
            } else {
                double helem[3][3];
                int s = nonsinge(helem, (const double (*)[3])co, cxm[i], cym[i],
                                 czm[i], etas + 3 * j, npg, gi, ome, c[2], c[3]);
                if (s > status) status = s;
                memcpy(blk, helem, 9 * sizeof(double));
            }
        }
    }
    if (hest) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < nbe; ++i)
                for (int jj = 0; jj < 3; ++jj)
                    for (int ii = 0; ii < 3; ++ii)
                        hest[(size_t)(3 * j + jj) * nn + 3 * i + ii] =
                            blocks[9 * ((size_t)j * nbe + i) + 3 * jj + ii];
    }
    /* RIGID_BODY, Ghmatece.for:258-282: HESTdiag(:,:,MA) = -sum_MB
     * HEST(block MA, MB), summed in the reference's MB order. */
#pragma omp parallel for
    for (int a = 0; a < nbe; ++a) {
        double acc[9] = {0};
        for (int b = 0; b < n; ++b) {
            const double *blk = blocks + 9 * ((size_t)b * nbe + a);
            for (int k = 0; k < 9; ++k) acc[k] = acc[k] - blk[k];
        }
        memcpy(hestdiag + 9 * a, acc, sizeof acc);
    }
    free(blocks);

    /* GEST_SINGULAR, Ghmatece.for:288-323. */
#pragma omp parallel for reduction(max : status)
    for (int j = 0; j < nbe; ++j) {
        double co[4][3], g[3][3];
        load_co(n, j, cone, cx, cy, cz, co);
        int s = singge(g, cxm[j], cym[j], czm[j], (const double (*)[3])co, npg,
                       gi, ome, c[0], c[1]);
        if (s > status) status = s;
        memcpy(gestdiag + 9 * j, g, 9 * sizeof(double));
    }
    return status;
}

/* Dynamic constants of Solfund.for:29-35 (independent of the point). */
typedef struct {
    zc zc0, zc1, zc2, zkp, zks;
    double pi;
} dyn_consts;

static dyn_consts make_dyn(zc zge, zc zcs, zc zcp, double fr)
{
    dyn_consts d;
    d.pi = 4.0 * atan(1.0);
    zc zwi = I * fr;
    d.zc0 = 1.0 / ((4.0 * d.pi) * zge);
    d.zc1 = (zcp / zcs) * (zcp / zcs);
    d.zc2 = (zcs / zcp) * (zcs / zcp);
    d.zkp = -zwi / zcp;
    d.zks = -zwi / zcs;
    return d;
}

/* The radial functions of Solfund.for:36-49. */
typedef struct {
    zc fhi, cappa, fhidr, cappadr, aa, bb, cc;
} stokes_radial;

static stokes_radial stokes(const dyn_consts *d, double r)
{
    stokes_radial s;
    zc zzp = d->zkp * r, zzs = d->zks * r;
    zc zezp = cexp(zzp), zezs = cexp(zzs);
    zc zp2 = zzp * zzp, zs2 = zzs * zzs;
    zc zc2 = d->zc2;
    s.fhi = (1.0 + 1.0 / zs2 - 1.0 / zzs) * zezs / r -
            zc2 * (1.0 / zp2 - 1.0 / zzp) * zezp / r;
    s.cappa = (1.0 + 3.0 / zs2 - 3.0 / zzs) * zezs / r -
              zc2 * (1.0 + 3.0 / zp2 - 3.0 / zzp) * zezp / r;
    s.fhidr = (-2.0 + zzs + 3.0 / zzs - 3.0 / zs2) * zezs / (r * r) -
              zc2 * (-1.0 + 3.0 / zzp - 3.0 / zp2) * zezp / (r * r);
    s.cappadr = (zzs - 4.0 + 9.0 / zzs - 9.0 / zs2) * zezs / (r * r) -
                zc2 * (zzp - 4.0 + 9.0 / zzp - 9.0 / zp2) * zezp / (r * r);
    s.aa = s.fhidr - s.cappa / r;
    s.bb = 4.0 * s.cappa / r - 2.0 * s.cappadr;
    s.cc = (d->zc1 - 2.0) * (s.aa + 5.0e-1 * s.bb - 3.0 * s.cappa / r) -
           2.0 * s.cappa / r;
    return s;
}

/* Solfund.for:18-60.  zu[j][i] == ZU(I,J). */
static void solfund(zc zu[3][3], zc zt[3][3], const dyn_consts *d, double cxp,
                    double cyp, double czp, double cxg, double cyg, double czg,
                    const double *rn)
{
    double r1 = cxg - cxp, r2 = cyg - cyp, r3 = czg - czp;
    double r = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
    double drn = (r1 * rn[0] + r2 * rn[1] + r3 * rn[2]) / r;
    double rd[3] = {r1 / r, r2 / r, r3 / r};
    stokes_radial s = stokes(d, r);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            zu[j][i] = d->zc0 * (s.fhi * kDelta[i][j] - s.cappa * rd[j] * rd[i]);
            zt[j][i] = (1.0 / (4.0 * d->pi)) *
                       ((s.aa * (drn * kDelta[i][j] + rd[j] * rn[i])) +
                        rd[i] * rd[j] * drn * s.bb + rd[i] * rn[j] * s.cc);
        }
}

/* Solfundif.for:18-69: Stokes minus Kelvin. */
static void solfundif(zc zu[3][3], zc zt[3][3], const dyn_consts *d,
                      const double *c, double cxp, double cyp, double czp,
                      double cxg, double cyg, double czg, const double *rn)
{
    double r1 = cxg - cxp, r2 = cyg - cyp, r3 = czg - czp;
    double r = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
    double drn = (r1 * rn[0] + r2 * rn[1] + r3 * rn[2]) / r;
    double rd[3] = {r1 / r, r2 / r, r3 / r};
    stokes_radial s = stokes(d, r);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            zu[j][i] = d->zc0 * (s.fhi * kDelta[i][j] - s.cappa * rd[j] * rd[i]) -
                       (c[0] / r) * (c[1] * kDelta[i][j] + rd[i] * rd[j]);
            zt[j][i] = (1.0 / (4.0 * d->pi)) *
                           ((s.aa * (drn * kDelta[i][j] + rd[j] * rn[i])) +
                            rd[i] * rd[j] * drn * s.bb + rd[i] * rn[j] * s.cc) -
                       (c[2] / (r * r)) *
                           (drn * (c[3] * kDelta[i][j] + 3.0 * rd[i] * rd[j]) +
                            c[3] * (rd[j] * rn[i] - rd[i] * rn[j]));
        }
}

void orc_solfund(const double *p, const double *g, const double *rn,
                 const double *zge, const double *zcs, const double *zcp,
                 double fr, double *zu, double *zt)
{
    dyn_consts d = make_dyn(zge[0] + I * zge[1], zcs[0] + I * zcs[1],
                            zcp[0] + I * zcp[1], fr);
    zc u[3][3], t[3][3];
    solfund(u, t, &d, p[0], p[1], p[2], g[0], g[1], g[2], rn);
    memcpy(zu, u, sizeof u);
    memcpy(zt, t, sizeof t);
}

/* Nonsingd.for:11-122 (diff=0) and Sing_de.for:13-113 (diff=1). */
static int nonsingd(zc zh[3][3], zc zg[3][3], const double co[4][3],
                    double xp, double yp, double zp, const double *eta,
                    const dyn_consts *d, const double *c, int diff, int npg,
                    const double *gi, const double *ome)
{
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) zh[j][i] = zg[j][i] = 0.0;
    for (int jg = 0; jg < npg; ++jg) {
        double g2 = gi[jg], p2 = ome[jg];
        for (int ig = 0; ig < npg; ++ig) {
            double g1 = gi[ig], p1 = ome[ig];
            double xg, yg, zgp, det;
            if (gauss_point(co, g1, g2, &xg, &yg, &zgp, &det)) return ORC_DEGENERATE;
            zc zu[3][3], zt[3][3];
            if (diff)
                solfundif(zu, zt, d, c, xp, yp, zp, xg, yg, zgp, eta);
            else
                solfund(zu, zt, d, xp, yp, zp, xg, yg, zgp, eta);
            double p12 = p1 * p2 * det;
            for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 3; ++i) {
                    zh[j][i] = zh[j][i] + zt[j][i] * p12;
                    zg[j][i] = zg[j][i] + zu[j][i] * p12;
                }
        }
    }
    return ORC_OK;
}

int orc_ghmatecd(int n, int nbe, int np, int npg, const int *cone,
                 const double *cx, const double *cy, const double *cz,
                 const double *cxm, const double *cym, const double *czm,
                 const double *etas, const double *gi, const double *ome,
                 const double *c, const double *zge, const double *zcs,
                 const double *zcp, double fr, const double *hestdiag,
                 const double *gestdiag, double *zh_, double *zg_)
{
    return orc_ghmatecd_cols(n, nbe, np, npg, cone, cx, cy, cz, cxm, cym, czm,
                             etas, gi, ome, c, zge, zcs, zcp, fr, hestdiag,
                             gestdiag, 0, nbe, zh_, zg_);
}

int orc_ghmatecd_cols(int n, int nbe, int np, int npg, const int *cone,
                      const double *cx, const double *cy, const double *cz,
                      const double *cxm, const double *cym, const double *czm,
                      const double *etas, const double *gi, const double *ome,
                      const double *c, const double *zge, const double *zcs,
                      const double *zcp, double fr, const double *hestdiag,
                      const double *gestdiag, int jlo, int jhi, double *zh_,
                      double *zg_)
{
    (void)np;
    const int nn = 3 * nbe;
    zc *zh = (zc *)zh_, *zg = (zc *)zg_;
    dyn_consts d = make_dyn(zge[0] + I * zge[1], zcs[0] + I * zcs[1],
                            zcp[0] + I * zcp[1], fr);
    int status = ORC_OK;
    /* Ghmatecd.for:113-166 (element columns jlo..jhi-1). */
#pragma omp parallel for schedule(dynamic, 4) reduction(max : status)
    for (int j = jlo; j < jhi; ++j) {
        double co[4][3];
        load_co(n, j, cone, cx, cy, cz, co);
        for (int i = 0; i < nbe; ++i) {
            zc h[3][3], g[3][3];
            int diag = (i == j);
            int s = nonsingd(h, g, (const double (*)[3])co, cxm[i], cym[i], czm[i],
                             etas + 3 * j, &d, c, diag, npg, gi, ome);
            if (s > status) status = s;
            if (diag) { /* Ghmatecd.for:150-153 */
                for (int jj = 0; jj < 3; ++jj)
                    for (int ii = 0; ii < 3; ++ii) {
                        g[jj][ii] = g[jj][ii] + gestdiag[9 * i + 3 * jj + ii];
                        h[jj][ii] = h[jj][ii] + hestdiag[9 * i + 3 * jj + ii];
                    }
            }
            for (int jj = 0; jj < 3; ++jj)
                for (int ii = 0; ii < 3; ++ii) {
                    size_t idx = (size_t)(3 * j + jj) * nn + 3 * i + ii;
                    zh[idx] = h[jj][ii];
                    zg[idx] = g[jj][ii];
                }
        }
    }
    return status;
}

void orc_boundary_conditions(int nn, double *zh_, double *zg_, const int *kode,
                             const double *zge_)
{
    zc *zh = (zc *)zh_, *zg = (zc *)zg_;
    zc zge = zge_[0] + I * zge_[1];
    /* Ghmatecd.for:324-332 with the dummies bound as at :168
     * (dummy ZG <- actual ZH, dummy ZH <- actual ZG). */
    for (int j = 0; j < nn; ++j) {
        if (kode[j] != 0) continue;
        for (int i = 0; i < nn; ++i) {
            size_t k = (size_t)j * nn + i;
            zc zch = zh[k] * zge;
            zh[k] = -zg[k];
            zg[k] = -zch;
        }
    }
}

void orc_zgemv(int nn, const double *a_, const double *x_, double *y_)
{
    const zc *a = (const zc *)a_, *x = (const zc *)x_;
    zc *y = (zc *)y_;
    for (int i = 0; i < nn; ++i) y[i] = 0.0;
    /* Column-oriented as in the reference BLAS ZGEMV 'N'. */
    for (int j = 0; j < nn; ++j) {
        zc t = x[j];
        if (t == 0.0) continue;
        const zc *col = a + (size_t)j * nn;
        for (int i = 0; i < nn; ++i) y[i] = y[i] + t * col[i];
    }
}

static inline double cabs1(zc z) { return fabs(creal(z)) + fabs(cimag(z)); }

int orc_zgesv(int nn, double *a_, int *ipiv, double *b_)
{
    zc *a = (zc *)a_, *b = (zc *)b_;
    int info = 0;
    /* ZGETRF, right-looking, one column at a time. */
    for (int k = 0; k < nn; ++k) {
        zc *colk = a + (size_t)k * nn;
        int p = k;
        double best = cabs1(colk[k]);
        for (int i = k + 1; i < nn; ++i) {
            double v = cabs1(colk[i]);
            if (v > best) { best = v; p = i; }
        }
        ipiv[k] = p + 1;
        if (colk[p] == 0.0) {
            if (info == 0) info = k + 1;
            continue;
        }
        if (p != k)
            for (int j = 0; j < nn; ++j) {
                zc *cj = a + (size_t)j * nn;
                zc t = cj[k]; cj[k] = cj[p]; cj[p] = t;
            }
        zc rpiv = 1.0 / colk[k];
        for (int i = k + 1; i < nn; ++i) colk[i] = colk[i] * rpiv;
#pragma omp parallel for if (nn - k > 256)
        for (int j = k + 1; j < nn; ++j) {
            zc *cj = a + (size_t)j * nn;
            zc u = cj[k];
            if (u == 0.0) continue;
            for (int i = k + 1; i < nn; ++i) cj[i] = cj[i] - colk[i] * u;
        }
    }
    if (info) return ORC_SINGULAR;
    /* ZGETRS 'N': b <- P b, L y = b, U x = y. */
    for (int k = 0; k < nn; ++k) {
        int p = ipiv[k] - 1;
        if (p != k) { zc t = b[k]; b[k] = b[p]; b[p] = t; }
    }
    for (int j = 0; j < nn; ++j) {
        zc t = b[j];
        if (t == 0.0) continue;
        const zc *cj = a + (size_t)j * nn;
        for (int i = j + 1; i < nn; ++i) b[i] = b[i] - t * cj[i];
    }
    for (int j = nn - 1; j >= 0; --j) {
        const zc *cj = a + (size_t)j * nn;
        b[j] = b[j] / cj[j];
        zc t = b[j];
        for (int i = 0; i < j; ++i) b[i] = b[i] - t * cj[i];
    }
    return ORC_OK;
}

void orc_unswap(int nn, const int *kode, const double *zge_, double *zfi_,
                double *zdfi_)
{
    zc *zfi = (zc *)zfi_, *zdfi = (zc *)zdfi_;
    zc zge = zge_[0] + I * zge_[1];
    for (int i = 0; i < nn; ++i) {
        if (kode[i] == 0) {
            zc zch = zfi[i] * zge;
            zfi[i] = zdfi[i];
            zdfi[i] = zch;
        }
    }
}

int orc_interior_disp(int n, int nbe, int np, int npg, const int *cone,
                      const double *cx, const double *cy, const double *cz,
                      const double *etas, const double *gi, const double *ome,
                      int l, const double *cxi, const double *cyi,
                      const double *czi, const double *zge, const double *zcs,
                      const double *zcp, double fr, const double *zfi_,
                      const double *zdfi_, double *zdsol_)
{
    (void)np;
    const zc *zfi = (const zc *)zfi_, *zdfi = (const zc *)zdfi_;
    zc *zdsol = (zc *)zdsol_;
    dyn_consts d = make_dyn(zge[0] + I * zge[1], zcs[0] + I * zcs[1],
                            zcp[0] + I * zcp[1], fr);
    int status = ORC_OK;
    for (int k = 0; k < 3 * l; ++k) zdsol[k] = 0.0;
    /* Interec.for:86-135; per-J partials are summed in J order so the
     * result does not depend on the thread count. */
    zc *part = calloc((size_t)nbe * 3 * l, sizeof(zc));
    if (!part) return -1;
#pragma omp parallel for schedule(dynamic, 4) reduction(max : status)
    for (int j = 0; j < nbe; ++j) {
        double co[4][3];
        load_co(n, j, cone, cx, cy, cz, co);
        for (int k = 0; k < l; ++k) {
            zc h[3][3], g[3][3];
            int s = nonsingd(h, g, (const double (*)[3])co, cxi[k], cyi[k], czi[k],
                             etas + 3 * j, &d, NULL, 0, npg, gi, ome);
            if (s > status) status = s;
            for (int i = 0; i < 3; ++i) {
                zc acc = 0.0, acc2 = 0.0;
                for (int jj = 0; jj < 3; ++jj) {
                    acc = acc + g[jj][i] * zdfi[3 * j + jj];
                    acc2 = acc2 + h[jj][i] * zfi[3 * j + jj];
                }
                part[(size_t)j * 3 * l + 3 * k + i] = acc - acc2;
            }
        }
    }
    for (int j = 0; j < nbe; ++j)
        for (int k = 0; k < 3 * l; ++k) zdsol[k] += part[(size_t)j * 3 * l + k];
    free(part);
    return status;
}

/* Sigmaec.for:9-212: ZD(3,3,3), ZS(3,3,3) stored zd[(j*3+i)*3+k] == ZD(K,I,J). */
static int sigmaec(zc zd[27], zc zs[27], const double co[4][3], double cxp,
                   double cyp, double czp, const double *rn,
                   const dyn_consts *d, zc zge, zc zcs, zc zcp, double rho,
                   double fr, int npg, const double *gi, const double *ome)
{
    const double pi = d->pi;
    for (int k = 0; k < 27; ++k) zd[k] = zs[k] = 0.0;
    zc zwi = I * fr;
    for (int jg = 0; jg < npg; ++jg) {
        double g2 = gi[jg], p2 = ome[jg];
        for (int ig = 0; ig < npg; ++ig) {
            double g1 = gi[ig], p1 = ome[ig];
            double cxg, cyg, czg, det;
            if (gauss_point(co, g1, g2, &cxg, &cyg, &czg, &det)) return ORC_DEGENERATE;
            double r1 = cxg - cxp, r2 = cyg - cyp, r3 = czg - czp;
            double r = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
            double drn = (r1 * rn[0] + r2 * rn[1] + r3 * rn[2]) / r;
            double rd[3] = {r1 / r, r2 / r, r3 / r};
            stokes_radial s = stokes(d, r);
            zc zk1 = zwi / zcp, zk2 = zwi / zcs;
            zc zek1 = cexp(-zk1 * r), zek2 = cexp(-zk2 * r);
            zc zmu = zge;
            zc zlamb = (zcp * zcp * rho) - (2.0 * zmu);
            zc k1r = zk1 * r, k2r = zk2 * r;
            zc k1r2 = k1r * k1r, k2r2 = k2r * k2r;
            double r3c = r * r * r;
            zc zcszcp = (zcs / zcp) * (zcs / zcp);
            zc zfhidrr =
                -(zcszcp * zek1 * (12.0 + 12.0 * zk1 * r + 5.0 * k1r2 + k1r2 * k1r) *
                  (1.0 / (k1r2 * r3c))) +
                zek2 * (12.0 + 12.0 * zk2 * r + 7.0 * k2r2 + 3.0 * (k2r2 * k2r) +
                        k2r2 * k2r2) *
                    (1.0 / (k2r2 * r3c));
            zc zcappadrr =
                -(zcszcp * zek1 *
                  (36.0 + 36.0 * zk1 * r + 17.0 * k1r2 + 5.0 * (k1r2 * k1r) +
                   k1r2 * k1r2) *
                  (1.0 / (k1r2 * r3c))) +
                zek2 *
                    (36.0 + 36.0 * zk2 * r + 17.0 * k2r2 + 5.0 * (k2r2 * k2r) +
                     k2r2 * k2r2) *
                    (1.0 / (k2r2 * r3c));
            zc zcappa = s.cappa, zfhidr = s.fhidr, zcappadr = s.cappadr;
            double r2s = r * r;
            zc lm = zlamb / zmu;
            zc zcte1 = 2.0 * (zcappa / r);
            zc zcte2 = lm * (zfhidr - zcappadr - zcte1);
            zc zcte3 = (zfhidr - zcappa / r);
            zc zcte4 = 2.0 * (zcappadr - zcte1);
            zc zcte5 = 4.0 * (zcappadrr - 5.0 * (zcappadr / r) + 8.0 * (zcappa / r2s));
            zc zcte6 = zfhidrr - (zfhidr / r) - 3.0 * (zcappadr / r) +
                       6.0 * (zcappa / r2s);
            zc zcte7 = 2.0 * (zcappadr / r) - 4.0 * (zcappa / r2s);
            zc zcte8 = lm * (zcappadrr + (zcappadr / r) - 4.0 * (zcappa / r2s) -
                             zfhidrr + (zfhidr / r));
            zc zcte9 = 2.0 * (zcte7 + zcte8);
            zc zcte10 = 4.0 * (zcappa / r2s) +
                        4.0 * lm * ((zcappadr / r) + 2.0 * (zcappa / r2s) - (zfhidr / r));
            zc zcte11 = (lm * lm) * (zcappadrr + 4.0 * (zcappadr / r) +
                                     2.0 * (zcappa / r2s) - zfhidrr -
                                     2.0 * (zfhidr / r));
            zc zcte12 = 2.0 * ((zfhidr / r) - (zcappa / r2s));
            double p12 = p1 * p2 * det;
            for (int kk = 0; kk < 3; ++kk)
                for (int ii = 0; ii < 3; ++ii)
                    for (int jj = 0; jj < 3; ++jj) {
                        double dji = kDelta[jj][ii], djk = kDelta[jj][kk],
                               dik = kDelta[ii][kk];
                        zc zdp = (1.0 / (4.0 * pi)) *
                                 ((zcte1 - zcte2) * dji * rd[kk] -
                                  zcte3 * (djk * rd[ii] + dik * rd[jj]) +
                                  zcte4 * rd[jj] * rd[ii] * rd[kk]);
                        zc zsp = (zmu / (4.0 * pi)) *
                                 ((zcte5 * rd[jj] * rd[ii] * rd[kk] -
                                   zcte6 * (djk * rd[ii] + dik * rd[jj]) +
                                   zcte9 * dji * rd[kk]) *
                                      drn +
                                  zcte9 * rd[jj] * rd[ii] * rn[kk] -
                                  zcte6 * (rd[ii] * rn[jj] + rd[jj] * rn[ii]) * rd[kk] +
                                  (zcte10 + zcte11) * dji * rn[kk] -
                                  zcte12 * (dik * rn[jj] + djk * rn[ii]));
                        int idx = (jj * 3 + ii) * 3 + kk;
                        zd[idx] = zd[idx] + zdp * p12;
                        zs[idx] = zs[idx] + zsp * p12;
                    }
        }
    }
    return ORC_OK;
}

int orc_interior_stress(int n, int nbe, int np, int npg, const int *cone,
                        const double *cx, const double *cy, const double *cz,
                        const double *etas, const double *gi,
                        const double *ome, int l, const double *cxi,
                        const double *cyi, const double *czi,
                        const double *zge_, const double *zcs_,
                        const double *zcp_, double rho, double fr,
                        const double *zfi_, const double *zdfi_, double *zssol_)
{
    (void)np;
    const zc *zfi = (const zc *)zfi_, *zdfi = (const zc *)zdfi_;
    zc *zssol = (zc *)zssol_;
    zc zge = zge_[0] + I * zge_[1], zcs = zcs_[0] + I * zcs_[1],
       zcp = zcp_[0] + I * zcp_[1];
    dyn_consts d = make_dyn(zge, zcs, zcp, fr);
    int status = ORC_OK;
    /* Interec.for:188-283: ZSSOL(9K-9+m) with m-1 = (I-1)+3(J-1) collects
     * sum_k ZDFI(3J'-3+k) ZD(k,I,J) - ZFI(3J'-3+k) ZS(k,I,J). */
#pragma omp parallel for schedule(dynamic, 1) reduction(max : status)
    for (int k = 0; k < l; ++k) {
        zc acc[9] = {0};
        for (int j = 0; j < nbe; ++j) {
            double co[4][3];
            zc zd[27], zs[27];
            load_co(n, j, cone, cx, cy, cz, co);
            int s = sigmaec(zd, zs, (const double (*)[3])co, cxi[k], cyi[k], czi[k],
                            etas + 3 * j, &d, zge, zcs, zcp, rho, fr, npg, gi, ome);
            if (s > status) status = s;
            for (int jj = 0; jj < 3; ++jj)
                for (int ii = 0; ii < 3; ++ii) {
                    int m = ii + 3 * jj;
                    const zc *dd = zd + (jj * 3 + ii) * 3;
                    const zc *ss = zs + (jj * 3 + ii) * 3;
                    acc[m] = acc[m] + zdfi[3 * j] * dd[0] + zdfi[3 * j + 1] * dd[1] +
                             zdfi[3 * j + 2] * dd[2] - zfi[3 * j] * ss[0] -
                             zfi[3 * j + 1] * ss[1] - zfi[3 * j + 2] * ss[2];
                }
        }
        for (int m = 0; m < 9; ++m) zssol[9 * k + m] = acc[m];
    }
    return status;
}

/* EXTENSION (the reference never solves a static system: it only keeps
 * HESTdiag and GESTdiag): the static boundary solve assembled from the
 * reference's own static pieces.  H: off-diagonal 3x3 blocks NONSINGE
 * (Kelvin T, Nonsinge.for:12-121), diagonal blocks HESTdiag (rigid body,
 * Ghmatece.for:258-282).  G: off-diagonal blocks NONSINGE_G (Kelvin U,
 * Singge.for:83-173 with SOLFUNE_G, Singge.for:195-198) over the element's
 * own four corners, diagonal blocks GESTdiag (SINGGE, Singge.for:11-81).
 * Rows and columns over the NBE boundary elements, as in GHMATECD; then the
 * boundary-condition swap of Ghmatecd.for:316-333 with the real GE, the
 * right-hand side G*DFI, the solve (ZGESV restated, imaginary parts zero)
 * and the un-swap of Interec.for:59-67.  h_out / g_out (nn x nn, after the
 * swap, column-major) may be NULL. */
int orc_static_solve(int n, int nbe, int np, int npg, const int *cone,
                     const double *cx, const double *cy, const double *cz,
                     const double *cxm, const double *cym, const double *czm,
                     const double *etas, const double *gi, const double *ome,
                     double ge, double rnu, const int *kode, const double *dfi,
                     double *disp, double *trac, double *h_out, double *g_out)
{
    const int nn = 3 * nbe;
    double c[4];
    orc_static_consts(ge, rnu, c);
    double *hd = malloc((size_t)9 * nbe * sizeof(double));
    double *gd = malloc((size_t)9 * nbe * sizeof(double));
    double *h = malloc((size_t)nn * nn * sizeof(double));
    double *g = malloc((size_t)nn * nn * sizeof(double));
    double *a = malloc((size_t)2 * nn * nn * sizeof(double));
    double *b = malloc((size_t)2 * nn * sizeof(double));
    int *ipiv = malloc((size_t)nn * sizeof(int));
    int status = -1;
    if (!hd || !gd || !h || !g || !a || !b || !ipiv) goto out;
    status = orc_ghmatece(n, nbe, np, npg, cone, cx, cy, cz, cxm, cym, czm, etas, gi, ome, ge,
                          rnu, hd, gd, NULL);
#pragma omp parallel for schedule(dynamic, 4) reduction(max : status)
    for (int j = 0; j < nbe; ++j) {
        double co[4][3];
        load_co(n, j, cone, cx, cy, cz, co);
        for (int i = 0; i < nbe; ++i) {
            double he[3][3], gel[3][3];
            if (i == j) {
                memcpy(he, hd + 9 * j, sizeof he);
                memcpy(gel, gd + 9 * j, sizeof gel);
            } else {
                int s = nonsinge(he, (const double (*)[3])co, cxm[i], cym[i], czm[i],
                                 etas + 3 * j, npg, gi, ome, c[2], c[3]);
                int s2 = nonsinge_g(gel, (const double (*)[3])co, cxm[i], cym[i], czm[i], npg,
                                    gi, ome, c[0], c[1]);
                if (s > status) status = s;
                if (s2 > status) status = s2;
            }
            for (int jj = 0; jj < 3; ++jj)
                for (int ii = 0; ii < 3; ++ii) {
                    size_t k = (size_t)(3 * j + jj) * nn + 3 * i + ii;
                    h[k] = he[jj][ii];
                    g[k] = gel[jj][ii];
                }
        }
    }
    /* Ghmatecd.for:324-332 (effective semantics) with real GE. */
    for (int col = 0; col < nn; ++col) {
        if (kode[col] != 0) continue;
        for (int i = 0; i < nn; ++i) {
            size_t k = (size_t)col * nn + i;
            double hg = h[k] * ge;
            h[k] = -g[k];
            g[k] = -hg;
        }
    }
    for (int i = 0; i < nn; ++i) {
        double acc = 0.0;
        for (int col = 0; col < nn; ++col) acc += g[(size_t)col * nn + i] * dfi[col];
        b[2 * i] = acc;
        b[2 * i + 1] = 0.0;
    }
    for (size_t k = 0; k < (size_t)nn * nn; ++k) {
        a[2 * k] = h[k];
        a[2 * k + 1] = 0.0;
    }
    if (h_out) memcpy(h_out, h, (size_t)nn * nn * sizeof(double));
    if (g_out) memcpy(g_out, g, (size_t)nn * nn * sizeof(double));
    if (orc_zgesv(nn, a, ipiv, b) != 0) {
        status = ORC_SINGULAR;
        goto out;
    }
    /* Interec.for:59-67 with real GE. */
    for (int i = 0; i < nn; ++i) {
        if (kode[i] == 0) {
            disp[i] = dfi[i];
            trac[i] = b[2 * i] * ge;
        } else {
            disp[i] = b[2 * i];
            trac[i] = dfi[i];
        }
    }
out:
    free(hd);
    free(gd);
    free(h);
    free(g);
    free(a);
    free(b);
    free(ipiv);
    return status;
}

