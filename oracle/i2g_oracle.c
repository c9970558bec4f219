/*
 * TEST INFRASTRUCTURE ONLY -- the oracle.  Sequential C restatement of the
 * I2ELVIS marker step; the CUDA path is checked against it and it is itself
 * pinned against the compiled, unmodified reference (oracle/_ref/ref64, built by
 * oracle/Makefile) on the same seeded inputs.
 *
 * Every function states the reference lines it follows.  Arithmetic is written
 * in the reference's evaluation order and built with -ffp-contract=off, so with
 * the same libm it reproduces the reference bit for bit.
 *
 * Scope (the rest is rejected by the product with I2G_EUNSUPPORTED): intermod =
 * intermod1 = 0, densimod 0|1|2, no immobile markers (type >= 100).  Radiogenic heating of rock types outside
 * the reference's lists (markmart.c:749-837) is 0 here; the reference leaves it
 * at the previous marker's value.
 */
#include "i2g_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ABSV(a) ((a) >= 0 ? (a) : -(a))

/* m1serch()/m2serch(), markmart.c:1051-1088: bisection for the last grid line
 * not right of x, clamped to n-2. */
int64_t ora_m1serch(const double *g, int64_t n, double x)
{
    int64_t m, m0 = 0, m1 = n - 1;
    do {
        m = (m0 + m1) / 2;
        if (g[m] > x) m1 = m; else m0 = m;
    } while ((m1 - m0) > 1);
    if (m0 > n - 2) m0 = n - 2;
    return m0;
}

/* fdweight(1, 0, xi), movemart.c:1269-1319, for two points: order-0 (linear)
 * interpolation weights, written in the recurrence's own operation order. */
void ora_fdweight1(double x0, double x1, double xi, double *w0, double *w1)
{
    double c5 = x0 - xi;   /* c4 before the i=1 update (movemart.c:1282) */
    double c4 = x1 - xi;   /* movemart.c:1297 */
    double c3 = x1 - x0;   /* movemart.c:1300; c2 = 1.0*c3 */
    *w1 = (-c5) / c3;      /* cn[1][0] = -c1*c5*cn[0][0]/c2, movemart.c:1307 */
    *w0 = c4 / c3;         /* cn[0][0] = c4*cn[0][0]/c3, movemart.c:1313 */
}

static double bil(const double *f, int64_t ny, int64_t m1, int64_t m2, double wx0, double wx1,
                  double wy0, double wy1)
{
    /* loop m1 outer, m2 inner, starting from 0 (markmart.c:1414-1421) */
    double s = 0;
    s += (wx0 * wy0) * f[m1 * ny + m2];
    s += (wx0 * wy1) * f[m1 * ny + m2 + 1];
    s += (wx1 * wy0) * f[(m1 + 1) * ny + m2];
    s += (wx1 * wy1) * f[(m1 + 1) * ny + m2 + 1];
    return s;
}

static void clampxy(const i2g_params *P, double *x, double *y)
{
    /* markmart.c:1389-1390 */
    if (*x < 0) *x = 0; else if (*x > P->xsize) *x = P->xsize;
    if (*y < 0) *y = 0; else if (*y > P->ysize) *y = P->ysize;
}

/* allinterv(), markmart.c:1378-1453 (intermod = 0): vx, vy at (x, y). */
void ora_allinterv(const i2g_params *P, const ora_grid *G, double x, double y, double *vxo, double *vyo)
{
    const int64_t nx = G->xnumx, ny = G->ynumy;
    const double *gx = G->gx, *gy = G->gy;
    double wx0, wx1, wy0, wy1;
    clampxy(P, &x, &y);
    int64_t m10 = ora_m1serch(gx, nx, x), m20 = ora_m1serch(gy, ny, y);
    /* vx: basic columns m10, m10+1; rows at y midpoints (markmart.c:1403-1409) */
    int64_t m2 = m20;
    if (y < (gy[m20] + gy[m20 + 1]) / 2.0) m2 -= 1;
    if (m2 < 0) m2 = 0;
    if (m2 > ny - 3) m2 = ny - 3;
    ora_fdweight1(gx[m10], gx[m10 + 1], x, &wx0, &wx1);
    ora_fdweight1((gy[m2] + gy[m2 + 1]) / 2.0, (gy[m2 + 1] + gy[m2 + 2]) / 2.0, y, &wy0, &wy1);
    *vxo = bil(G->vx, ny, m10, m2, wx0, wx1, wy0, wy1);
    /* vy: columns at x midpoints, basic rows m20, m20+1 (markmart.c:1431-1437) */
    int64_t m1 = m10;
    if (x < (gx[m10] + gx[m10 + 1]) / 2.0) m1 -= 1;
    if (m1 < 0) m1 = 0;
    if (m1 > nx - 3) m1 = nx - 3;
    ora_fdweight1((gx[m1] + gx[m1 + 1]) / 2.0, (gx[m1 + 1] + gx[m1 + 2]) / 2.0, x, &wx0, &wx1);
    ora_fdweight1(gy[m20], gy[m20 + 1], y, &wy0, &wy1);
    *vyo = bil(G->vy, ny, m1, m20, wx0, wx1, wy0, wy1);
}

/* allintere(), markmart.c:1458-1543 (intermod = 0).
 * e[0..7] = exy, sxy, exx, sxx, eyy, syy, pr, ga (eps[4],[5],[6],[7],[8],[9],[10],[49]). */
void ora_allintere(const i2g_params *P, const ora_grid *G, double x, double y, double *e, int64_t *cell)
{
    const int64_t nx = G->xnumx, ny = G->ynumy;
    const double *gx = G->gx, *gy = G->gy;
    double wx0, wx1, wy0, wy1;
    clampxy(P, &x, &y);
    int64_t m10 = ora_m1serch(gx, nx, x), m20 = ora_m1serch(gy, ny, y);
    if (cell) { cell[0] = m10; cell[1] = m20; }
    /* exy, sxy on interior basic nodes (markmart.c:1484-1504) */
    int64_t a = m10, b = m20;
    if (a < 1) a = 1;
    if (a > nx - 3) a = nx - 3;
    if (b < 1) b = 1;
    if (b > ny - 3) b = ny - 3;
    ora_fdweight1(gx[a], gx[a + 1], x, &wx0, &wx1);
    ora_fdweight1(gy[b], gy[b + 1], y, &wy0, &wy1);
    e[0] = G->exy ? bil(G->exy, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
    e[1] = G->sxy ? bil(G->sxy, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
    /* cell-centre fields (markmart.c:1514-1540) */
    a = m10;
    if (x > (gx[m10] + gx[m10 + 1]) / 2.0) a += 1;
    if (a < 1) a = 1;
    if (a > nx - 2) a = nx - 2;
    b = m20;
    if (y > (gy[m20] + gy[m20 + 1]) / 2.0) b += 1;
    if (b < 1) b = 1;
    if (b > ny - 2) b = ny - 2;
    ora_fdweight1((gx[a] + gx[a - 1]) / 2.0, (gx[a + 1] + gx[a]) / 2.0, x, &wx0, &wx1);
    ora_fdweight1((gy[b] + gy[b - 1]) / 2.0, (gy[b + 1] + gy[b]) / 2.0, y, &wy0, &wy1);
    e[2] = G->exx ? bil(G->exx, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
    e[3] = G->sxx ? bil(G->sxx, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
    e[4] = G->eyy ? bil(G->eyy, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
    e[5] = G->syy ? bil(G->syy, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
    e[6] = G->pr ? bil(G->pr, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
    e[7] = G->ga ? bil(G->ga, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
}

int64_t ora_cell_key(const i2g_params *P, const ora_grid *G, double x, double y)
{
    clampxy(P, &x, &y);
    int64_t m10 = ora_m1serch(G->gx, G->xnumx, x), m20 = ora_m1serch(G->gy, G->ynumy, y);
    return m10 * (G->ynumy - 1) + m20;
}

/* viscalc(), markmart.c:1855-2062. */
double ora_viscalc(const i2g_params *P, const i2g_types *T, double mtk, double mpb, double hi,
                   double eii, double sii, double rii, double timesum, int mm2)
{
    double rt = 8.314 * mtk, e1, k1, sduct, sbrit, nueff, abrit, bbrit, nubrit, nunewt, nupowl;
    double lamb, A, sig0, nupeierls, siginnew, epsin, sigin;
    if (mm2 > 20) return T->markn0[mm2];
    epsin = eii;
    sigin = sii;
    lamb = T->markll[mm2];
    abrit = T->marka0[mm2];
    bbrit = T->markb0[mm2];
    sbrit = abrit + bbrit * mpb * 1e+5 * lamb;
    if (T->marks0[mm2] <= 0 && sbrit > T->marks1[mm2]) sbrit = T->marks1[mm2];
    if (sbrit > 0 && hi > 0 &&
        ((timesum - (hi * 1.000e+6 * 365.250 * 24.000 * 3600.000)) <
         (P->relax_time * 1.000e+6 * 365.250 * 24.000 * 3600.000)))
        sbrit = 1.000e+6;
    nubrit = 0;
    if (epsin > 0 && (bbrit > 0 || abrit * lamb > 0)) {
        if (sbrit > 0) nubrit = 1.0 / (0.5 * sbrit / epsin / rii);
        else nubrit = 1.0 / T->markn0[mm2];
    }
    nupeierls = 0;
    if (T->marks0[mm2] > 0 && sigin > 1e+7 && epsin > 0) {
        A = T->marks0[mm2];
        sig0 = T->marks1[mm2];
        siginnew = sig0 * 0.95;
        for (int n2 = 0; n2 < 5; n2++) {
            siginnew = pow(-rt / (T->markdh[mm2] + T->markdv[mm2] * mpb) * log(epsin / A / siginnew / siginnew), 0.5);
            if (siginnew > 1.0) siginnew = -siginnew;
            siginnew = (1.0 - siginnew) * sig0;
        }
        if (siginnew > sig0) siginnew = sig0;
        nupeierls = 1.0 / (0.5 * siginnew / epsin);
    }
    nunewt = 0;
    nupowl = 0;
    const double nu0 = T->marknu[mm2], dh = T->markdh[mm2], dv = T->markdv[mm2];
    const double ss = T->markss[mm2], mm = T->markmm[mm2];
    if (nu0) {
        if (dh == 0 && dv == 0 && (ss == 0 || mm == 1.0)) nunewt = 1.0 / nu0;
        if ((dh != 0 || dv != 0) && (ss == 0 || mm == 1.0)) {
            e1 = (dh + dv * mpb) / rt;
            if (e1 > 150.0) e1 = 150.0;
            if (dh < 0 && dv > 0) {
                e1 = dh * (mtk - dv);
                if (e1 < -150.0) e1 = -150.0;
            }
            if (dh < 0 && dv < 0) {
                e1 = (-dh) * (1.0 - (mtk - (-dv)) / (-dv)) / 8.314 / (-dv);
                if (e1 > 150.0) e1 = 150.0;
            }
            nunewt = 1.0 / (nu0 * exp(e1));
        }
        if ((dh == 0 && dv == 0) && ss != 0 && mm != 1.0) {
            k1 = nu0 / pow(ss, mm - 1.0);
            nunewt = 1.0 / (0.5 * k1);
            sduct = pow(nu0 * epsin, 1.0 / mm);
            if (epsin > 0) nupowl = 1.0 / (0.5 * sduct / epsin);
        }
        if ((dh != 0 || dv != 0) && ss != 0 && mm != 1.0) {
            e1 = (dh + dv * mpb) / rt;
            if (e1 > 150.0) e1 = 150.0;
            e1 = exp(e1);
            k1 = nu0 / pow(ss, mm - 1.0);
            nunewt = 1.0 / (0.5 * k1 * e1);
            sduct = pow(nu0 * e1 * epsin, 1.0 / mm);
            if (epsin > 0) nupowl = 1.0 / (0.5 * sduct / epsin);
        }
    }
    nueff = nunewt + nupowl;
    if (nubrit > nueff) nueff = nubrit;
    if (nupeierls > nueff) nueff = nupeierls;
    if (nueff <= 0) nueff = 1.0 / T->markn1[mm2];
    nueff = 1.0 / nueff;
    if (nueff < T->markn0[mm2]) nueff = T->markn0[mm2];
    if (nueff > T->markn1[mm2]) nueff = T->markn1[mm2];
    if (nueff < P->nubeg) nueff = P->nubeg;
    if (nueff > P->nuend) nueff = P->nuend;
    return nueff;
}

/* Radiogenic heating per kg by rock type at time timesum, markmart.c:749-837
 * (the marker then contributes coefficient * density). */
double ora_radiogenic(int mm2, double timesum, double al2627_init, double fe6056_init)
{
    double timesumA = timesum / (365.250 * 24.000 * 3600.000);
    if (mm2 == 5 || mm2 == 6 || mm2 == 25 || mm2 == 26) {
        double init_al = 1.89716e+23 * al2627_init * 4.999e-13 / (3.264e+13);
        double init_k = 0.40689 * 1.430e-11, init_u = 2.990e-12, init_uu = 1.600e-12, init_th = 1.000e-12;
        double a = init_al * exp(-timesumA * 9.6673e-7);
        double k = init_k * exp(-timesumA * 4.9867e-10);
        double u = init_u * exp(-timesumA * 9.8458e-10);
        double uu = init_uu * exp(-timesumA * 1.5541e-10);
        double th = init_th * exp(-timesumA * 4.9511e-11);
        return a + k + u + uu + th;
    }
    if (mm2 == 7 || mm2 == 8 || mm2 == 9 || mm2 == 10 || mm2 == 17 || mm2 == 18 || mm2 == 19) {
        double init_fe = 1.971e+24 * fe6056_init * 4.3451e-13 / (1.183e+14);
        double init_ka = 0.090625 * 1.430e-11;
        double fe = init_fe * exp(-timesumA * 2.6660e-7);
        double ka = init_ka * exp(-timesumA * 4.9867e-10);
        return fe + ka;
    }
    if (mm2 == 15) {
        double init_al = 1.89716e+23 * al2627_init * 4.999e-13 / (3.264e+13);
        double init_u = 2.990e-12, init_uu = 1.600e-12, init_th = 1.000e-12;
        double init_fe = 1.971e+24 * fe6056_init * 4.3451e-13 / (1.183e+14);
        double init_k = 1.430e-11;
        double a = init_al * exp(-timesumA * 9.6673e-7);
        double u = init_u * exp(-timesumA * 9.8458e-10);
        double uu = init_uu * exp(-timesumA * 1.5541e-10);
        double th = init_th * exp(-timesumA * 4.9511e-11);
        double fe = init_fe * exp(-timesumA * 2.6660e-7);
        double k = init_k * exp(-timesumA * 4.9867e-10);
        return a + fe + k + u + uu + th;
    }
    return 0.0;
}

/* movemark(), markmart.c:3-188, for mobile markers (type < 100). */
int ora_movemark(const i2g_params *P, const i2g_types *Ty, const ora_grid *G, int64_t n, double *x,
                 double *y, double *T, double *eta, double *p, const int8_t *type, const double *hi,
                 double timestep, double timesum, uint32_t flags)
{
    double e[8];
    for (int64_t i = 0; i < n; i++) {
        int mt = type[i];
        if (mt >= 100 || mt < 0) return I2G_EUNSUPPORTED;
        int mm2 = mt;
        if (!(((x[i] >= 0 && y[i] >= 0 && x[i] <= P->xsize && y[i] <= P->ysize) || P->outgrid != 1) &&
              !Ty->markim[mm2]))
            continue;
        /* markmart.c:46-68 */
        ora_allintere(P, G, x[i], y[i], e, NULL);
        double eii = pow(0.5 * (e[2] * e[2] + e[4] * e[4]) + e[0] * e[0], 0.5);
        double sii = pow(0.5 * (e[3] * e[3] + e[5] * e[5]) + e[1] * e[1], 0.5);
        double rii = 1.0;
        if (eta[i] > 0) rii *= pow(0.5 * sii / eii / eta[i], 0.87);
        double mpb = e[6] * 1e-5, mtk = T[i];
        p[i] = e[6];
        if ((flags & I2G_MOVE_UPDATE_VISC) && mt < 50 && mtk > 0)
            eta[i] = ora_viscalc(P, Ty, mtk, mpb, hi ? hi[i] : 0.0, eii, sii, rii, timesum,
                                 mt < 20 ? mm2 : mm2 - 20);
        /* markmart.c:73-97 */
        double vx0, vy0;
        if (P->markmod == 1) {
            ora_allinterv(P, G, x[i], y[i], &vx0, &vy0);
        } else {
            double vx1, vy1, vx2, vy2, vx3, vy3, vx4, vy4;
            ora_allinterv(P, G, x[i], y[i], &vx1, &vy1);
            ora_allinterv(P, G, x[i] + vx1 * timestep / 2.0, y[i] + vy1 * timestep / 2.0, &vx2, &vy2);
            ora_allinterv(P, G, x[i] + vx2 * timestep / 2.0, y[i] + vy2 * timestep / 2.0, &vx3, &vy3);
            ora_allinterv(P, G, x[i] + vx3 * timestep, y[i] + vy3 * timestep, &vx4, &vy4);
            vx0 = (vx1 + 2.0 * vx2 + 2.0 * vx3 + vx4) / 6.0;
            vy0 = (vy1 + 2.0 * vy2 + 2.0 * vy3 + vy4) / 6.0;
        }
        /* markmart.c:100-105 */
        if (P->outgrid == 2) {
            if (x[i] < 0 || x[i] > P->xsize) vy0 = 0;
            if (y[i] < 0 || y[i] > P->ysize) vx0 = 0;
        }
        /* markmart.c:114-115 */
        x[i] += timestep * vx0;
        y[i] += timestep * vy0;
        /* markmart.c:149-152 */
        if (x[i] < 0 || y[i] < 0 || x[i] > P->xsize || y[i] > P->ysize) T[i] = 0;
    }
    return I2G_OK;
}

/* dencalc(), markmart.c:1024-1046 */
static double ora_dencalc(const i2g_params *P, const i2g_types *Ty, double mtk, double mpb, double por,
                          int mm2, double *beta)
{
    *beta = 0;
    if (P->densimod == 0) return Ty->markro[mm2];
    double ival = Ty->markro[mm2] * (1.0 - Ty->markbb[mm2] * (mtk - 298.15)) *
                  (1.0 + Ty->markaa[mm2] * (mpb - 1.0) * 1e-3) * (1.000 - por);
    *beta = Ty->markbb[mm2] / (1.0 - Ty->markbb[mm2] * (mtk - 298.15));
    return ival;
}

/* ---- densimod 2 ---------------------------------------------------------- */
/* meltpart1(), markmart.c:2336-2652: solidus/liquidus of the marker type at P
 * (bar), then the melt fractions and latent heats it leaves in eps[21], eps[22]
 * (silicate), eps[50], eps[51] (iron), eps[52], eps[53] (water ice): melt[0..5]. */
static void ora_meltpart1(const i2g_td_table *D, double mtk, double mpb, int mm2, double *melt)
{
    double xmelt, xmelt_fe, xmelt_ice, hlatent = 0, hlatent_fe = 0, hlatent_ice = 0;
    double ykm = mpb * 3e-3, ts = 0, ts_fe = 0, ts_ice = 0, tl = 0, tl_fe = 0, tl_ice = 0, t_shift = 10.000;
    int peridotite = (mm2 == 5 || mm2 == 25 || mm2 == 26 || mm2 == 6);
    if (mm2 == 11 || mm2 == 12 || mm2 == 31 || mm2 == 32) {
        /* markmart.c:2353-2370 */
        if (ykm < 48.0) ts = 972.6 - 2111.0 / (ykm + 10.63) + 70033.0 / (ykm + 10.63) / (ykm + 10.63);
        else ts = 935.4 + 0.1162 * ykm + 0.006937 * ykm * ykm;
        tl = 1423.15 + 3.5 * ykm;
        hlatent = 380000.0;
    }
    if (peridotite) {
        /* markmart.c:2372-2412 (types 5, 25, 26) and 2414-2432 (type 6): the same curves */
        if (D->si_melting == 0) {
            if (mpb < 10e+4) ts = 273.15 + 1120.661 + 132.899e-4 * mpb - 5.104e-8 * mpb * mpb;
            else ts = 273.15 + 1939.251 + 30.819e-4 * (mpb - 10e+4);
        } else if (D->si_melting == 1) {
            if (mpb < 21.50e+4)
                ts = 273.15 + 1143.04342 + 58.2946423e-4 * mpb + 52.3439318e-8 * mpb * mpb -
                     16.3201032e-12 * mpb * mpb * mpb + 2.29886314e-16 * pow(mpb, 4.000) -
                     0.180865486e-20 * pow(mpb, 5.000) + 0.00815679773e-24 * pow(mpb, 6.000) -
                     0.000197104325e-28 * pow(mpb, 7.000) + 1.97908526e-38 * pow(mpb, 8.000);
            else ts = 273.15 + 2157.500 + 11.7297e-4 * (mpb - 21.50e+4);
        }
        tl = 1973.000 + 28.570e-4 * mpb;
        hlatent = 400000.0;
    }
    if (mm2 == 6) {
        /* markmart.c:2434-2462 */
        if (D->ice_melting == 1) {
            if (mpb >= 0.000e6 && mpb < 2085.66) {
                ts_ice = 273.0159 - 0.0132 * mpb - 0.1577 * log(mpb) + 0.1516 * pow(mpb, 0.500);
                tl_ice = t_shift + 273.0159 - 0.0132 * mpb - 0.1577 * log(mpb) + 0.1516 * pow(mpb, 0.500);
            }
            if (mpb >= 2085.66 && mpb < 3501.0) {
                ts_ice = 10.277 + 0.0265 * mpb + 50.1624 * log(mpb) + (0.5868 / mpb) - 4.3288 * pow(mpb, 0.500);
                tl_ice = t_shift + 10.277 + 0.0265 * mpb + 50.1624 * log(mpb) + (0.5868 / mpb) -
                         4.3288 * pow(mpb, 0.500);
            }
            if (mpb >= 3501.0 && mpb < 6324.0) {
                ts_ice = 5.0321 - 0.0004 * mpb + 30.9482 * log(mpb) + (1.0018 / mpb);
                tl_ice = t_shift + 5.0321 - 0.0004 * mpb + 30.9482 * log(mpb) + (1.0018 / mpb);
            }
            if (mpb >= 6324.000 && mpb < 22160.0) {
                ts_ice = 4.2804 - 0.0013 * mpb + 21.8756 * log(mpb) + (1.0018 / mpb) + 1.0785 * pow(mpb, 0.500);
                tl_ice = t_shift + 4.2804 - 0.0013 * mpb + 21.8756 * log(mpb) + (1.0018 / mpb) +
                         1.0785 * pow(mpb, 0.500);
            }
            if (mpb >= 22160.0 && mpb < 4.000e5) {
                ts_ice = -1355.42 + 0.0018 * mpb + 167.0609 * log(mpb) + (-0.6633 / mpb);
                tl_ice = t_shift - 1355.42 + 0.0018 * mpb + 167.0609 * log(mpb) + (-0.6633 / mpb);
            }
            if (mpb >= 4.000e5 && mpb < 9.000e5) {
                ts_ice = 0.2524 + 0.0019 * mpb + 0.2795 * log(mpb) + (0.500 / mpb) + 1.1675 * pow(mpb, 0.500);
                tl_ice = t_shift + 0.2524 + 0.0019 * mpb + 0.2795 * log(mpb) + (0.500 / mpb) +
                         1.1675 * pow(mpb, 0.500);
            }
        }
        hlatent_ice = (284000.0 + 233000.0) * 0.3;
    }
    if (mm2 == 7 || mm2 == 8 || mm2 == 9 || mm2 == 10 || mm2 == 17 || mm2 == 18 || mm2 == 19) {
        /* markmart.c:2464-2580; tdbasecalc() never passes these types */
        if (D->fe_melting == 0) {
            double a = 0, b = 0;
            if (mpb >= 0.000e6 && mpb < 0.100e6) { a = 1761.000; b = 3.100e-3; }
            if (mpb >= 0.100e6 && mpb < 0.200e6) { a = 1863.000; b = 2.080e-3; }
            if (mpb >= 0.200e6 && mpb < 0.600e6) { a = 2071.800; b = 1.035e-3; }
            if (mpb >= 0.600e6 && mpb < 1.000e6) { a = 2382.800; b = 5.170e-4; }
            if (mpb >= 1.000e6) { a = 2900.000; b = (1.000 / 1.000e3); }
            if (a != 0) { ts_fe = a + b * mpb; tl_fe = t_shift + a + b * mpb; }
        } else if (D->fe_melting == 1) {
            /* the reference assigns tl_fe twice here; ts_fe stays 0 */
            if (mpb <= 0.4180e6)
                tl_fe = t_shift + 1260.1000 + 3.3171e-4 * mpb - 3.395e-9 * mpb * mpb + 2.660e-14 * mpb * mpb * mpb -
                        3.7688e-20 * pow(mpb, 4.000);
            else tl_fe = t_shift + 1597.7000 + 4.2635e-4 * (mpb - 0.4180e6);
        }
        hlatent_fe = 240000.0;
    }
    /* markmart.c:2598-2649 */
    melt[0] = melt[1] = 0;
    if (tl) {
        if (ts >= tl - 100.0) ts = tl - 100.0;
        xmelt = (mtk - ts) / (tl - ts);
        if (xmelt < 0.0000) xmelt = 0.0000;
        if (xmelt > 1.0000) xmelt = 1.0000;
        melt[0] = xmelt;
        melt[1] = hlatent * xmelt;
    }
    melt[2] = melt[3] = 0;
    if (tl_fe) {
        xmelt_fe = (mtk - ts_fe) / (tl_fe - ts_fe);
        if (xmelt_fe < 0.000) xmelt_fe = 0.0000;
        if (xmelt_fe > 1.000) xmelt_fe = 1.0000;
        melt[2] = xmelt_fe;
        melt[3] = hlatent_fe * xmelt_fe;
    }
    melt[4] = melt[5] = 0;
    if (tl_ice) {
        xmelt_ice = (mtk - ts_ice) / (tl_ice - ts_ice);
        if (xmelt_ice < 0.000) xmelt_ice = 0.0000;
        if (xmelt_ice > 1.000) xmelt_ice = 1.0000;
        melt[4] = xmelt_ice;
        melt[5] = hlatent_ice * xmelt_ice;
    }
}

static double td_at(const i2g_td_table *D, int n1, int n2, int mm3, int k)
{
    return D->td[(((size_t)n1 * (size_t)D->pbdim + (size_t)n2) * 2 + (size_t)mm3) * 5 + (size_t)k];
}

/* tdbasecalc(), markmart.c:2068-2276, for table type mm2: the table's density,
 * heat capacity and expansion term, the lattice + radiative conductivity, the
 * molten-rock mixture and the latent-heat terms.  *mnu is eps[48] in and out;
 * melt[] is the eps[] state, updated by every meltpart1 call.  Returns the
 * marker's new type (markmart.c:2180-2182). */
static int ora_tdbasecalc(const i2g_td_table *D, const i2g_types *Ty, double nubeg, double nuend, double mtk,
                          double mpb, int mm2, double *melt, double *mro_o, double *mcp_o, double *mbb_o,
                          double *mkt_o, double *mnu)
{
    double mkt1, krad, e, n, mro, mcp, mbb, mkt, ival, dmpb, lo;
    int n1, n2, mm3, nt;
    /* markmart.c:2086-2112 (only the 1 mm radiative term is used) */
    if (mpb < 235000.0) {
        mkt1 = (1.878 + 770.9 / (mtk <= 1200.0 ? mtk : 1200.0)) * (1.0 + 4.26e-6 * mpb);
        krad = pow(mtk / 1774.0, 3.0);
    } else {
        mkt1 = (1.291 + 1157.0 / (mtk <= 2100.0 ? mtk : 2100.0)) * (1.0 + 2.50e-6 * mpb);
        krad = pow(mtk / 2117.0, 3.0);
    }
    /* markmart.c:2118-2139 */
    mm3 = (mm2 == 11 || mm2 == 12 || mm2 == 31 || mm2 == 32) ? 1 : 0;
    e = (mtk - D->tkmin) / D->tkstp;
    if (e < 0) e = 0;
    if (e > (double)(D->tknum - 1)) e = (double)(D->tknum - 1);
    n = (mpb - D->pbmin) / D->pbstp;
    if (n < 0) n = 0;
    if (n > (double)(D->pbnum - 1)) n = (double)(D->pbnum - 1);
    n1 = (int)(e);
    if (n1 > D->tknum - 2) n1 = D->tknum - 2;
    n2 = (int)(n);
    if (n2 > D->pbnum - 2) n2 = D->pbnum - 2;
    e = (e - (double)(n1));
    n = (n - (double)(n2));
    /* markmart.c:2144-2170 */
    double R0 = td_at(D, n1, n2, mm3, 0) * 1000.0, R1 = td_at(D, n1, n2 + 1, mm3, 0) * 1000.0;
    double R2 = td_at(D, n1 + 1, n2, mm3, 0) * 1000.0, R3 = td_at(D, n1 + 1, n2 + 1, mm3, 0) * 1000.0;
    double H0 = td_at(D, n1, n2, mm3, 1) * 1000.0 * 4.1837, H1 = td_at(D, n1, n2 + 1, mm3, 1) * 1000.0 * 4.1837;
    double H2 = td_at(D, n1 + 1, n2, mm3, 1) * 1000.0 * 4.1837;
    double H3 = td_at(D, n1 + 1, n2 + 1, mm3, 1) * 1000.0 * 4.1837;
    mro = ((R0 * (1.0 - n) + R1 * n) * (1.0 - e) + (R2 * (1.0 - n) + R3 * n) * e);
    mcp = ((H2 - H0) * (1.0 - n) + (H3 - H1) * n) / D->tkstp;
    if (mcp < 1e+2) mcp = 1e+2;
    else if (mcp > 5e+4) mcp = 5e+4;
    mbb = (2.0 / (R1 + R0) - (H1 - H0) / D->pbstp / 1e+5) * (1.0 - e) +
          (2.0 / (R3 + R2) - (H3 - H2) / D->pbstp / 1e+5) * e;
    mbb *= mro / mtk;
    if (mbb < -1e-2) mbb = -1e-2;
    else if (mbb > 1e-2) mbb = 1e-2;
    mkt = mkt1 + krad;
    /* markmart.c:2178-2235: partially molten rock */
    ora_meltpart1(D, mtk, mpb, mm2, melt);
    nt = mm2;
    if (melt[0] > 0 && mm2 < 20) nt = mm2 + 20;
    if (melt[0] <= 0 && mm2 > 20) nt = mm2 - 20;
    if (nt > 20) {
        double xmelt = melt[0];
        mro = mro * (1.0 - xmelt) +
              xmelt * Ty->markro[nt] * (1.0 - Ty->markbb[nt] * (mtk - 298.15)) * (1.0 + Ty->markaa[nt] * (mpb - 1.0) * 1e-3);
        if (xmelt > 0.1) {
            double nueff = Ty->marknu[nt] * exp((2.500 + pow(((1.000 - xmelt) / xmelt), 0.480)) * (1.000 - xmelt));
            if (nueff < Ty->markn0[nt]) nueff = Ty->markn0[nt];
            if (nueff > Ty->markn1[nt]) nueff = Ty->markn1[nt];
            if (nueff < nubeg) nueff = nubeg;
            if (nueff > nuend) nueff = nuend;
            *mnu = nueff;
        }
        mkt = ((Ty->markkt[nt] + Ty->markkf[nt] / (mtk + 77.0)) * exp(Ty->markkp[nt] * mpb)) * xmelt +
              ((Ty->markkt[nt - 20] + Ty->markkf[nt - 20] / (mtk + 77.0)) * exp(Ty->markkp[nt - 20] * mpb)) *
                  (1.0 - xmelt);
        if (xmelt > 0 && xmelt < 1.0) {
            dmpb = mpb * 0.001;
            ora_meltpart1(D, mtk, mpb - dmpb, nt, melt);
            lo = melt[1];
            ora_meltpart1(D, mtk, mpb + dmpb, nt, melt);
            ival = lo - melt[1];
            ival *= mro / (mtk * 2.0 * dmpb * 1e+5);
            mbb += ival;
            ora_meltpart1(D, mtk + 1.0, mpb, nt, melt);
            lo = melt[1];
            ora_meltpart1(D, mtk - 1.0, mpb, nt, melt);
            ival = lo - melt[1];
            ival /= 2.0 * 1.0;
            mcp += ival;
        }
    }
    /* markmart.c:2237-2268: water ice of type 6 */
    ora_meltpart1(D, mtk, mpb, nt, melt);
    if (nt == 6) {
        double xmelt_ice = melt[4];
        if (xmelt_ice > 0 && xmelt_ice < 1.0) {
            dmpb = mpb * 0.001;
            ora_meltpart1(D, mtk, mpb - dmpb, nt, melt);
            lo = melt[5];
            ora_meltpart1(D, mtk, mpb + dmpb, nt, melt);
            ival = lo - melt[5];
            ival *= mro / (mtk * 2.0 * dmpb * 1e+5);
            mbb += ival;
            ora_meltpart1(D, mtk + 1.0, mpb, nt, melt);
            lo = melt[5];
            ora_meltpart1(D, mtk - 1.0, mpb, nt, melt);
            ival = lo - melt[5];
            ival /= 2.0 * 1.0;
            mcp += ival;
        }
    }
    *mro_o = mro;
    *mcp_o = mcp;
    *mbb_o = mbb;
    *mkt_o = mkt;
    return nt;
}

/* Cold pressing and hot sintering of porous solid silicate, markmart.c:362-466
 * (Henke et al. 2012; Schwenn & Goetze 1978).  por is markpor[] of a type 5/6
 * marker with 0 < por <= 0.85; returns its new value.  f32: markpor[] in the
 * reference's single-precision storage.  The grain-size search restarts from a
 * larger guess while its Newton iteration has not settled (markmart.c:426-432,
 * an unbounded goto there); after ORA_SINTER_TRIES restarts *stuck is set and
 * the porosity is returned unchanged. */
#define ORA_SINTER_TRIES 64
static double ora_sinter(double mpb, double mtk, double por, double por_init, double timestep, int f32, int *stuck)
{
    const double p_ref = 0.130, grain_orig = 1.000e-6, pivalue = 3.141592654;
    const double E_act = 85000.000, fact_a = 4.000e-5, r_gas = 1.9872;
#define ST(v) (f32 ? (double)(float)(v) : (v))
#define MINV(a, b) ((a) <= (b) ? (a) : (b))
    if (mtk < 700.000) {
        por = ST(MINV(por, (0.420 + 0.460 * pow((pow((mpb / p_ref), 1.720) + 1.000), (-1.000)))));
        por = ST(MINV(por, 0.850));
    }
    if (mtk >= 700.000) {
        double por_orig = MINV(por_init, (0.420 + 0.460 * pow((pow((mpb / p_ref), 1.720) + 1.000), (-1.000))));
        por_orig = MINV(por_orig, 0.850);
        double guess = grain_orig, old = 0.0, grain_corr = 0.0, por_change = 0.0;
        int n_count = 1;
        for (;;) {
            for (int it = 1; it < 100; it++) {
                old = guess;
                double funct = pow(guess, 3.000) + pow(grain_orig, 3.000) -
                               3.000 * pow(guess, 2.000) * grain_orig *
                                   pow(((1.000 - por_orig) / (1.000 - por)), (1.000 / 3.000)) +
                               pow(grain_orig, 3.000) * (1.000 - por_orig) / (1.000 - por);
                double drv = 3.000 * pow(guess, 2.000) -
                             6.000 * guess * grain_orig * pow(((1.000 - por_orig) / (1.000 - por)), (1.000 / 3.000));
                guess = old - (funct / drv);
            }
            double err = ABSV(guess - old);
            if ((err > 5.000e-2) || (guess <= grain_orig)) {
                if (++n_count > ORA_SINTER_TRIES) {
                    *stuck = 1;
                    return por;
                }
                guess = 1.250 * (double)(n_count)*grain_orig;
                continue;
            }
            break;
        }
        if (guess > grain_orig) grain_corr = guess;
        double cont_r = sqrt(pow(grain_corr, 2.000) -
                             pow(grain_orig, 2.000) * pow(((1.000 - por_orig) / (1.000 - por)), (2.000 / 3.000)));
        double c_fact = 2.000 * sqrt(3.000) * (pow(grain_corr, 2.000) - pow(cont_r, 2.000));
        double grain_stress = c_fact * mpb / (pivalue * pow(cont_r, 2.000));
        if (por > 0.100)
            por_change = fact_a * (1.000 - por) * pow(grain_stress, 1.500) / pow((100.000 * grain_corr), 3.000) *
                         exp(-E_act / (r_gas * mtk)) * timestep;
        if (por <= 0.100)
            por_change = 10.000 * por * fact_a * (1.000 - por) * pow(grain_stress, 1.500) /
                         pow((100.000 * grain_corr), 3.000) * exp(-E_act / (r_gas * mtk)) * timestep;
        if (por_change > 0.000) por = ST(por - por_change);
    }
#undef ST
#undef MINV
    return por;
}

typedef struct contrib {
    int64_t m10, m20;
    double wx0, wx1, wy0, wy1;
    double mro, mbb, mcp, mkt, mht, mtk, lnu;
    int valid, immobile;
} contrib;

/* one marker of the ronurecalc loop, markmart.c:277-845 */
static void marker_props(const i2g_params *P, const i2g_types *Ty, const ora_grid *G, int64_t i,
                         const double *x, const double *y, double *T, const double *eta,
                         int8_t *type, const double *hi, double *tmax, double *por, double timesum, double T0,
                         const double *radcoef, const i2g_td_table *td, double *melt, ora_sinter_args *sinter,
                         contrib *c)
{
    double e[8];
    int64_t cell[2];
    int mt = type[i], mm2 = mt;
    c->valid = 0;
    if (!(x[i] > 0 && y[i] > 0 && x[i] < P->xsize && y[i] < P->ysize && T[i] > 0 && mt < 50)) return;
    c->valid = 1;
    ora_allintere(P, G, x[i], y[i], e, cell);
    double mpb = e[6] * 1.0000e-5, mtk = T[i], mga = e[7];
    /* markmart.c:287-289: the melt fractions the last meltpart1 call left */
    double xmelt = melt[0], xmelt_fe = melt[2];
    /* markmart.c:296-309: sticky air held at the ambient temperature */
    if (mm2 < 2) { T[i] = P->tmp_ambient; mtk = T[i]; }
    /* markmart.c:320-340 */
    double mnu = eta[i];
    if (mnu <= 0) {
        double eii = pow(0.5 * (e[2] * e[2] + e[4] * e[4]) + e[0] * e[0], 0.5);
        double sii = pow(0.5 * (e[3] * e[3] + e[5] * e[5]) + e[1] * e[1], 0.5);
        mnu = ora_viscalc(P, Ty, mtk, mpb, hi ? hi[i] : 0.0, eii, sii, 1.0, timesum, mt < 20 ? mm2 : mm2 - 20);
    }
    double celdx = x[i] - P->xsize / 2.0, celdy = y[i] - P->ysize / 2.0;
    celdy = pow(celdx * celdx + celdy * celdy, 0.5);
    if (celdy > P->xsize / 2.0 * 0.95) mnu = 1.000e+22;
    /* markmart.c:347-360 */
    double mpor = por ? por[i] : 0.0;
    if (mm2 == 0 || mm2 >= 7) mpor = 0.0;
    if (tmax && mt != 0 && tmax[i] < T[i]) tmax[i] = T[i];
    /* markmart.c:362-466 */
    if ((mm2 == 5 || mm2 == 6) && (mpor > 0.000 && mpor <= 0.850))
        mpor = ora_sinter(mpb, mtk, mpor, P->por_init, sinter->timestep, sinter->f32, &sinter->stuck);
    if (mpor < 0.000) mpor = 0.000;
    if (mpor > 1.000) mpor = 1.000;
    if (por) por[i] = mpor;
    /* markmart.c:475-478 */
    double mbb;
    double mro = ora_dencalc(P, Ty, mtk, mpb, mpor, mm2, &mbb);
    double mcp = Ty->markcp[mm2];
    double mkt = (Ty->markkt[mm2] + Ty->markkf[mm2] / (mtk + 77.0)) * exp(Ty->markkp[mm2] * mpb);
    /* markmart.c:481-493: the table types of densimod 2 */
    if (P->densimod == 2 && (mm2 == 5 || mm2 == 6 || mm2 == 11 || mm2 == 12 || mm2 == 25 || mm2 == 26 ||
                             mm2 == 31 || mm2 == 32))
        type[i] = (int8_t)ora_tdbasecalc(td, Ty, P->nubeg, P->nuend, mtk, mpb, mm2, melt, &mro, &mcp, &mbb, &mkt,
                                         &mnu);
    /* markmart.c:509-610: conductivity of molten silicate and iron */
    if ((mm2 == 25 || mm2 == 26) && (timesum > P->core_form_time)) {
        double heat_flux, eta_fluid;
        if (xmelt >= 0.4000 && xmelt <= 0.6000) {
            eta_fluid = Ty->markn0[mm2] * exp((-172.690) * (xmelt - 0.400));
            heat_flux = 0.089 * pow(Ty->markkt[mm2], (2.000 / 3.000)) * pow(ABSV(T[i] - T0), (4.000 / 3.000)) *
                        pow((mro * mro * Ty->markbb[mm2] * mga * mcp / eta_fluid), (1.000 / 3.000));
            if (heat_flux <= 0.0001) mkt = Ty->markkt[mm2];
            else if (heat_flux > 0.0001)
                mkt = pow((heat_flux / 0.089), (3.000 / 2.000)) / (pow((T[i] - T0), 2.000) * mro) *
                      pow((Ty->markbb[mm2] * mga * mcp / mnu), (-1.000 / 2.000));
        }
        if (xmelt > 0.6000) {
            eta_fluid = 100.0000;
            heat_flux = 0.089 * pow(Ty->markkt[mm2], (2.000 / 3.000)) * pow(ABSV(T[i] - T0), (4.000 / 3.000)) *
                        pow((mro * mro * Ty->markbb[mm2] * mga * mcp / eta_fluid), (1.000 / 3.000));
            if (heat_flux <= 0.0001) mkt = Ty->markkt[mm2];
            else if (heat_flux > 0.0001)
                mkt = pow((heat_flux / 0.089), (3.000 / 2.000)) / (pow((T[i] - T0), 2.000) * mro) *
                      pow((Ty->markbb[mm2] * mga * mcp / mnu), (-1.000 / 2.000));
        }
    }
    if ((mm2 == 7 || mm2 == 8 || mm2 == 9 || mm2 == 10 || mm2 == 17 || mm2 == 18 || mm2 == 19) &&
        (timesum > P->core_form_time)) {
        double heat_flux, eta_fluid_fe;
        if (xmelt_fe < 1.0000) {
            eta_fluid_fe = 1.0000e12;
            heat_flux = 0.089 * pow(Ty->markkt[mm2], (2.000 / 3.000)) * pow(ABSV(T[i] - T0), (4.000 / 3.000)) *
                        pow((mro * mro * Ty->markbb[mm2] * mga * mcp / eta_fluid_fe), (1.000 / 3.000));
            if (heat_flux <= 0.0001) mkt = Ty->markkt[mm2];
            else if (heat_flux > 0.0001)
                mkt = pow((heat_flux / 0.089), (3.0000 / 2.0000)) / (pow((T[i] - T0), 2.000) * mro) *
                      pow((Ty->markbb[mm2] * mga * mcp / mnu), (-1.000 / 2.000));
        }
        if (xmelt_fe == 1.0000) {
            eta_fluid_fe = 0.010;
            heat_flux = 0.089 * pow(Ty->markkt[mm2], (2.000 / 3.000)) * pow(ABSV(T[i] - T0), (4.000 / 3.000)) *
                        pow((mro * mro * Ty->markbb[mm2] * mga * mcp / eta_fluid_fe), (1.000 / 3.000));
            if (heat_flux <= 0.0001) mkt = Ty->markkt[mm2];
            else if (heat_flux > 0.0001)
                mkt = pow((heat_flux / 0.089), (3.000 / 2.000)) / (pow((T[i] - T0), 2.000) * mro) *
                      pow((Ty->markbb[mm2] * mga * mcp / mnu), (-1.000 / 2.000));
        }
    }
    /* markmart.c:614-638: porosity-dependent conductivity of solid silicates */
    if (mm2 == 5 || mm2 == 6) {
        if (mpor < 0.200) mkt = Ty->markkt[mm2] * exp(-mpor / 0.080);
        if (mpor >= 0.200 && mpor <= 0.400)
            mkt = pow((pow((Ty->markkt[mm2] * exp(-mpor / 0.080)), 4.000) +
                       pow((Ty->markkt[mm2] * exp(-1.200 - (mpor / 0.167))), 4.000)), 0.250);
        if (mpor > 0.400) mkt = Ty->markkt[mm2] * exp(-1.200 - (mpor / 0.167));
    }
    /* markmart.c:641-648 */
    if (mkt <= 0.0010) mkt = 0.0010;
    if (mkt >= P->k_cutoff) mkt = P->k_cutoff;
    /* markmart.c:651-744: magnetisation of solid silicates below the Curie
     * temperatures (magnetite 851.16 K, hematite 948.16 K) */
    if (sinter->mg_old) {
        int mag = 3;
        const int old = sinter->mg_old[i];
        if (P->dynamo == 0) {
            if (mm2 == 5 || mm2 == 6) {
                if (mtk <= 851.16 && old == 2) mag = 2;
                else if ((mtk > 851.16 && mtk <= 948.16) && old == 2) mag = 1;
                else if (mtk <= 851.16 && old == 1) mag = 1;
                else if ((mtk > 851.16 && mtk <= 948.16) && old == 1) mag = 1;
                else if (mtk > 948.16) { mag = 0; sinter->mag_time = -1.000; }
            } else if (mm2 < 5 || mm2 > 6) {
                mag = 3;
                sinter->mag_time = -1.000;
            }
        } else if (P->dynamo == 1) {
            if (mm2 == 5 || mm2 == 6) {
                if (mtk <= 851.16) {
                    mag = 2;
                    if (old <= 1 || old == 3) sinter->mag_time = timesum / (3600.000 * 24.000 * 365.250 * 1.000e+6);
                } else if (mtk > 851.16 && mtk <= 948.16) {
                    mag = 1;
                    if (old == 0 || old == 3) sinter->mag_time = timesum / (3600.000 * 24.000 * 365.250 * 1.000e+6);
                } else if (mtk > 948.16) {
                    mag = 0;
                    sinter->mag_time = -1.000;
                }
            } else if (mm2 < 5 || mm2 > 6) {
                mag = 3;
                sinter->mag_time = -1.000;
            }
        }
        sinter->mg_old[i] = (int8_t)mag;
        sinter->mg_time[i] = sinter->mag_time;
    }
    /* markmart.c:843-855: linear weights of the marker's cell at its position */
    int64_t m10 = cell[0], m20 = cell[1];
    c->m10 = m10;
    c->m20 = m20;
    ora_fdweight1(G->gx[m10], G->gx[m10 + 1], x[i], &c->wx0, &c->wx1);
    ora_fdweight1(G->gy[m20], G->gy[m20 + 1], y[i], &c->wy0, &c->wy1);
    c->mro = mro;
    c->mbb = mbb;
    c->mcp = mcp;
    c->mkt = mkt;
    c->mht = radcoef[mm2] * mro;
    c->mtk = mtk;
    c->lnu = P->viscmod == 1 ? log(mnu) : (P->viscmod == 2 ? 1.0 / mnu : mnu);
    c->immobile = Ty->markim[mm2] != 0;
}

typedef struct acc {
    double *ro0, *et0, *nu0, *nd0, *cp0, *kt0, *ht0, *tk0, *w0, *w1, *wnu, *wnd;
} acc;

/* the 2x2 scatter of one marker into node nn (corner i,j), markmart.c:876-910 */
static void add_corner(const contrib *c, int i, int j, int64_t m3, acc *A)
{
    double ddx = i ? c->wx1 : c->wx0, ddy = j ? c->wy1 : c->wy0;
    double swt = 1.0 * ddx * ddy;
    if (ddx > 0.5 && ddy > 0.5) {
        double swt2 = 1.0 * 4.0 * (ddx - 0.5) * (ddy - 0.5);
        A->nu0[m3] += c->lnu * swt2;
        A->wnu[m3] += swt2;
    }
    A->ro0[m3] += c->mro * swt;
    A->et0[m3] += c->mbb * swt;
    A->cp0[m3] += c->mcp * swt;
    A->kt0[m3] += c->mkt * swt;
    A->ht0[m3] += c->mht * swt;
    A->w0[m3] += swt;
    if (!c->immobile) {
        A->tk0[m3] += c->mtk * swt;
        A->w1[m3] += swt;
    }
}

/* the cell-centre (normal viscosity) part, markmart.c:859-872 */
static void add_centre(const contrib *c, int64_t ny, acc *A)
{
    double ddx = 1.0 - ABSV(c->wx0 - 0.5), ddy = 1.0 - ABSV(c->wy0 - 0.5);
    if (ddx > 0.5 && ddy > 0.5) {
        int64_t m3 = (c->m10 + 1) * ny + c->m20 + 1;
        double swt2 = 1.0 * 4.0 * (ddx - 0.5) * (ddy - 0.5);
        A->nd0[m3] += c->lnu * swt2;
        A->wnd[m3] += swt2;
    }
}

/* ronurecalc(), markmart.c:192-1009 (tkrecalc() at :1013 stays with the caller). */
int ora_ronurecalc(const i2g_params *P, const i2g_types *Ty, const ora_grid *G, int64_t n,
                   const double *x, const double *y, double *T, const double *eta, int8_t *type,
                   const double *hi, double *tmax, double *por, double timesum, uint32_t flags, int order,
                   const i2g_td_table *td, double *melt_state, ora_sinter_args *sinter, ora_nodes *out,
                   double *numin_numax)
{
    (void)flags;
    if (P->densimod == 2 && !td) return I2G_EINVAL;
    double melt_local[6] = {P->xmelt_si, 0.0, P->xmelt_fe, 0.0, P->xmelt_ice, 0.0};
    double *melt = melt_state ? melt_state : melt_local;
    ora_sinter_args sa = {sinter ? sinter->timestep : 0.0, sinter ? sinter->f32 : 0, 0,
                          sinter ? sinter->mg_old : NULL, sinter ? sinter->mg_time : NULL,
                          sinter ? sinter->mag_time : -1.0};
    const int64_t nx = G->xnumx, ny = G->ynumy, nn = nx * ny;
    int gridmod = P->gridmod > 0 ? P->gridmod : 1;
    double radcoef[I2G_MAXTYPES];
    for (int t = 0; t < I2G_MAXTYPES; t++) radcoef[t] = ora_radiogenic(t, timesum, P->al2627_init, P->fe6056_init);
    for (int64_t i = 0; i < n; i++)
        if (type[i] < 0 || type[i] >= 100) return I2G_EUNSUPPORTED;
    acc A;
    double *buf = (double *)calloc((size_t)(12 * nn), sizeof(double));
    contrib *cs = (contrib *)calloc((size_t)(n > 0 ? n : 1), sizeof(contrib));
    if (!buf || !cs) { free(buf); free(cs); return I2G_ENOMEM; }
    A.ro0 = buf; A.et0 = buf + nn; A.nu0 = buf + 2 * nn; A.nd0 = buf + 3 * nn; A.cp0 = buf + 4 * nn;
    A.kt0 = buf + 5 * nn; A.ht0 = buf + 6 * nn; A.tk0 = buf + 7 * nn; A.w0 = buf + 8 * nn;
    A.w1 = buf + 9 * nn; A.wnu = buf + 10 * nn; A.wnd = buf + 11 * nn;
    /* markk[0] as the molten-material branches read it (markmart.c:522): marker 0 is
     * processed first, so every marker sees it after its own sticky-air reset */
    double T0 = 0.0;
    if (n > 0) {
        T0 = T[0];
        if (x[0] > 0 && y[0] > 0 && x[0] < P->xsize && y[0] < P->ysize && T[0] > 0 && type[0] < 2)
            T0 = P->tmp_ambient;
    }
    for (int64_t i = 0; i < n; i += gridmod)
        marker_props(P, Ty, G, i, x, y, T, eta, type, hi, tmax, por, timesum, T0, radcoef, td, melt, &sa, &cs[i]);
    if (order == ORA_ORDER_REFERENCE) {
        for (int64_t i = 0; i < n; i += gridmod) {
            const contrib *c = &cs[i];
            if (!c->valid) continue;
            add_centre(c, ny, &A);
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) add_corner(c, a, b, (c->m10 + a) * ny + c->m20 + b, &A);
        }
    } else {
        /* The CUDA summation order: per cell, corner sums over its markers by
         * ascending index, each from 0; per node, 0 + its four cells' corner sums
         * in the order (m1-1,m2-1), (m1-1,m2), (m1,m2-1), (m1,m2). */
        int64_t nc = (nx - 1) * (ny - 1);
        double *part = (double *)calloc((size_t)(42 * nc), sizeof(double));
        acc C;
        if (!part) { free(buf); free(cs); return I2G_ENOMEM; }
        for (int64_t i = 0; i < n; i += gridmod) {
            const contrib *c = &cs[i];
            if (!c->valid) continue;
            int64_t cell = c->m10 * (ny - 1) + c->m20;
            double *q = part + 42 * cell;
            /* corner (a,b) of the cell is a 1-node "grid" with stride 0 */
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    double *r = q + 10 * (a * 2 + b);
                    C.ro0 = r + 0; C.et0 = r + 1; C.cp0 = r + 2; C.kt0 = r + 3; C.ht0 = r + 4;
                    C.w0 = r + 5; C.tk0 = r + 6; C.w1 = r + 7; C.nu0 = r + 8; C.wnu = r + 9;
                    add_corner(c, a, b, 0, &C);
                }
            {
                double ddx = 1.0 - ABSV(c->wx0 - 0.5), ddy = 1.0 - ABSV(c->wy0 - 0.5);
                if (ddx > 0.5 && ddy > 0.5) {
                    double swt2 = 1.0 * 4.0 * (ddx - 0.5) * (ddy - 0.5);
                    q[40] += c->lnu * swt2;
                    q[41] += swt2;
                }
            }
        }
        for (int64_t m1 = 0; m1 < nx; m1++)
            for (int64_t m2 = 0; m2 < ny; m2++) {
                int64_t m3 = m1 * ny + m2;
                double sm[10] = {0};
                for (int qd = 0; qd < 4; qd++) {
                    int64_t c1 = m1 - 1 + (qd >> 1), c2 = m2 - 1 + (qd & 1);
                    if (c1 < 0 || c2 < 0 || c1 > nx - 2 || c2 > ny - 2) continue;
                    const double *r = part + 42 * (c1 * (ny - 1) + c2) + 10 * (3 - qd);
                    for (int f = 0; f < 10; f++) sm[f] += r[f];
                }
                A.ro0[m3] = sm[0]; A.et0[m3] = sm[1]; A.cp0[m3] = sm[2]; A.kt0[m3] = sm[3];
                A.ht0[m3] = sm[4]; A.w0[m3] = sm[5]; A.tk0[m3] = sm[6]; A.w1[m3] = sm[7];
                A.nu0[m3] = sm[8]; A.wnu[m3] = sm[9];
                if (m1 >= 1 && m2 >= 1) {
                    const double *r = part + 42 * ((m1 - 1) * (ny - 1) + (m2 - 1));
                    A.nd0[m3] = 0.0 + r[40];
                    A.wnd[m3] = 0.0 + r[41];
                }
            }
        free(part);
    }
    /* node loop, markmart.c:917-994 */
    double numin = 0, numax = 0;
    for (int64_t m3 = 0; m3 < nn; m3++) {
        if (A.wnu[m3]) {
            double v;
            if (G->mu && G->mu[m3]) v = G->mu[m3];
            else {
                v = A.nu0[m3] / A.wnu[m3];
                if (P->viscmod == 1) v = exp(v);
                if (P->viscmod == 2) v = 1.0 / v;
            }
            if (v < P->nubeg) v = P->nubeg;
            if (v > P->nuend) v = P->nuend;
            if (numin == 0 || v < numin) numin = v;
            if (numax == 0 || v > numax) numax = v;
            out->nu[m3] = v;
        }
        if (A.wnd[m3]) {
            double v;
            if (G->mu && G->mu[m3]) v = G->mu[m3];
            else {
                v = A.nd0[m3] / A.wnd[m3];
                if (P->viscmod == 1) v = exp(v);
                if (P->viscmod == 2) v = 1.0 / v;
            }
            if (v < P->nubeg) v = P->nubeg;
            if (v > P->nuend) v = P->nuend;
            if (numin == 0 || v < numin) numin = v;
            if (numax == 0 || v > numax) numax = v;
            out->nd[m3] = v;
            out->po[m3] = 0.0 / A.wnd[m3]; /* po0[] is never accumulated (markmart.c:968) */
        }
        if (A.w0[m3]) {
            out->ro[m3] = A.ro0[m3] / A.w0[m3];
            out->et[m3] = A.et0[m3] / A.w0[m3];
            out->cp[m3] = A.cp0[m3] / A.w0[m3];
            out->kt[m3] = A.kt0[m3] / A.w0[m3];
            out->ht[m3] = A.ht0[m3] / A.w0[m3];
            if (A.w1[m3]) out->tk[m3] = A.tk0[m3] / A.w1[m3];
        }
    }
    /* contrast limit, markmart.c:1002-1009 */
    if (P->nucontr >= 1.0) numax = numin * P->nucontr; else numin = numax * P->nucontr;
    for (int64_t m3 = 0; m3 < nn; m3++) {
        if (out->nu[m3] < numin) out->nu[m3] = numin;
        if (out->nu[m3] > numax) out->nu[m3] = numax;
        if (out->nd[m3] < numin) out->nd[m3] = numin;
        if (out->nd[m3] > numax) out->nd[m3] = numax;
    }
    if (numin_numax) { numin_numax[0] = numin; numin_numax[1] = numax; }
    free(buf);
    free(cs);
    if (sinter) sinter->mag_time = sa.mag_time;
    return sa.stuck ? I2G_ETIMEOUT : I2G_OK;
}

/* ---------------------------------------------------------------- titerate markers */

/* allintert(), markmart.c:1687-1745 (intermod = 0) for a point inside the box:
 * the basic cell and its weights; the caller interpolates with bil(). */
static void tweights(const ora_grid *G, double x, double y, int64_t *m10, int64_t *m20, double *wx0, double *wx1,
                     double *wy0, double *wy1)
{
    *m10 = ora_m1serch(G->gx, G->xnumx, x);
    *m20 = ora_m1serch(G->gy, G->ynumy, y);
    ora_fdweight1(G->gx[*m10], G->gx[*m10 + 1], x, wx0, wx1);
    ora_fdweight1(G->gy[*m20], G->gy[*m20 + 1], y, wy0, wy1);
}

void ora_interp_tnode(const i2g_params *P, const ora_grid *G, int64_t n, const double *x, const double *y,
                      const double *tk, const double *tk2, double *out, double *out2)
{
    for (int64_t i = 0; i < n; i++) {
        double xi = x[i], yi = y[i];
        /* markmart.c:1697-1698 */
        if (xi < 0) xi = 0; else if (xi > P->xsize) xi = P->xsize;
        if (yi < 0) yi = 0; else if (yi > P->ysize) yi = P->ysize;
        int64_t m10, m20;
        double wx0, wx1, wy0, wy1;
        tweights(G, xi, yi, &m10, &m20, &wx0, &wx1, &wy0, &wy1);
        out[i] = bil(tk, G->ynumy, m10, m20, wx0, wx1, wy0, wy1);
        if (tk2 && out2) out2[i] = bil(tk2, G->ynumy, m10, m20, wx0, wx1, wy0, wy1);
    }
}

int ora_titerate_markers(const i2g_params *P, const ora_grid *G, int64_t n, const double *x, const double *y,
                         double *T, const int8_t *type, const double *tk_new, const double *tk_old,
                         const double *kt, const double *cp, const double *ro, double heatdif, double timestep,
                         int order)
{
    const int64_t nx = G->xnumx, ny = G->ynumy, nn = nx * ny, nc = (nx - 1) * (ny - 1);
    for (int64_t i = 0; i < n; i++)
        if (type[i] < 0 || type[i] >= 100) return I2G_EUNSUPPORTED;
    double *sol0 = (double *)calloc((size_t)nn, sizeof(double));
    double *sol1 = (double *)calloc((size_t)nn, sizeof(double));
    double *part = order == ORA_ORDER_CELL ? (double *)calloc((size_t)(8 * nc), sizeof(double)) : NULL;
    if (!sol0 || !sol1 || (order == ORA_ORDER_CELL && !part)) {
        free(sol0); free(sol1); free(part);
        return I2G_ENOMEM;
    }
#define INSIDE(i) (x[i] > 0 && y[i] > 0 && x[i] < P->xsize && y[i] < P->ysize)
    int64_t m10, m20;
    double wx0, wx1, wy0, wy1;
    /* fluid markers take the new node temperature (heatmart.c:523-533) */
    for (int64_t i = 0; i < n; i++)
        if (INSIDE(i) && type[i] >= 50 && type[i] < 100) {
            tweights(G, x[i], y[i], &m10, &m20, &wx0, &wx1, &wy0, &wy1);
            T[i] = bil(tk_new, ny, m10, m20, wx0, wx1, wy0, wy1);
        }
    /* rock markers: reset, subgrid diffusion, node change (heatmart.c:538-628) */
    for (int64_t i = 0; i < n; i++) {
        if (!(INSIDE(i) && type[i] < 50)) continue;
        tweights(G, x[i], y[i], &m10, &m20, &wx0, &wx1, &wy0, &wy1);
        const double tn = bil(tk_new, ny, m10, m20, wx0, wx1, wy0, wy1);
        const double to = bil(tk_old, ny, m10, m20, wx0, wx1, wy0, wy1);
        if (T[i] <= 0) T[i] = to;
        if (heatdif) {
            const double dtk = to - T[i];
            const double celdx = G->gx[m10 + 1] - G->gx[m10], celdy = G->gy[m20 + 1] - G->gy[m20];
            const double mkt = bil(kt, ny, m10, m20, wx0, wx1, wy0, wy1);
            const double mcp = bil(cp, ny, m10, m20, wx0, wx1, wy0, wy1);
            const double mro = bil(ro, ny, m10, m20, wx0, wx1, wy0, wy1);
            double dtk1 = -heatdif * mkt / mro / mcp * 2.0 * (1.0 / celdx / celdx + 1.0 / celdy / celdy) * timestep;
            if (dtk1 < -150.0) dtk1 = -150.0;
            dtk1 = dtk * (1.0 - exp(dtk1));
            T[i] += dtk1;
            /* node weights and diffusion changes (heatmart.c:606-621), swt1 = 1 */
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    const double ival = (a ? wx1 : wx0) * (b ? wy1 : wy0) * 1.0;
                    if (order == ORA_ORDER_REFERENCE) {
                        const int64_t m4 = (m10 + a) * ny + m20 + b;
                        sol0[m4] += ival;
                        sol1[m4] += dtk1 * ival;
                    } else {
                        double *q = part + 8 * (m10 * (ny - 1) + m20) + 2 * (a * 2 + b);
                        q[0] += ival;
                        q[1] += dtk1 * ival;
                    }
                }
        }
        T[i] += tn - to;
    }
    if (heatdif) {
        if (order == ORA_ORDER_CELL) {
            /* per node: 0 + its four cells' corner sums, cells (m1-1,m2-1), (m1-1,m2), (m1,m2-1), (m1,m2) */
            for (int64_t a = 0; a < nx; a++)
                for (int64_t b = 0; b < ny; b++) {
                    double s0 = 0, s1 = 0;
                    for (int qd = 0; qd < 4; qd++) {
                        const int64_t c1 = a - 1 + (qd >> 1), c2 = b - 1 + (qd & 1);
                        if (c1 < 0 || c2 < 0 || c1 > nx - 2 || c2 > ny - 2) continue;
                        const double *r = part + 8 * (c1 * (ny - 1) + c2) + 2 * (3 - qd);
                        s0 += r[0];
                        s1 += r[1];
                    }
                    sol0[a * ny + b] = s0;
                    sol1[a * ny + b] = s1;
                }
        }
        /* averaged node change (heatmart.c:638-652), then antidiffusion (:654-693) */
        for (int64_t m = 0; m < nn; m++)
            if (sol0[m]) sol1[m] /= sol0[m];
        for (int64_t i = 0; i < n; i++) {
            if (!(INSIDE(i) && type[i] < 50)) continue;
            tweights(G, x[i], y[i], &m10, &m20, &wx0, &wx1, &wy0, &wy1);
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    const int64_t m4 = (m10 + a) * ny + m20 + b;
                    const double ival = (a ? wx1 : wx0) * (b ? wy1 : wy0);
                    if (sol1[m4]) T[i] -= sol1[m4] * ival;
                }
        }
    }
#undef INSIDE
    free(sol0);
    free(sol1);
    free(part);
    return I2G_OK;
}
