// Device-side data views and the marker-step physics shared by every kernel.
//
// The physics follows the reference marker step:
//   cell search         m1serch/m2serch        markmart.c:1051-1088
//   linear weights      fdweight(1,0,x)        movemart.c:1269-1319 via nodewt markmart.c:1292-1373
//   velocity gather     allinterv              markmart.c:1378-1453
//   P/strain gather     allintere              markmart.c:1458-1543
//   rheology            viscalc                markmart.c:1855-2062
//   density             dencalc                markmart.c:1024-1046
//
// Two precision forms are instantiated from the same templates:
//   MIXED=false  every operation in FP64, written in the reference's evaluation
//                order.  The translation unit that instantiates it is compiled
//                with --fmad=false, so no multiply-add is contracted and marker
//                positions/pressures match the reference arithmetic bit for bit.
//   MIXED=true   weights, interpolated fields and property x weight products in
//                FP32; the cell search, stencil switches, marker coordinates, the
//                RK4 displacement sum, log-viscosity products and all per-node
//                accumulation stay FP64.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/i2g.h"

namespace i2g {

constexpr int kTypes = I2G_MAXTYPES;

// grid fields and derived lookup tables, all in device memory
struct GridView {
    int64_t nx, ny;  // xnumx, ynumy (grid lines)
    double xsize, ysize;
    double inv_x, inv_y;  // (n-1)/(g[n-1]-g[0]): first guess of the cell search
    const double *gx, *gy;
    const double *xmid, *ymid;  // (g[i]+g[i+1])/2.0, i < n-1: staggered node coordinates
    const double *vx, *vy, *pr, *ga;
    const double *exx, *eyy, *exy, *sxx, *syy, *sxy;  // NULL when absent (all zero)
    const double *mu;                                  // NULL when absent
    // FP32 copies for the mixed form
    const float *vxf, *vyf, *prf, *gaf;
    const float *exxf, *eyyf, *exyf, *sxxf, *syyf, *sxyf;  // NULL when absent (all zero)
    // mixed form: bilinear coefficients of each 2x2 stencil of vx, vy, pr at its
    // lower-left node, {a, c-a, b-a, a-b-c+d} for a=f(m1,m2), b=f(m1,m2+1),
    // c=f(m1+1,m2), d=f(m1+1,m2+1): one 16-byte load per interpolation
    const float4 *vxq, *vyq, *prq;
    // uniform grid, mixed form: per quarter cell (half a cell along each axis,
    // index (2 i + qx) * 2 (ny - 1) + 2 j + qy) the bilinear forms of vx and vy in
    // the quarter's own coordinates, two float4; NULL when absent
    const float4 *vq4;
    const float *ixb, *iyb;  // 1/(g[i+1]-g[i])
    const float *ixm, *iym;  // 1/(mid[i+1]-mid[i])
    const float4 *lx, *ly;   // per grid line: {width, 1/width, 1/mid spacing, 0}
    // uniform axes (uni != 0): every line i within 1e-9 of a width of g[0] + i w,
    // so cells and offsets follow from arithmetic instead of the line tables
    int32_t uni;
    double gx0, gy0;          // first lines
    double wx, wy, iwx, iwy;  // width and its inverse, FP64
    float fwx, fwy, fiwx, fiwy;  // the same, FP32
};

// markers in device (cell-sorted) order
struct MarkerView {
    int64_t n;
    double *x, *y, *T, *eta, *p;
    double *tmax, *hi, *por;  // NULL when not tracked
    int8_t *type;
    int32_t *id;  // caller index of the marker held in each slot
    int8_t *mgo;  // magnetisation state and time (markmg_old, markmg_time); NULL when not produced
    double *mgt;
};

struct DevTypes {
    i2g_types t;
};

struct MoveArgs {
    double timestep, timesum, relax_time, nubeg, nuend;
    int32_t markmod, outgrid;
    uint32_t flags;
    // markers held in the reference's single-precision storage (headmart.c:122):
    // the position update rounds like markx[] += (float)(timestep * vx0)
    // (markmart.c:119-120), the displacement to FP32, then the FP32 sum
    int32_t f32pos;
};

// x + dt v, or, for markers in single-precision storage, the FP32 sum of the
// position and the FP32 displacement (x holds an FP32 value there)
__device__ __forceinline__ double advance(double x, double dt, double v, int f32pos)
{
    if (f32pos) return (double)((float)x + (float)(dt * v));
    return x + dt * v;
}

// the densimod 2 table and the melt state the table markers pass on
// (i2g_td.cuh); rh is NULL unless the call has densimod 2
struct TdArgs {
    // (density kg/m^3, enthalpy J/kg) per [database][tk][pb] node: the
    // reference's td[tk][pb][db][0] * 1000.0 and td[tk][pb][db][1] * 1000.0 * 4.1837
    // (markmart.c:2147-2154), products formed once on the host in that order
    const double2 *rh;
    double tkmin, pbmin, tkstp, pbstp;
    int32_t tknum, pbnum;
    int32_t si_melting, ice_melting;
    // 1 (FP64 form): the reference's own expressions, libm pow included; 0 (mixed
    // form): the same polynomials by Horner's rule, integer powers as products,
    // pow(x, 0.5) as sqrt
    int32_t exact;
    const int32_t *prev;    // inclusive max-scan of the table markers' caller indices (-1: none yet)
    const int32_t *last;    // prev[n - 1]: the caller index of the call's last table marker
    const double *si;       // eps[21] each table marker leaves, by caller index
    const double *melt_in;  // eps[21], eps[22], eps[50], eps[51], eps[52], eps[53] before the call
    double *melt_out;       // the same after it: written by the last table marker
};

// per-call constants of the averaging
struct AvgArgsK {
    double timesum, tmp_ambient, core_form_time, k_cutoff, relax_time, nubeg, nuend;
    double xmelt_si, xmelt_fe;
    double rad_si, rad_fe, rad_ch;  // radiogenic heating per kg, markmart.c:749-837
    // smallest squared distance from the box centre whose square root exceeds
    // 0.95 xsize / 2 (the radmax test, markmart.c:268, 335-340): rad2 is the smallest
    // double whose pow(., 0.5) in the host's libm exceeds the radius, so
    // "d2 >= rad2" is the reference's "pow(d2, 0.5) > 0.95 xsize / 2" wherever that
    // pow is monotone
    double rad2;
    int32_t gridmod, densimod, viscmod, track_tmax;
    TdArgs td;
    // porosity sintering (markmart.c:362-466): the global timestep it reads, the
    // initial porosity, markpor[] in single-precision storage, and a counter of
    // grain-size searches that gave up (NULL: the call tracks no porosity)
    double timestep, por_init;
    int32_t f32por;
    unsigned int *sinter_stuck;
    // magnetisation (markmart.c:651-744): ronurecalc's local mag_time carries the
    // last assigned time from marker to marker: per caller index the value a
    // marker assigns (mag_val) and, by an inclusive max-scan, the last assigning
    // marker so far (mag_prev, -1: none); mag_in / mag_out the value before and
    // after the call (written by the last assigning marker, mag_last)
    int32_t dynamo;
    const int32_t *mag_prev;
    const double *mag_val;
    const double *mag_in;
    double *mag_out;
    const int32_t *mag_last;
};

// node outputs of ronurecalc()
struct NodeOut {
    double *ro, *nu, *nd, *et, *cp, *kt, *ht, *tk, *po;
    double *w1;  // optional: temperature weight sum per node (for the adjoint)
};

// ------------------------------------------------------------------ search
// Largest m in [0, n-2] with g[m] <= x (0 when x < g[0]): exactly the result of
// the reference's bisection for a strictly increasing g (checked at i2g_set_grid).
// A one-step guess from the mean spacing is verified with the same comparison the
// bisection uses; anything else falls back to the bisection itself.
__device__ __forceinline__ int64_t cell_search(const double *__restrict__ g, int64_t n, double inv,
                                               double x)
{
    if (!(x == x)) return n - 2;  // NaN: every "g[m] > x" test is false
    double t = (x - g[0]) * inv;
    int64_t m;
    if (!(t > 0.0)) m = 0;
    else if (t >= (double)(n - 2)) m = n - 2;
    else m = (int64_t)t;
    double gm = __ldg(g + m);
    if (gm <= x) {
        if (m == n - 2 || __ldg(g + m + 1) > x) return m;
        if (m + 1 == n - 2 || __ldg(g + m + 2) > x) return m + 1;
    } else {
        if (m == 0) return 0;
        if (__ldg(g + m - 1) <= x) return m - 1;
    }
    int64_t lo = 0, hi = n - 1;
    do {
        int64_t mid = (lo + hi) / 2;
        if (__ldg(g + mid) > x) hi = mid; else lo = mid;
    } while ((hi - lo) > 1);
    if (lo > n - 2) lo = n - 2;
    return lo;
}

// cell_search started from a nearby cell m in [0, n-2] (a marker's cell at an
// earlier point of its step): walks to the same result, largest m in [0, n-2]
// with g[m] <= x, 0 when x < g[0], n-2 for NaN.
__device__ __forceinline__ int cell_walk(const double *__restrict__ g, int n, int m, double x)
{
    if (!(x == x)) return n - 2;
    if (__ldg(g + m) > x) {
        do {
            --m;
        } while (m > 0 && __ldg(g + m) > x);
        return m;
    }
    while (m < n - 2 && __ldg(g + m + 1) <= x) ++m;
    return m;
}

// ------------------------------------------------------------------ weights
// Two-point order-0 Fornberg weights in the reference's operation order.
__device__ __forceinline__ void fdw64(double x0, double x1, double xi, double &w0, double &w1)
{
    double c5 = x0 - xi, c4 = x1 - xi, c3 = x1 - x0;
    w1 = (-c5) / c3;
    w0 = c4 / c3;
}

// FP32 weights from an FP64 offset and a precomputed FP32 reciprocal spacing.
__device__ __forceinline__ void fdw32(double x0, float inv_h, double xi, float &w0, float &w1)
{
    w1 = (float)(xi - x0) * inv_h;
    w0 = 1.0f - w1;
}

// sum over the 2x2 stencil, m1 outer / m2 inner, from 0 (markmart.c:1414-1421)
__device__ __forceinline__ double bil64(const double *__restrict__ f, int64_t ny, int64_t m1, int64_t m2,
                                        double wx0, double wx1, double wy0, double wy1)
{
    const double *p0 = f + m1 * ny + m2, *p1 = p0 + ny;
    double s = 0.0;
    s += (wx0 * wy0) * __ldg(p0);
    s += (wx0 * wy1) * __ldg(p0 + 1);
    s += (wx1 * wy0) * __ldg(p1);
    s += (wx1 * wy1) * __ldg(p1 + 1);
    return s;
}

__device__ __forceinline__ float bil32(const float *__restrict__ f, int64_t ny, int64_t m1, int64_t m2,
                                       float wx0, float wx1, float wy0, float wy1)
{
    const float *p0 = f + m1 * ny + m2, *p1 = p0 + ny;
    return wx0 * (wy0 * __ldg(p0) + wy1 * __ldg(p0 + 1)) + wx1 * (wy0 * __ldg(p1) + wy1 * __ldg(p1 + 1));
}

__device__ __forceinline__ void clampxy(const GridView &G, double &x, double &y)
{
    if (x < 0) x = 0; else if (x > G.xsize) x = G.xsize;
    if (y < 0) y = 0; else if (y > G.ysize) y = G.ysize;
}

// ------------------------------------------------------------------ gathers
// allinterv(): velocity at (x, y).  Returns FP64 components in both forms.
template <bool MIXED>
__device__ __forceinline__ void interp_v(const GridView &G, double x, double y, double &vxo, double &vyo)
{
    clampxy(G, x, y);
    const int64_t nx = G.nx, ny = G.ny;
    const int64_t m10 = cell_search(G.gx, nx, G.inv_x, x), m20 = cell_search(G.gy, ny, G.inv_y, y);
    int64_t m2 = m20;
    if (y < __ldg(G.ymid + m20)) m2 -= 1;
    if (m2 < 0) m2 = 0;
    if (m2 > ny - 3) m2 = ny - 3;
    int64_t m1 = m10;
    if (x < __ldg(G.xmid + m10)) m1 -= 1;
    if (m1 < 0) m1 = 0;
    if (m1 > nx - 3) m1 = nx - 3;
    if (!MIXED) {
        double wx0, wx1, wy0, wy1;
        fdw64(__ldg(G.gx + m10), __ldg(G.gx + m10 + 1), x, wx0, wx1);
        fdw64(__ldg(G.ymid + m2), __ldg(G.ymid + m2 + 1), y, wy0, wy1);
        vxo = bil64(G.vx, ny, m10, m2, wx0, wx1, wy0, wy1);
        fdw64(__ldg(G.xmid + m1), __ldg(G.xmid + m1 + 1), x, wx0, wx1);
        fdw64(__ldg(G.gy + m20), __ldg(G.gy + m20 + 1), y, wy0, wy1);
        vyo = bil64(G.vy, ny, m1, m20, wx0, wx1, wy0, wy1);
    } else {
        float wx0, wx1, wy0, wy1;
        fdw32(__ldg(G.gx + m10), __ldg(G.ixb + m10), x, wx0, wx1);
        fdw32(__ldg(G.ymid + m2), __ldg(G.iym + m2), y, wy0, wy1);
        vxo = (double)bil32(G.vxf, ny, m10, m2, wx0, wx1, wy0, wy1);
        fdw32(__ldg(G.xmid + m1), __ldg(G.ixm + m1), x, wx0, wx1);
        fdw32(__ldg(G.gy + m20), __ldg(G.iyb + m20), y, wy0, wy1);
        vyo = (double)bil32(G.vyf, ny, m1, m20, wx0, wx1, wy0, wy1);
    }
}

// cell-centre stencil of allintere() (markmart.c:1514-1522): lower index a, b >= 1
__device__ __forceinline__ void centre_stencil(const GridView &G, int64_t m10, int64_t m20, double x, double y,
                                               int64_t &a, int64_t &b)
{
    a = m10;
    if (x > __ldg(G.xmid + m10)) a += 1;
    if (a < 1) a = 1;
    if (a > G.nx - 2) a = G.nx - 2;
    b = m20;
    if (y > __ldg(G.ymid + m20)) b += 1;
    if (b < 1) b = 1;
    if (b > G.ny - 2) b = G.ny - 2;
}

// allintere(): pressure and gravity (and, if wanted, strain rates / stresses) at (x, y).
// e[0..5] = exy, sxy, exx, sxx, eyy, syy (only when full=true).
template <bool MIXED>
__device__ __forceinline__ void interp_e(const GridView &G, double x, double y, double &pr, double &ga,
                                         bool want_ga, bool full, double *e, int64_t &m10o, int64_t &m20o)
{
    clampxy(G, x, y);
    const int64_t nx = G.nx, ny = G.ny;
    const int64_t m10 = cell_search(G.gx, nx, G.inv_x, x), m20 = cell_search(G.gy, ny, G.inv_y, y);
    m10o = m10;
    m20o = m20;
    int64_t a, b;
    centre_stencil(G, m10, m20, x, y, a, b);
    double wx0, wx1, wy0, wy1;
    if (!MIXED) {
        fdw64(__ldg(G.xmid + a - 1), __ldg(G.xmid + a), x, wx0, wx1);
        fdw64(__ldg(G.ymid + b - 1), __ldg(G.ymid + b), y, wy0, wy1);
        pr = bil64(G.pr, ny, a, b, wx0, wx1, wy0, wy1);
        ga = (want_ga && G.ga) ? bil64(G.ga, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
    } else {
        float fx0, fx1, fy0, fy1;
        fdw32(__ldg(G.xmid + a - 1), __ldg(G.ixm + a - 1), x, fx0, fx1);
        fdw32(__ldg(G.ymid + b - 1), __ldg(G.iym + b - 1), y, fy0, fy1);
        pr = (double)bil32(G.prf, ny, a, b, fx0, fx1, fy0, fy1);
        ga = (want_ga && G.gaf) ? (double)bil32(G.gaf, ny, a, b, fx0, fx1, fy0, fy1) : 0.0;
        wx0 = fx0; wx1 = fx1; wy0 = fy0; wy1 = fy1;
    }
    if (full) {
        // cell-centre strain/stress reuse the centre weights; shear components on
        // interior basic nodes (markmart.c:1484-1504).  Kept in FP64 in both forms
        // (viscosity only; never on the throughput path).
        if (MIXED) {
            fdw64(__ldg(G.xmid + a - 1), __ldg(G.xmid + a), x, wx0, wx1);
            fdw64(__ldg(G.ymid + b - 1), __ldg(G.ymid + b), y, wy0, wy1);
        }
        e[2] = G.exx ? bil64(G.exx, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
        e[3] = G.sxx ? bil64(G.sxx, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
        e[4] = G.eyy ? bil64(G.eyy, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
        e[5] = G.syy ? bil64(G.syy, ny, a, b, wx0, wx1, wy0, wy1) : 0.0;
        int64_t c = m10, d = m20;
        if (c < 1) c = 1;
        if (c > nx - 3) c = nx - 3;
        if (d < 1) d = 1;
        if (d > ny - 3) d = ny - 3;
        fdw64(__ldg(G.gx + c), __ldg(G.gx + c + 1), x, wx0, wx1);
        fdw64(__ldg(G.gy + d), __ldg(G.gy + d + 1), y, wy0, wy1);
        e[0] = G.exy ? bil64(G.exy, ny, c, d, wx0, wx1, wy0, wy1) : 0.0;
        e[1] = G.sxy ? bil64(G.sxy, ny, c, d, wx0, wx1, wy0, wy1) : 0.0;
    }
}

// ------------------------------------------------------------------ rheology
// pow(v, 0.5) of the reference, by sqrt: within one unit in the last place of the
// reference's libm pow (which is not correctly rounded: about 0.08% of doubles
// come out one unit away from the correctly rounded sqrt), where CUDA's pow is
// within 2 ulp and far slower.  pow's +0 for -0 and +inf for -inf (C99 F.9.4.4)
// are kept; sqrt alone gives -0 and NaN.
__device__ __forceinline__ double pow_half(double v) { return v == -INFINITY ? INFINITY : sqrt(v) + 0.0; }

// viscalc(), markmart.c:1855-2062.  mm2 is the table index the caller selected
// (type, or type-20 for partially molten types, markmart.c:59-66).
__device__ inline double viscalc(const i2g_types &T, double mtk, double mpb, double hi, double epsin,
                                 double sigin, double rii, double timesum, double relax_time, double nubeg,
                                 double nuend, int mm2)
{
    if (mm2 > 20) return T.markn0[mm2];
    double rt = 8.314 * mtk;
    double lamb = T.markll[mm2], abrit = T.marka0[mm2], bbrit = T.markb0[mm2];
    double sbrit = abrit + bbrit * mpb * 1e+5 * lamb;
    if (T.marks0[mm2] <= 0 && sbrit > T.marks1[mm2]) sbrit = T.marks1[mm2];
    if (sbrit > 0 && hi > 0 &&
        ((timesum - (hi * 1.000e+6 * 365.250 * 24.000 * 3600.000)) <
         (relax_time * 1.000e+6 * 365.250 * 24.000 * 3600.000)))
        sbrit = 1.000e+6;
    double nubrit = 0;
    if (epsin > 0 && (bbrit > 0 || abrit * lamb > 0)) {
        if (sbrit > 0) nubrit = 1.0 / (0.5 * sbrit / epsin / rii);
        else nubrit = 1.0 / T.markn0[mm2];
    }
    double nupeierls = 0;
    if (T.marks0[mm2] > 0 && sigin > 1e+7 && epsin > 0) {
        double A = T.marks0[mm2], sig0 = T.marks1[mm2], s = sig0 * 0.95;
        for (int n2 = 0; n2 < 5; n2++) {
            s = pow_half(-rt / (T.markdh[mm2] + T.markdv[mm2] * mpb) * log(epsin / A / s / s));
            if (s > 1.0) s = -s;
            s = (1.0 - s) * sig0;
        }
        if (s > sig0) s = sig0;
        nupeierls = 1.0 / (0.5 * s / epsin);
    }
    double nunewt = 0, nupowl = 0;
    const double nu0 = T.marknu[mm2], dh = T.markdh[mm2], dv = T.markdv[mm2];
    const double ss = T.markss[mm2], mm = T.markmm[mm2];
    if (nu0) {
        if (dh == 0 && dv == 0 && (ss == 0 || mm == 1.0)) nunewt = 1.0 / nu0;
        if ((dh != 0 || dv != 0) && (ss == 0 || mm == 1.0)) {
            double e1 = (dh + dv * mpb) / rt;
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
            double k1 = nu0 / pow(ss, mm - 1.0);
            nunewt = 1.0 / (0.5 * k1);
            double sduct = pow(nu0 * epsin, 1.0 / mm);
            if (epsin > 0) nupowl = 1.0 / (0.5 * sduct / epsin);
        }
        if ((dh != 0 || dv != 0) && ss != 0 && mm != 1.0) {
            double e1 = (dh + dv * mpb) / rt;
            if (e1 > 150.0) e1 = 150.0;
            e1 = exp(e1);
            double k1 = nu0 / pow(ss, mm - 1.0);
            nunewt = 1.0 / (0.5 * k1 * e1);
            double sduct = pow(nu0 * e1 * epsin, 1.0 / mm);
            if (epsin > 0) nupowl = 1.0 / (0.5 * sduct / epsin);
        }
    }
    double nueff = nunewt + nupowl;
    if (nubrit > nueff) nueff = nubrit;
    if (nupeierls > nueff) nueff = nupeierls;
    if (nueff <= 0) nueff = 1.0 / T.markn1[mm2];
    nueff = 1.0 / nueff;
    if (nueff < T.markn0[mm2]) nueff = T.markn0[mm2];
    if (nueff > T.markn1[mm2]) nueff = T.markn1[mm2];
    if (nueff < nubeg) nueff = nubeg;
    if (nueff > nuend) nueff = nuend;
    return nueff;
}

// strain-rate and stress invariants (markmart.c:47-48)
__device__ __forceinline__ void invariants(const double *e, double &eii, double &sii)
{
    eii = pow_half(0.5 * (e[2] * e[2] + e[4] * e[4]) + e[0] * e[0]);
    sii = pow_half(0.5 * (e[3] * e[3] + e[5] * e[5]) + e[1] * e[1]);
}

// ------------------------------------------------------------------ mixed fast path
// One axis of a gather point, FP32: the basic cell m (exact FP64 search) with its
// weights, and the staggered (midpoint) stencil with its weights, both from the
// FP32 offset of the point inside cell m.  The staggered choice compares that
// offset with half the cell width in FP32 instead of x with the FP64 midpoint
// (markmart.c:1406/1431/1514), which can pick the other, equally valid stencil
// for a point within FP32 rounding of a midpoint; both give the same bilinear
// value up to rounding.
struct AxisF {
    int b, m;          // basic cell, lower staggered index
    float b0, b1;      // basic weights
    float m0, m1;      // staggered weights
};

// the tail of axis_fast: weights of the basic cell b at FP32 offset d from g[b],
// and the staggered stencil with its weights
__device__ __forceinline__ void axis_tail(const float4 *__restrict__ L, int64_t n, int b, float d, AxisF &A)
{
    const float4 lb = __ldg(L + b);
    A.b = b;
    A.b1 = d * lb.y;
    A.b0 = 1.0f - A.b1;
    int m = (A.b1 < 0.5f) ? b - 1 : b;
    if (m < 0) m = 0;
    if (m > (int)n - 3) m = (int)n - 3;
    float t;
    if (m == b) {
        t = (d - 0.5f * lb.x) * lb.z;
    } else {
        const float4 lp = __ldg(L + b - 1);
        t = (d + 0.5f * lp.x) * lp.z;
    }
    A.m = m;
    A.m1 = t;
    A.m0 = 1.0f - t;
}

__device__ __forceinline__ void axis_fast(const double *__restrict__ g, const float4 *__restrict__ L, int64_t n,
                                          double inv, double x, int hint, AxisF &A)
{
    const int b = hint >= 0 ? cell_walk(g, (int)n, hint, x) : (int)cell_search(g, n, inv, x);
    axis_tail(L, n, b, (float)(x - __ldg(g + b)), A);
}

// One axis of a marker's RK4 in the mixed form: the first stage's basic cell b,
// the marker's FP32 offset du from g[b] (unclamped) and the box [0, size] as
// offsets from g[b].  The later stage points are FP32 offsets du + c dt v from
// g[b] (a stage moves a marker by a fraction of a cell): clamped to the box and
// walked to their cell over the FP32 cell widths, without FP64 arithmetic.
struct AxisRK {
    int b;
    float du, lo, hi;
};

__device__ __forceinline__ void axis_stage(const float4 *__restrict__ L, int64_t n, const AxisRK &R, float e,
                                           AxisF &A)
{
    if (e < R.lo) e = R.lo;
    if (e > R.hi) e = R.hi;
    int b = R.b;
    while (e < 0.0f && b > 0) {
        --b;
        e += __ldg(L + b).x;
    }
    while (b < (int)n - 2) {
        const float w = __ldg(L + b).x;
        if (!(e >= w)) break;
        e -= w;
        ++b;
    }
    axis_tail(L, n, b, e, A);
}

__device__ __forceinline__ float bil32i(const float *__restrict__ f, int ny, int m1, int m2, float wx0, float wx1,
                                        float wy0, float wy1)
{
    const float *p0 = f + m1 * ny + m2, *p1 = p0 + ny;
    return wx0 * (wy0 * __ldg(p0) + wy1 * __ldg(p0 + 1)) + wx1 * (wy0 * __ldg(p1) + wy1 * __ldg(p1 + 1));
}

// the bilinear interpolation of a stencil from its coefficients (the same
// weighted sum as bil32i, regrouped as a + wx1 (c-a) + wy1 (b-a) + wx1 wy1 (a-b-c+d))
__device__ __forceinline__ float bilq(const float4 *__restrict__ q, int ny, int m1, int m2, float wx1, float wy1)
{
    const float4 c = __ldg(q + m1 * ny + m2);
    return fmaf(wx1 * wy1, c.w, fmaf(wy1, c.z, fmaf(wx1, c.y, c.x)));
}

// First RK4 stage of the mixed form (allinterv() at the marker): vx (basic x,
// staggered y), vy (staggered x, basic y) and, when pr is given, the cell-centre
// pressure of allintere() (staggered x and y, index + 1); exact FP64 cell search
// and offsets.  Returns the axis data of the later stages.
__device__ __forceinline__ void stage1_fast(const GridView &G, double x, double y, double &vx, double &vy, double *pr,
                                            AxisRK &RX, AxisRK &RY, AxisF *Xo = nullptr, AxisF *Yo = nullptr)
{
    double xc = x, yc = y;
    clampxy(G, xc, yc);
    const int bx = (int)cell_search(G.gx, G.nx, G.inv_x, xc), by = (int)cell_search(G.gy, G.ny, G.inv_y, yc);
    const double gbx = __ldg(G.gx + bx), gby = __ldg(G.gy + by);
    AxisF X, Y;
    axis_tail(G.lx, G.nx, bx, (float)(xc - gbx), X);
    axis_tail(G.ly, G.ny, by, (float)(yc - gby), Y);
    RX.b = bx;
    RX.du = (float)(x - gbx);
    RX.lo = (float)(0.0 - gbx);
    RX.hi = (float)(G.xsize - gbx);
    RY.b = by;
    RY.du = (float)(y - gby);
    RY.lo = (float)(0.0 - gby);
    RY.hi = (float)(G.ysize - gby);
    const int ny = (int)G.ny;
    vx = (double)bilq(G.vxq, ny, X.b, Y.m, X.b1, Y.m1);
    vy = (double)bilq(G.vyq, ny, X.m, Y.b, X.m1, Y.b1);
    if (pr) *pr = (double)bilq(G.prq, ny, X.m + 1, Y.m + 1, X.m1, Y.m1);
    if (Xo) {
        *Xo = X;
        *Yo = Y;
    }
}

// a later RK4 stage of the mixed form at offsets (ex, ey) from the first stage's cell
__device__ __forceinline__ void stage_fast(const GridView &G, const AxisRK &RX, const AxisRK &RY, float ex, float ey,
                                           float &vx, float &vy)
{
    AxisF X, Y;
    axis_stage(G.lx, G.nx, RX, ex, X);
    axis_stage(G.ly, G.ny, RY, ey, Y);
    const int ny = (int)G.ny;
    vx = bilq(G.vxq, ny, X.b, Y.m, X.b1, Y.m1);
    vy = bilq(G.vyq, ny, X.m, Y.b, X.m1, Y.b1);
}

// the mixed RK4 velocity of a marker: (vx1, vy1, pr) at the marker, then the three
// later stages in FP32 offsets; the stage sum in FP64 (markmart.c:73-115)
__device__ __forceinline__ void rk4_mixed(const GridView &G, double x, double y, double dt, int markmod, double &vx0,
                                          double &vy0, double *pr, int &hx, int &hy, AxisF *X1 = nullptr,
                                          AxisF *Y1 = nullptr)
{
    double vx1, vy1;
    AxisRK RX, RY;
    stage1_fast(G, x, y, vx1, vy1, pr, RX, RY, X1, Y1);
    hx = RX.b;
    hy = RY.b;
    if (markmod == 1) {
        vx0 = vx1;
        vy0 = vy1;
        return;
    }
    const float h = (float)(dt / 2.0), f = (float)dt;
    float v2x, v2y, v3x, v3y, v4x, v4y;
    stage_fast(G, RX, RY, RX.du + h * (float)vx1, RY.du + h * (float)vy1, v2x, v2y);
    stage_fast(G, RX, RY, RX.du + h * v2x, RY.du + h * v2y, v3x, v3y);
    stage_fast(G, RX, RY, RX.du + f * v3x, RY.du + f * v3y, v4x, v4y);
    // times 1/6 rather than an IEEE division (a last-bit difference, within this
    // form's bar, for two FP64 division sequences less per marker)
    constexpr double sixth = 1.0 / 6.0;
    vx0 = (vx1 + 2.0 * (double)v2x + 2.0 * (double)v3x + (double)v4x) * sixth;
    vy0 = (vy1 + 2.0 * (double)v2y + 2.0 * (double)v3y + (double)v4y) * sixth;
}

// allintere()'s strain rates and stresses (markmart.c:1476-1504) in the mixed
// form from the first stage's stencils: exx, sxx, eyy, syy at the cell centres
// with the pressure's weights; exy, sxy on the interior basic nodes (the cell
// clamped to [1, n-3]), with the basic weights or, at a clamped edge cell, the
// FP32 weights from the shifted node.  e[0..5] = exy, sxy, exx, sxx, eyy, syy.
__device__ __forceinline__ void strain_mixed(const GridView &G, double x, double y, const AxisF &X, const AxisF &Y,
                                             double *e)
{
    const int ny = (int)G.ny, a = X.m + 1, b = Y.m + 1;
    e[2] = G.exxf ? (double)bil32i(G.exxf, ny, a, b, X.m0, X.m1, Y.m0, Y.m1) : 0.0;
    e[3] = G.sxxf ? (double)bil32i(G.sxxf, ny, a, b, X.m0, X.m1, Y.m0, Y.m1) : 0.0;
    e[4] = G.eyyf ? (double)bil32i(G.eyyf, ny, a, b, X.m0, X.m1, Y.m0, Y.m1) : 0.0;
    e[5] = G.syyf ? (double)bil32i(G.syyf, ny, a, b, X.m0, X.m1, Y.m0, Y.m1) : 0.0;
    int c = X.b, d = Y.b;
    if (c < 1) c = 1;
    if (c > (int)G.nx - 3) c = (int)G.nx - 3;
    if (d < 1) d = 1;
    if (d > ny - 3) d = ny - 3;
    float wx0 = X.b0, wx1 = X.b1, wy0 = Y.b0, wy1 = Y.b1;
    if (c != X.b || d != Y.b) {
        double xc = x, yc = y;
        clampxy(G, xc, yc);
        if (c != X.b) fdw32(__ldg(G.gx + c), __ldg(G.ixb + c), xc, wx0, wx1);
        if (d != Y.b) fdw32(__ldg(G.gy + d), __ldg(G.iyb + d), yc, wy0, wy1);
    }
    e[0] = G.exyf ? (double)bil32i(G.exyf, ny, c, d, wx0, wx1, wy0, wy1) : 0.0;
    e[1] = G.sxyf ? (double)bil32i(G.sxyf, ny, c, d, wx0, wx1, wy0, wy1) : 0.0;
}

// cell index in x-major order, matching the node layout; (cx, cy): a nearby cell
// to start the searches from (-1: none)
__device__ __forceinline__ int32_t cell_key(const GridView &G, double x, double y, int cx = -1, int cy = -1)
{
    clampxy(G, x, y);
    const int64_t m10 = cx >= 0 ? cell_walk(G.gx, (int)G.nx, cx, x) : cell_search(G.gx, G.nx, G.inv_x, x);
    const int64_t m20 = cy >= 0 ? cell_walk(G.gy, (int)G.ny, cy, y) : cell_search(G.gy, G.ny, G.inv_y, y);
    return (int32_t)(m10 * (G.ny - 1) + m20);
}

}  // namespace i2g
