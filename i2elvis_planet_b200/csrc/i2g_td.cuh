// The thermodynamic-table property model of densimod 2: tdbasecalc()
// (markmart.c:2068-2276) and the parts of meltpart1() (markmart.c:2336-2652) it
// reaches.
//
// ronurecalc() hands the table types (5, 6, 11, 12, 25, 26, 31, 32;
// markmart.c:481-493) to tdbasecalc(), which interpolates density and enthalpy
// in a P-T table, adds the melt (and, for type 6, water-ice) terms, and flips
// the marker between its solid (< 20) and molten (> 20) type.  meltpart1() leaves
// its melt fractions in the globals eps[21], eps[50], eps[52]; ronurecalc()
// reads them at the top of the NEXT marker (markmart.c:287-289), so the melt
// fraction a molten marker's conductivity sees (markmart.c:509-560) is that of
// the table marker before it in the caller's order.  The device form keeps that
// dependence without a sequential loop: k_td_melt stores, per caller index, the
// silicate melt fraction each table marker leaves behind; an inclusive
// max-scan over caller indices gives every marker its predecessor; the
// averaging reads the predecessor's value.  The last table marker writes the
// six globals' values after the call (melt_out).
//
// meltpart1() is only reached with table types, so its iron branch
// (markmart.c:2464-2580) never runs here: eps[50] and eps[51] are zero after any
// table marker.
#pragma once

#include "i2g_dev.cuh"

namespace i2g {

__host__ __device__ __forceinline__ bool td_type(int t)
{
    return t == 5 || t == 6 || t == 11 || t == 12 || t == 25 || t == 26 || t == 31 || t == 32;
}

// Silicate solidus, liquidus and latent heat of a table type (markmart.c:2352-2412)
__device__ __forceinline__ void si_curve(double mpb, int mm2, int si_melting, bool exact, double &ts, double &tl,
                                         double &hl)
{
    ts = 0.0;
    tl = 0.0;
    hl = 0.0;
    if (mm2 == 11 || mm2 == 12 || mm2 == 31 || mm2 == 32) {
        // wet basalt solidus (Schmidt & Poli 1998), dry tholeiite liquidus (Hess 1989)
        const double ykm = mpb * 3e-3;
        if (ykm < 48.0)
            ts = 972.6 - 2111.0 / (ykm + 10.63) + 70033.0 / (ykm + 10.63) / (ykm + 10.63);
        else
            ts = 935.4 + 0.1162 * ykm + 0.006937 * ykm * ykm;
        tl = 1423.15 + 3.5 * ykm;
        hl = 380000.0;
        return;
    }
    // peridotite (5, 25, 26) and wet planetesimal material (6)
    if (si_melting == 0) {
        // Hirschmann (2000), linear above 10 GPa
        if (mpb < 10e+4)
            ts = 273.15 + 1120.661 + 132.899e-4 * mpb - 5.104e-8 * mpb * mpb;
        else
            ts = 273.15 + 1939.251 + 30.819e-4 * (mpb - 10e+4);
    } else if (si_melting == 1) {
        // Herzberg et al. (2000), linear above 21.5 GPa
        if (mpb < 21.50e+4 && exact)
            ts = 273.15 + 1143.04342 + 58.2946423e-4 * mpb + 52.3439318e-8 * mpb * mpb -
                 16.3201032e-12 * mpb * mpb * mpb + 2.29886314e-16 * pow(mpb, 4.000) -
                 0.180865486e-20 * pow(mpb, 5.000) + 0.00815679773e-24 * pow(mpb, 6.000) -
                 0.000197104325e-28 * pow(mpb, 7.000) + 1.97908526e-38 * pow(mpb, 8.000);
        else if (mpb < 21.50e+4)
            ts = 273.15 + 1143.04342 +
                 mpb * (58.2946423e-4 +
                        mpb * (52.3439318e-8 +
                               mpb * (-16.3201032e-12 +
                                      mpb * (2.29886314e-16 +
                                             mpb * (-0.180865486e-20 +
                                                    mpb * (0.00815679773e-24 +
                                                           mpb * (-0.000197104325e-28 + mpb * 1.97908526e-38)))))));
        else
            ts = 273.15 + 2157.500 + 11.7297e-4 * (mpb - 21.50e+4);
    }
    tl = 1973.000 + 28.570e-4 * mpb;  // Wade & Wood (2005)
    hl = 400000.0;
}

// eps[21] (melt fraction) and eps[22] (latent heat) of meltpart1 (markmart.c:2598-2613)
__device__ __forceinline__ double si_frac(double mtk, double ts, double tl)
{
    if (!(tl != 0.0)) return 0.0;
    if (ts >= tl - 100.0) ts = tl - 100.0;
    double x = (mtk - ts) / (tl - ts);
    if (x < 0.0000) x = 0.0000;
    if (x > 1.0000) x = 1.0000;
    return x;
}

// A type's solidus, liquidus and latent heat at one pressure.  The melt
// fractions at several temperatures and the same pressure (and type class: a
// flip by 20 keeps the class) share one curve evaluation.
struct SiCurve {
    double ts, tl, hl;
    __device__ __forceinline__ double frac(double mtk) const { return si_frac(mtk, ts, tl); }
    __device__ __forceinline__ double latent(double mtk) const { return (tl != 0.0) ? hl * si_frac(mtk, ts, tl) : 0.0; }
};

static __device__ __noinline__ SiCurve si_at(double mpb, int mm2, int si_melting, bool exact)
{
    SiCurve c;
    si_curve(mpb, mm2, si_melting, exact, c.ts, c.tl, c.hl);
    return c;
}

// Water-ice melting of type 6 (Dunaeva et al. 2010, markmart.c:2414-2460) with the
// 10 K gap between onset and full melting; ts = tl = 0 outside the fitted range
__device__ __forceinline__ void ice_curve(double mpb, bool exact, double &ts, double &tl)
{
    const double t_shift = 10.000;
    ts = 0.0;
    tl = 0.0;
    if (!exact) {
        // one log and one square root for both curves (tl = ts + the shift)
        if (!(mpb >= 0.000e6 && mpb < 9.000e5)) return;
        const double lg = log(mpb), sq = sqrt(mpb);
        if (mpb < 2085.66) ts = 273.0159 - 0.0132 * mpb - 0.1577 * lg + 0.1516 * sq;
        else if (mpb < 3501.0) ts = 10.277 + 0.0265 * mpb + 50.1624 * lg + (0.5868 / mpb) - 4.3288 * sq;
        else if (mpb < 6324.0) ts = 5.0321 - 0.0004 * mpb + 30.9482 * lg + (1.0018 / mpb);
        else if (mpb < 22160.0) ts = 4.2804 - 0.0013 * mpb + 21.8756 * lg + (1.0018 / mpb) + 1.0785 * sq;
        else if (mpb < 4.000e5) ts = -1355.42 + 0.0018 * mpb + 167.0609 * lg + (-0.6633 / mpb);
        else ts = 0.2524 + 0.0019 * mpb + 0.2795 * lg + (0.500 / mpb) + 1.1675 * sq;
        tl = ts + t_shift;
        return;
    }
    if (mpb >= 0.000e6 && mpb < 2085.66) {
        ts = 273.0159 - 0.0132 * mpb - 0.1577 * log(mpb) + 0.1516 * pow(mpb, 0.500);
        tl = t_shift + 273.0159 - 0.0132 * mpb - 0.1577 * log(mpb) + 0.1516 * pow(mpb, 0.500);
    }
    if (mpb >= 2085.66 && mpb < 3501.0) {
        ts = 10.277 + 0.0265 * mpb + 50.1624 * log(mpb) + (0.5868 / mpb) - 4.3288 * pow(mpb, 0.500);
        tl = t_shift + 10.277 + 0.0265 * mpb + 50.1624 * log(mpb) + (0.5868 / mpb) - 4.3288 * pow(mpb, 0.500);
    }
    if (mpb >= 3501.0 && mpb < 6324.0) {
        ts = 5.0321 - 0.0004 * mpb + 30.9482 * log(mpb) + (1.0018 / mpb);
        tl = t_shift + 5.0321 - 0.0004 * mpb + 30.9482 * log(mpb) + (1.0018 / mpb);
    }
    if (mpb >= 6324.000 && mpb < 22160.0) {
        ts = 4.2804 - 0.0013 * mpb + 21.8756 * log(mpb) + (1.0018 / mpb) + 1.0785 * pow(mpb, 0.500);
        tl = t_shift + 4.2804 - 0.0013 * mpb + 21.8756 * log(mpb) + (1.0018 / mpb) + 1.0785 * pow(mpb, 0.500);
    }
    if (mpb >= 22160.0 && mpb < 4.000e5) {
        ts = -1355.42 + 0.0018 * mpb + 167.0609 * log(mpb) + (-0.6633 / mpb);
        tl = t_shift - 1355.42 + 0.0018 * mpb + 167.0609 * log(mpb) + (-0.6633 / mpb);
    }
    if (mpb >= 4.000e5 && mpb < 9.000e5) {
        ts = 0.2524 + 0.0019 * mpb + 0.2795 * log(mpb) + (0.500 / mpb) + 1.1675 * pow(mpb, 0.500);
        tl = t_shift + 0.2524 + 0.0019 * mpb + 0.2795 * log(mpb) + (0.500 / mpb) + 1.1675 * pow(mpb, 0.500);
    }
}

// eps[52] (ice melt fraction) and eps[53] (its latent heat), markmart.c:2635-2649;
// zero for every type but 6 and when ice melting is off
static __device__ __noinline__ double ice_melt(double mtk, double mpb, int mm2, int ice_melting, bool exact,
                                              double *latent)
{
    double x = 0.0, h = 0.0;
    if (mm2 == 6 && ice_melting == 1) {
        double ts, tl;
        ice_curve(mpb, exact, ts, tl);
        if (tl != 0.0) {  // the reference's "if(tl_ice)" (true for NaN as well)
            x = (mtk - ts) / (tl - ts);
            if (x < 0.000) x = 0.0000;
            if (x > 1.000) x = 1.0000;
            h = (284000.0 + 233000.0) * 0.3 * x;
        }
    }
    if (latent) *latent = h;
    return x;
}

// tdbasecalc (markmart.c:2068-2276) for table type mm2 at temperature mtk (K) and
// pressure mpb (bar): the table's density, heat capacity and expansion term, the
// lattice + radiative conductivity (markmart.c:2086-2112; of the radiative terms
// only the 1 mm one is used), then the molten-rock mixture, molten viscosity and
// latent-heat terms.  mnu holds eps[48] (the viscosity so far) in and out.
// Returns the marker's new type (markmart.c:2180-2181).
static __device__ __noinline__ int td_props(const TdArgs &D, const i2g_types &T, double nubeg, double nuend, double mtk,
                                     double mpb, int mm2, double &mro_o, double &mcp_o, double &mbb_o, double &mkt_o,
                                     double &mnu)
{
    double mkt1, krad;
    if (mpb < 235000.0) {
        mkt1 = (1.878 + 770.9 / (mtk <= 1200.0 ? mtk : 1200.0)) * (1.0 + 4.26e-6 * mpb);
        const double t = mtk / 1774.0;
        krad = D.exact ? pow(t, 3.0) : t * t * t;
    } else {
        mkt1 = (1.291 + 1157.0 / (mtk <= 2100.0 ? mtk : 2100.0)) * (1.0 + 2.50e-6 * mpb);
        const double t = mtk / 2117.0;
        krad = D.exact ? pow(t, 3.0) : t * t * t;
    }
    // bilinear cell of the table (markmart.c:2118-2139); a NaN coordinate, which
    // the reference turns into an undefined index, is held at the first node
    const int mm3 = (mm2 == 11 || mm2 == 12 || mm2 == 31 || mm2 == 32) ? 1 : 0;
    double e = (mtk - D.tkmin) / D.tkstp;
    if (e < 0) e = 0;
    if (e > (double)(D.tknum - 1)) e = (double)(D.tknum - 1);
    double n = (mpb - D.pbmin) / D.pbstp;
    if (n < 0) n = 0;
    if (n > (double)(D.pbnum - 1)) n = (double)(D.pbnum - 1);
    int n1 = (e == e) ? (int)e : 0;
    if (n1 > D.tknum - 2) n1 = D.tknum - 2;
    int n2 = (n == n) ? (int)n : 0;
    if (n2 > D.pbnum - 2) n2 = D.pbnum - 2;
    e = e - (double)n1;
    n = n - (double)n2;
    const double2 *q = D.rh + ((int64_t)mm3 * D.tknum + n1) * D.pbnum + n2;
    const double2 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + D.pbnum), q3 = __ldg(q + D.pbnum + 1);
    const double R0 = q0.x, R1 = q1.x, R2 = q2.x, R3 = q3.x;
    const double H0 = q0.y, H1 = q1.y, H2 = q2.y, H3 = q3.y;
    // markmart.c:2155-2176
    double mro = ((R0 * (1.0 - n) + R1 * n) * (1.0 - e) + (R2 * (1.0 - n) + R3 * n) * e);
    double mcp = ((H2 - H0) * (1.0 - n) + (H3 - H1) * n) / D.tkstp;
    if (mcp < 1e+2) mcp = 1e+2;
    else if (mcp > 5e+4) mcp = 5e+4;
    double mbb = (2.0 / (R1 + R0) - (H1 - H0) / D.pbstp / 1e+5) * (1.0 - e) +
                 (2.0 / (R3 + R2) - (H3 - H2) / D.pbstp / 1e+5) * e;
    mbb *= mro / mtk;
    if (mbb < -1e-2) mbb = -1e-2;
    else if (mbb > 1e-2) mbb = 1e-2;
    double mkt = mkt1 + krad;
    // partially molten rock (markmart.c:2178-2235)
    const SiCurve c0 = si_at(mpb, mm2, D.si_melting, D.exact);
    const double xm = c0.frac(mtk);
    int nt = mm2;
    if (xm > 0 && mm2 < 20) nt = mm2 + 20;
    if (xm <= 0 && mm2 > 20) nt = mm2 - 20;
    if (nt > 20) {
        mro = mro * (1.0 - xm) +
              xm * T.markro[nt] * (1.0 - T.markbb[nt] * (mtk - 298.15)) * (1.0 + T.markaa[nt] * (mpb - 1.0) * 1e-3);
        if (xm > 0.1) {
            // Pinkerton & Stevenson (1992) eq. 5, clamped
            double nueff = T.marknu[nt] * exp((2.500 + pow(((1.000 - xm) / xm), 0.480)) * (1.000 - xm));
            if (nueff < T.markn0[nt]) nueff = T.markn0[nt];
            if (nueff > T.markn1[nt]) nueff = T.markn1[nt];
            if (nueff < nubeg) nueff = nubeg;
            if (nueff > nuend) nueff = nuend;
            mnu = nueff;
        }
        // exp(0 x mpb) is 1 exactly for a finite pressure: skip the call there
        const bool fin = isfinite(mpb);
        const double e1 = (T.markkp[nt] == 0.0 && fin) ? 1.0 : exp(T.markkp[nt] * mpb);
        const double e0 = (T.markkp[nt - 20] == 0.0 && fin) ? 1.0 : exp(T.markkp[nt - 20] * mpb);
        mkt = ((T.markkt[nt] + T.markkf[nt] / (mtk + 77.0)) * e1) * xm +
              ((T.markkt[nt - 20] + T.markkf[nt - 20] / (mtk + 77.0)) * e0) * (1.0 - xm);
        if (xm > 0 && xm < 1.0) {
            // latent heat by central differences: -ro dH/dP / T and dH/dT
            const double dmpb = mpb * 0.001;
            double ival = si_at(mpb - dmpb, nt, D.si_melting, D.exact).latent(mtk) -
                          si_at(mpb + dmpb, nt, D.si_melting, D.exact).latent(mtk);
            ival *= mro / (mtk * 2.0 * dmpb * 1e+5);
            mbb += ival;
            ival = c0.latent(mtk + 1.0) - c0.latent(mtk - 1.0);
            ival /= 2.0 * 1.0;
            mcp += ival;
        }
    }
    // water ice of type 6 (markmart.c:2237-2268)
    if (nt == 6) {
        const double xi = ice_melt(mtk, mpb, 6, D.ice_melting, D.exact, nullptr);
        if (xi > 0 && xi < 1.0) {
            const double dmpb = mpb * 0.001;
            double lo, hi;
            ice_melt(mtk, mpb - dmpb, 6, D.ice_melting, D.exact, &lo);
            ice_melt(mtk, mpb + dmpb, 6, D.ice_melting, D.exact, &hi);
            double ival = lo - hi;
            ival *= mro / (mtk * 2.0 * dmpb * 1e+5);
            mbb += ival;
            ice_melt(mtk + 1.0, mpb, 6, D.ice_melting, D.exact, &hi);
            ice_melt(mtk - 1.0, mpb, 6, D.ice_melting, D.exact, &lo);
            ival = hi - lo;
            ival /= 2.0 * 1.0;
            mcp += ival;
        }
    }
    mro_o = mro;
    mcp_o = mcp;
    mbb_o = mbb;
    mkt_o = mkt;
    return nt;
}

// The eps[] state tdbasecalc leaves for the table marker at (mtk, mpb, type mm2):
// its last meltpart1 call is at (mtk - 1, mpb) when a type-6 marker's ice is
// partly molten (markmart.c:2263), else at (mtk, mpb) with the new type
// (markmart.c:2237).  out[] (optional) = eps[21], 22, 50, 51, 52, 53.  Returns eps[21].
static __device__ __noinline__ double td_last_melt(const TdArgs &D, double mtk, double mpb, int mm2, double *out)
{
    const SiCurve c0 = si_at(mpb, mm2, D.si_melting, D.exact);  // the flip keeps the curve's class
    const double xm = c0.frac(mtk);
    int nt = mm2;
    if (xm > 0 && mm2 < 20) nt = mm2 + 20;
    if (xm <= 0 && mm2 > 20) nt = mm2 - 20;
    double t = mtk;
    if (nt == 6) {
        const double xi = ice_melt(mtk, mpb, 6, D.ice_melting, D.exact, nullptr);
        if (xi > 0 && xi < 1.0) t = mtk - 1.0;
    }
    const double si = c0.frac(t);
    if (out) {
        out[0] = si;
        out[1] = c0.latent(t);
        out[2] = 0.0;  // meltpart1's iron fractions: zero for every table type
        out[3] = 0.0;
        out[4] = ice_melt(t, mpb, nt, D.ice_melting, D.exact, &out[5]);
    }
    return si;
}

// eps[21] and eps[50] as a marker reads them (markmart.c:287-288): left by the
// table marker before it in the caller's order, else the state the call began with
__device__ __forceinline__ void td_prev_melt(const TdArgs &D, int32_t id, double &xsi, double &xfe)
{
    const int32_t p = id > 0 ? __ldg(D.prev + id - 1) : -1;
    if (p >= 0) {
        xsi = __ldg(D.si + p);
        xfe = 0.0;
    } else {
        xsi = __ldg(D.melt_in + 0);
        xfe = __ldg(D.melt_in + 2);
    }
}

// The table markers of a call, one thread per storage slot: flag[id] = id for a
// table marker (the filter of markmart.c:277 and the types of markmart.c:482),
// else -1; si[id] = the eps[21] it leaves (td_last_melt) at the pressure the
// averaging interpolates for it (allintere, markmart.c:281).
template <bool MIXED>
__global__ void __launch_bounds__(256) k_td_melt(const __grid_constant__ GridView G,
                                                 const __grid_constant__ MarkerView A,
                                                 const __grid_constant__ TdArgs D, int32_t gridmod,
                                                 int32_t *__restrict__ flag, double *__restrict__ si)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const int32_t id = A.id[i];
    const int mt = A.type[i];
    const double x = A.x[i], y = A.y[i], Tm = A.T[i];
    const bool ok = (gridmod <= 1 || (id % gridmod) == 0) && td_type(mt) && x > 0 && y > 0 && x < G.xsize &&
                    y < G.ysize && Tm > 0;
    if (ok) {
        double pr, ga, e[6];
        int64_t m10, m20;
        interp_e<MIXED>(G, x, y, pr, ga, false, false, e, m10, m20);
        si[id] = td_last_melt(D, Tm, pr * 1.0000e-5, mt, nullptr);
    }
    flag[id] = ok ? id : -1;
}

// the eps[] state after the call, from the last table marker (markmart.c:2237-2275)
static __device__ __noinline__ void td_write_state(const TdArgs &D, double mtk, double mpb, int mm2)
{
    double out[6];
    td_last_melt(D, mtk, mpb, mm2, out);
    for (int k = 0; k < 6; k++) D.melt_out[k] = out[k];
}

}  // namespace i2g
