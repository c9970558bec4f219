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

struct TdArgs {
    // (density kg/m^3, enthalpy J/kg) per [database][tk][pb] node: the
    // reference's td[tk][pb][db][0] * 1000.0 and td[tk][pb][db][1] * 1000.0 * 4.1837
    // (markmart.c:2147-2154), products formed once on the host in that order
    const double2 *rh;
    double tkmin, pbmin, tkstp, pbstp;
    int32_t tknum, pbnum;
    int32_t si_melting, ice_melting;
    const int32_t *prev;    // inclusive max-scan of the table markers' caller indices (-1: none yet)
    const double *si;       // eps[21] each table marker leaves, by caller index
    const double *melt_in;  // eps[21], eps[22], eps[50], eps[51], eps[52], eps[53] before the call
    double *melt_out;       // the same after it: written by the last table marker
};

__host__ __device__ __forceinline__ bool td_type(int t)
{
    return t == 5 || t == 6 || t == 11 || t == 12 || t == 25 || t == 26 || t == 31 || t == 32;
}

// Silicate solidus, liquidus and latent heat of a table type (markmart.c:2352-2412)
__device__ __forceinline__ void si_curve(double mpb, int mm2, int si_melting, double &ts, double &tl, double &hl)
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
        if (mpb < 21.50e+4)
            ts = 273.15 + 1143.04342 + 58.2946423e-4 * mpb + 52.3439318e-8 * mpb * mpb -
                 16.3201032e-12 * mpb * mpb * mpb + 2.29886314e-16 * pow(mpb, 4.000) -
                 0.180865486e-20 * pow(mpb, 5.000) + 0.00815679773e-24 * pow(mpb, 6.000) -
                 0.000197104325e-28 * pow(mpb, 7.000) + 1.97908526e-38 * pow(mpb, 8.000);
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

__device__ __noinline__ double si_melt(double mtk, double mpb, int mm2, int si_melting, double *latent)
{
    double ts, tl, hl;
    si_curve(mpb, mm2, si_melting, ts, tl, hl);
    const double x = si_frac(mtk, ts, tl);
    if (latent) *latent = (tl != 0.0) ? hl * x : 0.0;
    return x;
}

// Water-ice melting of type 6 (Dunaeva et al. 2010, markmart.c:2414-2460) with the
// 10 K gap between onset and full melting; ts = tl = 0 outside the fitted range
__device__ __forceinline__ void ice_curve(double mpb, double &ts, double &tl)
{
    const double t_shift = 10.000;
    ts = 0.0;
    tl = 0.0;
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
__device__ __noinline__ double ice_melt(double mtk, double mpb, int mm2, int ice_melting, double *latent)
{
    double x = 0.0, h = 0.0;
    if (mm2 == 6 && ice_melting == 1) {
        double ts, tl;
        ice_curve(mpb, ts, tl);
        if (tl != 0.0 || tl != tl) {  // the reference's "if(tl_ice)": NaN is true
            x = (mtk - ts) / (tl - ts);
            if (x < 0.000) x = 0.0000;
            if (x > 1.000) x = 1.0000;
            h = (284000.0 + 233000.0) * 0.3 * x;
        }
    }
    if (latent) *latent = h;
    return x;
}
