// Magnetisation of solid silicates below the Curie temperatures of magnetite
// (851.16 K) and hematite (948.16 K), markmart.c:651-744.
//
// Per processed marker of ronurecalc(): the state (0 none, 1 hematite, 2
// magnetite and hematite, 3 cannot magnetise) from the rock type, temperature,
// the previous state and the dynamo switch; and the magnetisation time, which
// the reference keeps in a local variable (mag_time) that only some branches
// assign: a marker that assigns none stores the value the last assigning marker
// before it left.  The device keeps that order-dependence the way it keeps the
// melt state of the table path: per caller index the value a marker assigns,
// an inclusive max-scan over the caller indices of the assigning markers, and
// the averaging reads its predecessor's value (or the call's carried one).
#pragma once

#include "i2g_dev.cuh"

namespace i2g {

// The new state of a marker of type mm2 at temperature mtk with previous state
// old; assigns: whether the branch taken sets mag_time, to val.
__device__ __forceinline__ int mag_state(int dynamo, int mm2, double mtk, int old, double timesum, bool &assigns,
                                         double &val)
{
    constexpr double kMa = 3600.000 * 24.000 * 365.250 * 1.000e+6;  // seconds per Myr
    int mag = 3;
    assigns = false;
    val = 0.0;
    const bool sil = mm2 == 5 || mm2 == 6;
    if (dynamo == 0) {
        if (sil) {
            if (mtk <= 851.16 && old == 2) mag = 2;
            else if ((mtk > 851.16 && mtk <= 948.16) && old == 2) mag = 1;
            else if (mtk <= 851.16 && old == 1) mag = 1;
            else if ((mtk > 851.16 && mtk <= 948.16) && old == 1) mag = 1;
            else if (mtk > 948.16) { mag = 0; assigns = true; val = -1.000; }
        } else {  // mm2 < 5 || mm2 > 6: never magnetised, time reset
            mag = 3;
            assigns = true;
            val = -1.000;
        }
    } else if (dynamo == 1) {
        if (sil) {
            if (mtk <= 851.16) {
                mag = 2;
                if (old <= 1 || old == 3) { assigns = true; val = timesum / kMa; }
            } else if (mtk > 851.16 && mtk <= 948.16) {
                mag = 1;
                if (old == 0 || old == 3) { assigns = true; val = timesum / kMa; }
            } else if (mtk > 948.16) {
                mag = 0;
                assigns = true;
                val = -1.000;
            }
        } else {
            mag = 3;
            assigns = true;
            val = -1.000;
        }
    }
    return mag;
}

// the magnetisation time a marker stores: its own assignment, else that of the
// last assigning marker before it in the caller's order, else the call's carried one
__device__ __forceinline__ double mag_time_of(const AvgArgsK &A, int32_t id, bool assigns, double val)
{
    if (assigns) {
        if (id == __ldg(A.mag_last)) *A.mag_out = val;
        return val;
    }
    const int32_t p = id > 0 ? __ldg(A.mag_prev + id - 1) : -1;
    return p >= 0 ? __ldg(A.mag_val + p) : __ldg(A.mag_in);
}

}  // namespace i2g
