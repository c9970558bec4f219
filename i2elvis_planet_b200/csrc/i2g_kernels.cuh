// Marker-step kernels, templated on the precision form (see i2g_dev.cuh).
//
//   k_move     movemark() per marker (markmart.c:23-155): pressure gather at the
//              old position, optional viscalc, RK4 through the staggered velocity,
//              orthogonal-only motion outside the box, out-of-box T reset; writes
//              the marker's new cell key for the next sort.
//   marker_contrib  one marker of the ronurecalc() loop (markmart.c:277-855): the
//              property model and the marker's bilinear weights; the streaming
//              averaging kernel (i2g_avg.cuh) sums these per cell and per node.
#pragma once

#include "i2g_dev.cuh"
#include "i2g_td.cuh"
#include "i2g_mag.cuh"

namespace i2g {

// cell-corner partial sums: 4 corners x {ro, et, cp, kt, ht, w0, tk, w1, nu, wnu}
// + cell-centre {nd, wnd}; stored field-major [kPart][ncells]
constexpr int kPart = 42;
// the averaging takes rock types below 50 only (markmart.c:277)
constexpr int kAvgTypes = 50;
enum { F_RO = 0, F_ET, F_CP, F_KT, F_HT, F_W0, F_TK, F_W1, F_NU, F_WNU };


__device__ __forceinline__ double radcoef(const AvgArgsK &A, int mt)
{
    if (mt == 5 || mt == 6 || mt == 25 || mt == 26) return A.rad_si;
    if (mt == 7 || mt == 8 || mt == 9 || mt == 10 || mt == 17 || mt == 18 || mt == 19) return A.rad_fe;
    if (mt == 15) return A.rad_ch;
    return 0.0;
}


// Markers further than 0.95 xsize / 2 from the box centre get eta = 1e22
// (markmart.c:268, 335-340; pow(., 0.5) there, an exact threshold on the square here)
__device__ __forceinline__ bool outside_radmax(const GridView &G, const AvgArgsK &A, double x, double y)
{
    const double celdx = x - G.xsize / 2.0, celdy = y - G.ysize / 2.0;
    return celdx * celdx + celdy * celdy >= A.rad2;
}

// ----------------------------------------------------------------- movemark
// the viscosity update of movemark() (markmart.c:46-68) from the strain rates and
// stresses e[] (exy, sxy, exx, sxx, eyy, syy) and the pressure at the marker
__device__ __forceinline__ void visc_update(const MarkerView &M, const i2g_types &T, const MoveArgs &A, int64_t i,
                                            int mt, double pr, const double *e)
{
    const double Tm = M.T[i];
    if (mt < 50 && Tm > 0) {
        double eii, sii;
        invariants(e, eii, sii);
        double rii = 1.0;
        const double et = M.eta[i];
        if (et > 0) rii *= pow(0.5 * sii / eii / et, 0.87);
        M.eta[i] = viscalc(T, Tm, pr * 1e-5, M.hi ? M.hi[i] : 0.0, eii, sii, rii, A.timesum, A.relax_time, A.nubeg,
                           A.nuend, mt < 20 ? mt : mt - 20);
    }
}

// One marker of movemark() (markmart.c:23-155); returns the marker's new cell.
template <bool MIXED, bool VISC>
__device__ __forceinline__ int32_t move_marker(const GridView &G, const MarkerView &M, const i2g_types &T,
                                               const MoveArgs &A, int32_t *__restrict__ key, int64_t i)
{
    const int mt = M.type[i];
    double x = M.x[i], y = M.y[i];
    const bool inbox = (x >= 0 && y >= 0 && x <= G.xsize && y <= G.ysize);
    int hx = -1, hy = -1;  // the marker's cell at the start of the step (mixed form)
    if ((inbox || A.outgrid != 1) && !T.markim[mt]) {
        double pr, vx0, vy0;
        const double dt = A.timestep;
        if (MIXED) {
            // pressure and the first RK4 velocity share one stencil evaluation; the
            // later stages run in FP32 offsets from the first stage's cell, and the
            // new cell key searches from that cell.  The strain rates and stresses
            // of the viscosity update come from the first stage's stencils too.
            AxisF X1, Y1;
            rk4_mixed(G, x, y, dt, A.markmod, vx0, vy0, &pr, hx, hy, VISC ? &X1 : nullptr, VISC ? &Y1 : nullptr);
            M.p[i] = pr;
            if (VISC) {
                double e[6];
                strain_mixed(G, x, y, X1, Y1, e);
                visc_update(M, T, A, i, mt, pr, e);
            }
        } else {
            double ga, e[6];
            int64_t c1, c2;
            interp_e<MIXED>(G, x, y, pr, ga, false, VISC, e, c1, c2);
            M.p[i] = pr;
            if (VISC) visc_update(M, T, A, i, mt, pr, e);
            if (A.markmod == 1) {
                interp_v<MIXED>(G, x, y, vx0, vy0);
            } else {
                double vx1, vy1, vx2, vy2, vx3, vy3, vx4, vy4;
                interp_v<MIXED>(G, x, y, vx1, vy1);
                interp_v<MIXED>(G, x + vx1 * dt / 2.0, y + vy1 * dt / 2.0, vx2, vy2);
                interp_v<MIXED>(G, x + vx2 * dt / 2.0, y + vy2 * dt / 2.0, vx3, vy3);
                interp_v<MIXED>(G, x + vx3 * dt, y + vy3 * dt, vx4, vy4);
                vx0 = (vx1 + 2.0 * vx2 + 2.0 * vx3 + vx4) / 6.0;
                vy0 = (vy1 + 2.0 * vy2 + 2.0 * vy3 + vy4) / 6.0;
            }
        }
        if (A.outgrid == 2) {
            if (x < 0 || x > G.xsize) vy0 = 0;
            if (y < 0 || y > G.ysize) vx0 = 0;
        }
        x = advance(x, dt, vx0, A.f32pos);
        y = advance(y, dt, vy0, A.f32pos);
        M.x[i] = x;
        M.y[i] = y;
        if (x < 0 || y < 0 || x > G.xsize || y > G.ysize) M.T[i] = 0;
    }
    const int32_t k = cell_key(G, x, y, hx, hy);
    key[i] = k;
    return k;
}

// sub: the marker's arrival index in its new cell (the count before it), so the
// sort places it at cstart[key] + sub without atomics of its own
template <bool MIXED, bool VISC>
__global__ void __launch_bounds__(256) k_move(const __grid_constant__ GridView G, const __grid_constant__ MarkerView M,
                                              const DevTypes *__restrict__ Ty, const __grid_constant__ MoveArgs A,
                                              int32_t *__restrict__ key, int32_t *__restrict__ count,
                                              int32_t *__restrict__ sub)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M.n; i += stride) {
        const int32_t k = move_marker<MIXED, VISC>(G, M, Ty->t, A, key, i);
        // per-cell counts for the next sort (warp-aggregated integer atomics: exact)
        const unsigned peers = __match_any_sync(__activemask(), k);
        const int leader = __ffs(peers) - 1, lane = (int)(threadIdx.x & 31);
        int32_t base = 0;
        if (lane == leader) base = atomicAdd(count + k, __popc(peers));
        base = __shfl_sync(peers, base, leader);
        sub[i] = base + __popc(peers & ((1u << lane) - 1u));
    }
}

// ----------------------------------------------------------------- ronurecalc, marker side
// Conductivity of molten silicate / iron (markmart.c:509-610), soft-turbulence model.
__device__ __forceinline__ double molten_k(const i2g_types &T, int mm2, double mkt, double Tm, double T0,
                                           double mro, double mga, double mcp, double mnu, double eta_fluid)
{
    double heat_flux = 0.089 * pow(T.markkt[mm2], (2.000 / 3.000)) * pow(fabs(Tm - T0), (4.000 / 3.000)) *
                       pow((mro * mro * T.markbb[mm2] * mga * mcp / eta_fluid), (1.000 / 3.000));
    if (heat_flux <= 0.0001) return T.markkt[mm2];
    if (heat_flux > 0.0001)
        return pow((heat_flux / 0.089), (3.000 / 2.000)) / (pow((Tm - T0), 2.000) * mro) *
               pow((T.markbb[mm2] * mga * mcp / mnu), (-1.000 / 2.000));
    return mkt;  // NaN heat flux leaves mkt unchanged, as the reference's if/else-if does
}

// The rarely taken branches of the averaging's property model live out of line
// so that the common path keeps few registers (and the averaging kernel its
// occupancy): the pressure gather with viscalc, the molten-material
// conductivity and the porous-silicate conductivity.

// allintere() (markmart.c:281) and, for markers without a viscosity, viscalc()
template <bool MIXED>
__device__ __noinline__ void pressure_visc(const GridView &G, const i2g_types &T, const AvgArgsK &A, double x,
                                           double y, double mtk, double hi, int mt, bool molten, bool needvisc,
                                           double &pr, double &mga, double &mnu, int64_t &m10, int64_t &m20)
{
    double e[6];
    interp_e<MIXED>(G, x, y, pr, mga, molten, needvisc, e, m10, m20);
    if (needvisc) {
        double eii, sii;
        invariants(e, eii, sii);
        mnu = viscalc(T, mtk, pr * 1.0000e-5, hi, eii, sii, 1.0, A.timesum, A.relax_time, A.nubeg, A.nuend,
                      mt < 20 ? mt : mt - 20);
    }
}

// conductivity of molten silicate / iron by melt fraction (markmart.c:509-610);
// the melt fractions are eps[21] / eps[50] as the marker reads them (markmart.c:287-288)
static __device__ __noinline__ double molten_branch(const i2g_types &T, const AvgArgsK &A, int32_t id, int mm2,
                                                    double mkt, double mtk, double T0, double mro, double mga,
                                                    double mcp, double mnu)
{
    double xm = A.xmelt_si, xfe = A.xmelt_fe;
    if (A.densimod == 2) td_prev_melt(A.td, id, xm, xfe);
    if (mm2 == 25 || mm2 == 26) {
        if (xm >= 0.4000 && xm <= 0.6000)
            mkt = molten_k(T, mm2, mkt, mtk, T0, mro, mga, mcp, mnu, T.markn0[mm2] * exp((-172.690) * (xm - 0.400)));
        if (xm > 0.6000) mkt = molten_k(T, mm2, mkt, mtk, T0, mro, mga, mcp, mnu, 100.0000);
    } else {
        if (xfe < 1.0000) mkt = molten_k(T, mm2, mkt, mtk, T0, mro, mga, mcp, mnu, 1.0000e12);
        if (xfe == 1.0000) mkt = molten_k(T, mm2, mkt, mtk, T0, mro, mga, mcp, mnu, 0.010);
    }
    return mkt;
}

// the table types of densimod 2 (markmart.c:481-493): tdbasecalc's values replace
// the density, heat capacity, expansion term, conductivity and viscosity; the
// marker's type flips with its melt; the call's last table marker leaves the
// melt state
static __device__ __noinline__ int td_branch(const i2g_types &T, const AvgArgsK &A, int32_t id, int mm2,
                                             double mtk, double mpb, double &mro, double &mcp, double &mbb,
                                             double &mkt, double &mnu)
{
    const int nt = td_props(A.td, T, A.nubeg, A.nuend, mtk, mpb, mm2, mro, mcp, mbb, mkt, mnu);
    if (id == __ldg(A.td.last)) td_write_state(A.td, mtk, mpb, mm2);
    return nt;
}

// conductivity of porous solid silicate, porosity > 0 (markmart.c:614-638)
static __device__ __noinline__ double porous_k(const i2g_types &T, int mm2, double mpor, double mkt)
{
    if (mpor < 0.200) mkt = T.markkt[mm2] * exp(-mpor / 0.080);
    if (mpor >= 0.200 && mpor <= 0.400)
        mkt = pow((pow((T.markkt[mm2] * exp(-mpor / 0.080)), 4.000) +
                   pow((T.markkt[mm2] * exp(-1.200 - (mpor / 0.167))), 4.000)),
                  0.250);
    if (mpor > 0.400) mkt = T.markkt[mm2] * exp(-1.200 - (mpor / 0.167));
    return mkt;
}

// Cold pressing and hot sintering of porous solid silicate (markmart.c:362-466;
// Henke et al. 2012, Schwenn & Goetze 1978) for a type 5/6 marker with porosity
// in (0, 0.85] at pressure mpb (bar) and temperature mtk.  The grain-size search
// restarts from a larger guess while its Newton iteration has not settled
// (markmart.c:426-432, an unbounded goto there); after kSinterTries restarts the
// marker keeps its porosity and the call's counter records it.
constexpr int kSinterTries = 64;
static __device__ __noinline__ double sinter(const AvgArgsK &A, double mpb, double mtk, double por)
{
    const double p_ref = 0.130, grain_orig = 1.000e-6, pivalue = 3.141592654;
    const double E_act = 85000.000, fact_a = 4.000e-5, r_gas = 1.9872;
    const bool f32 = A.f32por != 0;
    if (mtk < 700.000) {  // cold pressing: porosity only decreases (eq. 15)
        const double lim = (0.420 + 0.460 * pow((pow((mpb / p_ref), 1.720) + 1.000), (-1.000)));
        por = por <= lim ? por : lim;
        if (f32) por = (double)(float)por;
        por = por <= 0.850 ? por : 0.850;
        if (f32) por = (double)(float)por;
    }
    if (mtk >= 700.000) {  // hot sintering (eqs. 34-44)
        const double lim = (0.420 + 0.460 * pow((pow((mpb / p_ref), 1.720) + 1.000), (-1.000)));
        double por_orig = A.por_init <= lim ? A.por_init : lim;
        por_orig = por_orig <= 0.850 ? por_orig : 0.850;
        const double k = pow(((1.000 - por_orig) / (1.000 - por)), (1.000 / 3.000));
        double guess = grain_orig, old = 0.0;
        int n_count = 1;
        for (;;) {
            for (int it = 1; it < 100; it++) {
                old = guess;
                const double funct = pow(guess, 3.000) + pow(grain_orig, 3.000) - 3.000 * pow(guess, 2.000) * grain_orig * k +
                                     pow(grain_orig, 3.000) * (1.000 - por_orig) / (1.000 - por);
                const double drv = 3.000 * pow(guess, 2.000) - 6.000 * guess * grain_orig * k;
                guess = old - (funct / drv);
            }
            const double d = guess - old;
            const double err = d >= 0 ? d : -d;
            if ((err > 5.000e-2) || (guess <= grain_orig)) {
                if (++n_count > kSinterTries) {
                    if (A.sinter_stuck) atomicAdd(A.sinter_stuck, 1u);
                    return por;
                }
                guess = 1.250 * (double)n_count * grain_orig;
                continue;
            }
            break;
        }
        const double grain_corr = guess > grain_orig ? guess : 0.0;
        const double cont_r = sqrt(pow(grain_corr, 2.000) -
                                   pow(grain_orig, 2.000) * pow(((1.000 - por_orig) / (1.000 - por)), (2.000 / 3.000)));
        const double c_fact = 2.000 * sqrt(3.000) * (pow(grain_corr, 2.000) - pow(cont_r, 2.000));
        const double grain_stress = c_fact * mpb / (pivalue * pow(cont_r, 2.000));
        double por_change = 0.000;
        if (por > 0.100)
            por_change = fact_a * (1.000 - por) * pow(grain_stress, 1.500) / pow((100.000 * grain_corr), 3.000) *
                         exp(-E_act / (r_gas * mtk)) * A.timestep;
        if (por <= 0.100)
            por_change = 10.000 * por * fact_a * (1.000 - por) * pow(grain_stress, 1.500) /
                         pow((100.000 * grain_corr), 3.000) * exp(-E_act / (r_gas * mtk)) * A.timestep;
        if (por_change > 0.000) {
            por = por - por_change;
            if (f32) por = (double)(float)por;
        }
    }
    return por;
}

// Natural log for the mixed form: the binary exponent exactly, the log of the
// mantissa in [1, 2) with the FP32 log2f, combined in FP64.  Absolute error about
// 1e-7, i.e. about 1e-7 relative in a node viscosity exp(mean log).  Zero,
// negative, subnormal and non-finite arguments take the FP64 log.
__device__ __forceinline__ double log_mixed(double v)
{
    const long long bits = __double_as_longlong(v);
    const int ex = (int)((bits >> 52) & 0x7ff);
    if (!(v > 0.0) || ex == 0 || ex == 0x7ff) return log(v);
    const double m = __longlong_as_double((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
    return ((double)(ex - 1023) + (double)log2f((float)m)) * 0.69314718055994530942;
}

struct MarkerContrib {
    double wx0, wx1, wy0, wy1;
    double mro, mbb, mcp, mkt, mht, mtk, lnu;
    bool immobile;
};

// one marker's state as the averaging reads and updates it
struct MarkerRec {
    double x, y, T, eta, p, tmax, hi, por;
    int type;
    int32_t id;
    int mgo;     // magnetisation state and time, when produced
    double mgt;
};

// One marker of the ronurecalc loop (markmart.c:277-855).  Returns false when the
// marker fails the filter of markmart.c:277.  Updates the marker side effects in
// the record (sticky-air T, marktmax, porosity clamp).  (c1, c2) is the marker's
// cell, which the cell sort has already found with the reference's search.
template <bool MIXED>
__device__ __forceinline__ bool marker_contrib(const GridView &G, const i2g_types &T, const AvgArgsK &A,
                                              double T0, MarkerRec &r, bool has_tmax, bool has_por,
                                              int64_t c1, int64_t c2, MarkerContrib &c)
{
    const double x = r.x, y = r.y;
    double Tm = r.T;
    const int mt = r.type;
    if (!(x > 0 && y > 0 && x < G.xsize && y < G.ysize && Tm > 0 && mt < kAvgTypes)) return false;
    const int mm2 = mt;
    const double eta = r.eta;
    const bool needvisc = eta <= 0;
    const bool molten = (A.timesum > A.core_form_time) &&
                        (mm2 == 25 || mm2 == 26 || mm2 == 7 || mm2 == 8 || mm2 == 9 || mm2 == 10 || mm2 == 17 ||
                         mm2 == 18 || mm2 == 19);
    // allintere() (markmart.c:281) feeds only viscalc, dencalc (densimod 1), the
    // pressure factor of the conductivity and the molten-material branches; when
    // none of them reads it the gather is skipped (the cell is the sort cell).
    const bool porous = has_por && (mm2 == 5 || mm2 == 6) && r.por > 0.000 && r.por <= 0.850;
    const bool need_p = needvisc || molten || porous || A.densimod != 0 || T.markkp[mm2] != 0.0;
    // sticky air held at the ambient temperature (markmart.c:296-309)
    if (mm2 < 2) Tm = A.tmp_ambient;
    r.T = Tm;
    const double mtk = Tm;
    double pr = 0.0, mga = 0.0, mnu = eta;
    int64_t m10 = c1, m20 = c2;
    if (need_p) pressure_visc<MIXED>(G, T, A, x, y, mtk, r.hi, mt, molten, needvisc, pr, mga, mnu, m10, m20);
    const double mpb = pr * 1.0000e-5;
    if (outside_radmax(G, A, x, y)) mnu = 1.000e+22;
    // porosity and maximum temperature (markmart.c:347-360, 462-472)
    double mpor = has_por ? r.por : 0.0;
    if (mm2 == 0 || mm2 >= 7) mpor = 0.0;
    if (has_tmax && mt != 0 && r.tmax < mtk) r.tmax = mtk;
    if (porous) mpor = sinter(A, mpb, mtk, mpor);  // markmart.c:362-466
    if (mpor < 0.000) mpor = 0.000;
    if (mpor > 1.000) mpor = 1.000;
    if (has_por) r.por = mpor;
    // density (dencalc, markmart.c:1024-1046), heat capacity, conductivity (markmart.c:475-478)
    double mro, mbb = 0;
    if (A.densimod == 0) {
        mro = T.markro[mm2];
    } else {
        mro = T.markro[mm2] * (1.0 - T.markbb[mm2] * (mtk - 298.15)) * (1.0 + T.markaa[mm2] * (mpb - 1.0) * 1e-3) *
              (1.000 - mpor);
        mbb = T.markbb[mm2] / (1.0 - T.markbb[mm2] * (mtk - 298.15));
    }
    double mcp = T.markcp[mm2];
    double mkt = T.markkt[mm2];
    if (T.markkf[mm2] != 0.0) mkt += T.markkf[mm2] / (mtk + 77.0);  // 0/(T+77) adds exactly 0
    if (T.markkp[mm2] != 0.0) mkt *= exp(T.markkp[mm2] * mpb);  // exp(0) == 1 exactly
    if (A.densimod == 2 && td_type(mm2)) r.type = td_branch(T, A, r.id, mm2, mtk, mpb, mro, mcp, mbb, mkt, mnu);
    if (molten) mkt = molten_branch(T, A, r.id, mm2, mkt, mtk, T0, mro, mga, mcp, mnu);
    // porosity-dependent conductivity of solid silicates (markmart.c:614-638)
    if (mm2 == 5 || mm2 == 6) mkt = (mpor == 0.0) ? T.markkt[mm2] : porous_k(T, mm2, mpor, mkt);
    if (mkt <= 0.0010) mkt = 0.0010;
    if (mkt >= A.k_cutoff) mkt = A.k_cutoff;
    // magnetisation state and time (markmart.c:651-744)
    if (A.mag_prev) {
        bool as;
        double v;
        r.mgo = mag_state(A.dynamo, mm2, mtk, r.mgo, A.timesum, as, v);
        r.mgt = mag_time_of(A, r.id, as, v);
    }
    // weights of the marker's cell at its position (nodewt(...,0,0), markmart.c:848-855)
    if (!MIXED) {
        fdw64(__ldg(G.gx + m10), __ldg(G.gx + m10 + 1), x, c.wx0, c.wx1);
        fdw64(__ldg(G.gy + m20), __ldg(G.gy + m20 + 1), y, c.wy0, c.wy1);
    } else {
        float a0, a1, b0, b1;
        fdw32(__ldg(G.gx + m10), __ldg(G.ixb + m10), x, a0, a1);
        fdw32(__ldg(G.gy + m20), __ldg(G.iyb + m20), y, b0, b1);
        c.wx0 = a0; c.wx1 = a1; c.wy0 = b0; c.wy1 = b1;
    }
    c.mro = mro;
    c.mbb = mbb;
    c.mcp = mcp;
    c.mkt = mkt;
    c.mht = radcoef(A, mm2) * mro;
    c.mtk = mtk;
    c.lnu = A.viscmod == 1 ? (MIXED ? log_mixed(mnu) : log(mnu)) : (A.viscmod == 2 ? 1.0 / mnu : mnu);
    c.immobile = T.markim[mm2] != 0;
    return true;
}

}  // namespace i2g
