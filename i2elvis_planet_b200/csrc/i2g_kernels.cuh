// Marker-step kernels, templated on the precision form (see i2g_dev.cuh).
//
//   k_move     movemark() per marker (markmart.c:23-155): pressure gather at the
//              old position, optional viscalc, RK4 through the staggered velocity,
//              orthogonal-only motion outside the box, out-of-box T reset; writes
//              the marker's new cell key for the next sort.
//   k_cellsum  the ronurecalc() marker loop (markmart.c:271-913), one thread per
//              cell over that cell's markers (cell-sorted, ascending caller index):
//              property model + 2x2 bilinear and quadrant weights, summed per
//              cell corner in FP64 registers.
//   k_nodesum  the node loop (markmart.c:917-993): each node adds the corner sums
//              of its four cells in a fixed order, normalises, takes exp()/inverse
//              per viscmod, applies mu[] and the [nubeg, nuend] clamp and reduces
//              the viscosity range per block.
//   k_clamp    contrast limit (markmart.c:995-1009).
// Node sums are deterministic and use no global atomics: every node's value is a
// fixed-order reduction over fixed-order cell sums.
#pragma once

#include "i2g_dev.cuh"

namespace i2g {

// cell-corner partial sums: 4 corners x {ro, et, cp, kt, ht, w0, tk, w1, nu, wnu}
// + cell-centre {nd, wnd}; stored field-major [kPart][ncells]
constexpr int kPart = 42;
enum { F_RO = 0, F_ET, F_CP, F_KT, F_HT, F_W0, F_TK, F_W1, F_NU, F_WNU };

struct AvgArgsK {
    double timesum, tmp_ambient, core_form_time, k_cutoff, relax_time, nubeg, nuend;
    double xmelt_si, xmelt_fe;
    double rad_si, rad_fe, rad_ch;  // radiogenic heating per kg, markmart.c:749-837
    int32_t gridmod, densimod, viscmod;
};

__device__ __forceinline__ double radcoef(const AvgArgsK &A, int mt)
{
    if (mt == 5 || mt == 6 || mt == 25 || mt == 26) return A.rad_si;
    if (mt == 7 || mt == 8 || mt == 9 || mt == 10 || mt == 17 || mt == 18 || mt == 19) return A.rad_fe;
    if (mt == 15) return A.rad_ch;
    return 0.0;
}

struct NodeOut {
    double *ro, *nu, *nd, *et, *cp, *kt, *ht, *tk, *po;
};

// ----------------------------------------------------------------- movemark
template <bool MIXED>
__global__ void __launch_bounds__(256) k_move(GridView G, MarkerView M, const DevTypes *__restrict__ Ty,
                                              MoveArgs A, int32_t *__restrict__ key)
{
    const i2g_types &T = Ty->t;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M.n; i += stride) {
        const int mt = M.type[i];
        double x = M.x[i], y = M.y[i];
        const bool inbox = (x >= 0 && y >= 0 && x <= G.xsize && y <= G.ysize);
        if ((inbox || A.outgrid != 1) && !T.markim[mt]) {
            const bool visc = (A.flags & I2G_MOVE_UPDATE_VISC) != 0;
            double pr, ga, e[6];
            int64_t c1, c2;
            interp_e<MIXED>(G, x, y, pr, ga, false, visc, e, c1, c2);
            M.p[i] = pr;
            if (visc) {
                const double Tm = M.T[i];
                if (mt < 50 && Tm > 0) {
                    double eii, sii;
                    invariants(e, eii, sii);
                    double rii = 1.0;
                    const double et = M.eta[i];
                    if (et > 0) rii *= pow(0.5 * sii / eii / et, 0.87);
                    M.eta[i] = viscalc(T, Tm, pr * 1e-5, M.hi ? M.hi[i] : 0.0, eii, sii, rii, A.timesum,
                                       A.relax_time, A.nubeg, A.nuend, mt < 20 ? mt : mt - 20);
                }
            }
            double vx0, vy0;
            const double dt = A.timestep;
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
            if (A.outgrid == 2) {
                if (x < 0 || x > G.xsize) vy0 = 0;
                if (y < 0 || y > G.ysize) vx0 = 0;
            }
            x += dt * vx0;
            y += dt * vy0;
            M.x[i] = x;
            M.y[i] = y;
            if (x < 0 || y < 0 || x > G.xsize || y > G.ysize) M.T[i] = 0;
        }
        key[i] = cell_key(G, x, y);
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

struct MarkerContrib {
    double wx0, wx1, wy0, wy1;
    double mro, mbb, mcp, mkt, mht, mtk, lnu;
    bool immobile;
};

// One marker of the ronurecalc loop (markmart.c:277-855).  Returns false when the
// marker fails the filter of markmart.c:277.  Writes the marker side effects.
template <bool MIXED>
__device__ __forceinline__ bool marker_contrib(const GridView &G, const MarkerView &M, const i2g_types &T,
                                              const AvgArgsK &A, double T0, int64_t k, MarkerContrib &c)
{
    const double x = M.x[k], y = M.y[k];
    double Tm = M.T[k];
    const int mt = M.type[k];
    if (!(x > 0 && y > 0 && x < G.xsize && y < G.ysize && Tm > 0 && mt < 50)) return false;
    const int mm2 = mt;
    const double eta = M.eta[k];
    const bool needvisc = eta <= 0;
    const bool molten = (A.timesum > A.core_form_time) &&
                        (mm2 == 25 || mm2 == 26 || mm2 == 7 || mm2 == 8 || mm2 == 9 || mm2 == 10 || mm2 == 17 ||
                         mm2 == 18 || mm2 == 19);
    double pr, mga, e[6];
    int64_t m10, m20;
    interp_e<MIXED>(G, x, y, pr, mga, molten, needvisc, e, m10, m20);
    const double mpb = pr * 1.0000e-5;
    // sticky air held at the ambient temperature (markmart.c:296-309)
    if (mm2 < 2) {
        if (Tm != A.tmp_ambient) M.T[k] = A.tmp_ambient;
        Tm = A.tmp_ambient;
    }
    const double mtk = Tm;
    double mnu = eta;
    if (needvisc) {
        double eii, sii;
        invariants(e, eii, sii);
        mnu = viscalc(T, mtk, mpb, M.hi ? M.hi[k] : 0.0, eii, sii, 1.0, A.timesum, A.relax_time, A.nubeg,
                      A.nuend, mt < 20 ? mm2 : mm2 - 20);
    }
    {
        double celdx = x - G.xsize / 2.0, celdy = y - G.ysize / 2.0;
        celdy = pow(celdx * celdx + celdy * celdy, 0.5);
        if (celdy > G.xsize / 2.0 * 0.95) mnu = 1.000e+22;
    }
    // porosity and maximum temperature (markmart.c:347-360, 462-472)
    double mpor = M.por ? M.por[k] : 0.0;
    if (mm2 == 0 || mm2 >= 7) mpor = 0.0;
    if (M.tmax && mt != 0 && M.tmax[k] < mtk) M.tmax[k] = mtk;
    if (mpor < 0.000) mpor = 0.000;
    if (mpor > 1.000) mpor = 1.000;
    if (M.por && M.por[k] != mpor) M.por[k] = mpor;
    // density (dencalc, markmart.c:1024-1046), heat capacity, conductivity (markmart.c:475-478)
    double mro, mbb = 0;
    if (A.densimod == 0) {
        mro = T.markro[mm2];
    } else {
        mro = T.markro[mm2] * (1.0 - T.markbb[mm2] * (mtk - 298.15)) * (1.0 + T.markaa[mm2] * (mpb - 1.0) * 1e-3) *
              (1.000 - mpor);
        mbb = T.markbb[mm2] / (1.0 - T.markbb[mm2] * (mtk - 298.15));
    }
    const double mcp = T.markcp[mm2];
    double mkt = (T.markkt[mm2] + T.markkf[mm2] / (mtk + 77.0)) * exp(T.markkp[mm2] * mpb);
    if (molten) {
        if (mm2 == 25 || mm2 == 26) {
            const double xm = A.xmelt_si;
            if (xm >= 0.4000 && xm <= 0.6000)
                mkt = molten_k(T, mm2, mkt, mtk, T0, mro, mga, mcp, mnu, T.markn0[mm2] * exp((-172.690) * (xm - 0.400)));
            if (xm > 0.6000) mkt = molten_k(T, mm2, mkt, mtk, T0, mro, mga, mcp, mnu, 100.0000);
        } else {
            if (A.xmelt_fe < 1.0000) mkt = molten_k(T, mm2, mkt, mtk, T0, mro, mga, mcp, mnu, 1.0000e12);
            if (A.xmelt_fe == 1.0000) mkt = molten_k(T, mm2, mkt, mtk, T0, mro, mga, mcp, mnu, 0.010);
        }
    }
    // porosity-dependent conductivity of solid silicates (markmart.c:614-638)
    if (mm2 == 5 || mm2 == 6) {
        if (mpor < 0.200) mkt = T.markkt[mm2] * exp(-mpor / 0.080);
        if (mpor >= 0.200 && mpor <= 0.400)
            mkt = pow((pow((T.markkt[mm2] * exp(-mpor / 0.080)), 4.000) +
                       pow((T.markkt[mm2] * exp(-1.200 - (mpor / 0.167))), 4.000)),
                      0.250);
        if (mpor > 0.400) mkt = T.markkt[mm2] * exp(-1.200 - (mpor / 0.167));
    }
    if (mkt <= 0.0010) mkt = 0.0010;
    if (mkt >= A.k_cutoff) mkt = A.k_cutoff;
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
    c.lnu = A.viscmod == 1 ? log(mnu) : (A.viscmod == 2 ? 1.0 / mnu : mnu);
    c.immobile = T.markim[mm2] != 0;
    return true;
}

// add one marker into the cell's corner sums (markmart.c:859-910)
template <bool MIXED>
__device__ __forceinline__ void accumulate(const MarkerContrib &c, double *acc)
{
    {
        const double ddx = 1.0 - fabs(c.wx0 - 0.5), ddy = 1.0 - fabs(c.wy0 - 0.5);
        if (ddx > 0.5 && ddy > 0.5) {
            const double swt2 = MIXED ? (double)(4.0f * (float)(ddx - 0.5) * (float)(ddy - 0.5))
                                      : 1.0 * 4.0 * (ddx - 0.5) * (ddy - 0.5);
            acc[40] += c.lnu * swt2;
            acc[41] += swt2;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double wx = (q >> 1) ? c.wx1 : c.wx0;
        const double wy = (q & 1) ? c.wy1 : c.wy0;
        double *a = acc + q * 10;
        if (!MIXED) {
            const double swt = 1.0 * wx * wy;
            if (wx > 0.5 && wy > 0.5) {
                const double swt2 = 1.0 * 4.0 * (wx - 0.5) * (wy - 0.5);
                a[F_NU] += c.lnu * swt2;
                a[F_WNU] += swt2;
            }
            a[F_RO] += c.mro * swt;
            a[F_ET] += c.mbb * swt;
            a[F_CP] += c.mcp * swt;
            a[F_KT] += c.mkt * swt;
            a[F_HT] += c.mht * swt;
            a[F_W0] += swt;
            if (!c.immobile) {
                a[F_TK] += c.mtk * swt;
                a[F_W1] += swt;
            }
        } else {
            // FP32 weights and property products, FP64 accumulation
            const float fx = (float)wx, fy = (float)wy;
            const float swt = fx * fy;
            if (fx > 0.5f && fy > 0.5f) {
                const float swt2 = 4.0f * (fx - 0.5f) * (fy - 0.5f);
                a[F_NU] += c.lnu * (double)swt2;
                a[F_WNU] += (double)swt2;
            }
            a[F_RO] += (double)((float)c.mro * swt);
            a[F_ET] += (double)((float)c.mbb * swt);
            a[F_CP] += (double)((float)c.mcp * swt);
            a[F_KT] += (double)((float)c.mkt * swt);
            a[F_HT] += (double)((float)c.mht * swt);
            a[F_W0] += (double)swt;
            if (!c.immobile) {
                a[F_TK] += (double)((float)c.mtk * swt);
                a[F_W1] += (double)swt;
            }
        }
    }
}

template <bool MIXED>
__global__ void __launch_bounds__(128) k_cellsum(GridView G, MarkerView M, const DevTypes *__restrict__ Ty,
                                                 AvgArgsK A, const int32_t *__restrict__ cstart, int64_t ncells,
                                                 const double *__restrict__ T0p, double *__restrict__ part,
                                                 unsigned long long *__restrict__ navg)
{
    const i2g_types &T = Ty->t;
    const double T0 = *T0p;
    unsigned long long cnt = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += stride) {
        double acc[kPart];
#pragma unroll
        for (int f = 0; f < kPart; f++) acc[f] = 0.0;
        const int32_t k0 = cstart[c], k1 = cstart[c + 1];
        for (int32_t k = k0; k < k1; k++) {
            if (A.gridmod > 1 && (M.id[k] % A.gridmod) != 0) continue;
            MarkerContrib mc;
            if (!marker_contrib<MIXED>(G, M, T, A, T0, k, mc)) continue;
            accumulate<MIXED>(mc, acc);
            cnt++;
        }
#pragma unroll
        for (int f = 0; f < kPart; f++) part[(int64_t)f * ncells + c] = acc[f];
    }
    if (navg) {
        // per-warp totals; integer atomics keep the count exact and order-free
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(navg, cnt);
    }
}

}  // namespace i2g
