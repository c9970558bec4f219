// The mixed-precision marker step in two passes over memory: movemark() with the
// marker's averaging contribution (markmart.c:23-155 then the marker loop of
// markmart.c:271-913), and the per-cell sums with the node loop
// (markmart.c:917-993) in one kernel.
//
//   k_move_fused   persistent CTAs over tiles of 256 markers in storage order,
//                  the next tile's fields staged in shared memory: RK4 through
//                  the staggered grid (on a uniform grid from arithmetic and the
//                  per-quarter-cell velocity forms, no line tables), the new
//                  position and pressure, then the marker's 16-byte averaging
//                  record at its new cell: fixed-point weights, temperature, the
//                  type's slot, and the log-viscosity in the spare bits.  The
//                  record goes to the next free place of its cell's bucket
//                  (ncells x cap places; a full bucket spills to an overflow
//                  list).  No sort: the markers stay where they are.
//   k_cellnodes    a CTA per tile of 31 x (8G - 1) nodes: a warp per cell column,
//                  a lane per cell, each lane adds its cell's records into
//                  per-slot sums and forms its corner sums, the warps exchange
//                  the halves of every node's sum in shared memory, and the nodes
//                  are finished in place.
//
// Order independence.  The records arrive in their buckets in whatever order the
// atomics grant, so every sum is made exact, and exact sums do not depend on the
// order of their terms:
//   - every term of a sum (corner, quadrant and cell-centre weights, temperature
//     x weight, log-viscosity x weight) is rounded to a quantum q of its own sum,
//     a power of two fixed per call by the largest |term| and the largest cell
//     count, after which its FP64 sums are exact;
//   - density, heat capacity, conductivity and heat depend on the rock type alone
//     on these calls, so their sums are per-type weight sums (exact) times the
//     type's values, combined in a fixed order.
// The node values are therefore bitwise the same for every run, launch shape and
// marker storage order.  A node whose temperature or viscosity weight sum is so
// small that the quantum would cost more than 1e-9 of the value is recomputed by
// k_node_guard with quanta of its own.
#pragma once

#include "i2g_avg.cuh"

namespace i2g {

// ----------------------------------------------------------------- layout
constexpr int kFusedParts = 64;  // per-block statistics are spread over this many slots

struct FusedCounters {
    // per slot (block index mod kFusedParts): largest cell count, largest |tk|
    // and |log-viscosity| (FP32 bit patterns of upper bounds), averaged markers
    uint32_t part[kFusedParts][4];
    int32_t novf, ntreset;  // overflow records, pending sticky-air resets
    int32_t ndefer, pad0;   // records whose log-viscosity k_fused_deferred writes
    int32_t nguard, any;    // nodes for k_node_guard; any node viscosity written
    unsigned long long kmin, kmax;  // ordered keys of the smallest / largest node viscosity
};

struct OvfRec {
    float4 a;      // the record (rec_pack)
    double lnu;    // its log-viscosity, unrounded (not read by the sums)
    int32_t cell, pad;
};

struct FusedMove {
    AvgArgsK avg;                // the averaging's constants
    uint8_t tinfo[kAvgTypes];    // per rock type: bits 0-1 type slot, bit 2 immobile
    int32_t cap;                 // places per bucket
    float4 *ra;                  // [ncells * cap] the records (rec_pack)
    OvfRec *ovf;                 // [markers]
    int32_t *count;              // [ncells] records per cell (zeroed before the launch)
    FusedCounters *ctr;          // part/novf/ntreset zeroed before the launch
    int32_t *treset;             // [markers] markers whose T the averaging resets
    int2 *defer;                 // [markers] {marker, record place} of markers without a viscosity
    // a step replayed from a CUDA graph: the step's timesum from a device table
    // (stepc[4 * *stepi]) instead of avg.timesum; NULL otherwise
    const double *stepc;
    const int32_t *stepi;
};

// ----------------------------------------------------------------- uniform axes
// Floors and small int -> float/double casts without conversion instructions
// (which share the SM's narrow XU pipe with log2f and the FP32/FP64 casts):
// adding 2^52 to an FP64 t in [-2^51, 2^51] with rounding down leaves
// 2^52 + floor(t), whose low word is floor(t); adding 1.5 x 2^23 to an FP32 u
// with |u| < 2^22 rounding down leaves a number whose bit pattern counts units
// from 1.5 x 2^23.  The results equal __double2int_rd, __float2int_rd and the
// casts exactly.
constexpr float kF32Magic = 12582912.0f;  // 1.5 x 2^23, bit pattern 0x4B400000
__device__ __forceinline__ int floor_dm(double t) { return __double2loint(__dadd_rd(t, 0x1p52)); }
__device__ __forceinline__ double dbl_of(int k) { return __hiloint2double(0x43300000, k) - 0x1p52; }  // k >= 0
__device__ __forceinline__ int floor_fm(float u, float &fl)
{
    const float s = __fadd_rd(u, kF32Magic);
    fl = s - kF32Magic;
    return __float_as_int(s) - 0x4B400000;
}
__device__ __forceinline__ float flt_of(int d) { return __int_as_float(0x4B400000 + d) - kF32Magic; }  // |d| < 2^22
// The stencil choice and weights of one axis (AxisF) on a uniform axis: b1 is the
// coordinate inside basic cell b in cells; the staggered stencil is the lower or
// upper neighbour by the half-cell, clamped to [0, n-3], with its weight
// (markmart.c:1403-1409, 1431-1437, 1514-1520).
__device__ __forceinline__ void uni_tail(int n, int b, float b1, AxisF &A)
{
    A.b = b;
    A.b1 = b1;
    A.b0 = 1.0f - b1;
    int m = (b1 < 0.5f) ? b - 1 : b;
    if (m < 0) m = 0;
    if (m > n - 3) m = n - 3;
    const float t = b1 - 0.5f + (m != b ? 1.0f : 0.0f);  // (float)(b - m): 0 or 1
    A.m = m;
    A.m1 = t;
    A.m0 = 1.0f - t;
}

// The marker's coordinate x (FP64) on a uniform axis: its cell in the box
// [0, size], the axis data of the first RK4 stage and the offsets of the later
// ones (relative to the cell's lower line, in metres).
__device__ __forceinline__ void uni_axis1(double x, double size, double g0, double w, double iw, float fiw, int n,
                                          AxisF &A, AxisRK &R)
{
    const double xc = x < 0 ? 0.0 : (x > size ? size : x);
    const int b = min(max(floor_dm((xc - g0) * iw), 0), n - 2);
    const double gb = fma(dbl_of(b), w, g0);
    uni_tail(n, b, (float)(xc - gb) * fiw, A);
    R.b = b;
    R.du = (float)(x - gb);
    R.lo = (float)(0.0 - gb);
    R.hi = (float)(size - gb);
}

// a later stage point at offset e (metres from the first stage's line)
__device__ __forceinline__ void uni_stage(const AxisRK &R, float e, float fiw, int n, AxisF &A)
{
    if (e < R.lo) e = R.lo;
    if (e > R.hi) e = R.hi;
    const float u = e * fiw;
    int b = R.b + __float2int_rd(u);
    b = min(max(b, 0), n - 2);
    uni_tail(n, b, u - (float)(b - R.b), A);
}

// A later stage point at offset e on a uniform axis (metres from the first
// stage's line, clamped to the box), in half cells: its quarter index along the
// axis (2 b + upper half, within [0, nh - 1]) and its coordinate in that half
// cell.  fiw2 = 2 / width.
__device__ __forceinline__ void uni_half(const AxisRK &R, float e, float fiw2, int nh, int &h, float &f)
{
    if (e < R.lo) e = R.lo;
    if (e > R.hi) e = R.hi;
    const float s = e * fiw2;
    float fl;
    const int k0 = 2 * R.b + floor_fm(s, fl);
    const int k = min(max(k0, 0), nh - 1);
    h = k;
    f = s - (fl - flt_of(k0 - k));  // s - (float)(k - 2 R.b)
}

// vx and vy at a point of quarter cell (hx, hy) with coordinates (fx, fy) in it,
// from the quarter's two forms (GridView.vq4)
__device__ __forceinline__ void quarter_v(const float4 *__restrict__ q, int nhy, int hx, int hy, float fx, float fy,
                                          float &vx, float &vy)
{
    const float4 *p = q + 2 * (hx * nhy + hy);
    const float4 a = __ldg(p), b = __ldg(p + 1);
    const float fxy = fx * fy;
    vx = fmaf(fxy, a.w, fmaf(fy, a.z, fmaf(fx, a.y, a.x)));
    vy = fmaf(fxy, b.w, fmaf(fy, b.z, fmaf(fx, b.y, b.x)));
}

// The mixed RK4 velocity (markmart.c:73-115) on a uniform grid: vx1, vy1 and the
// pressure at the marker, three later stages in FP32 offsets, the stage sum in
// FP64.  X, Y: the first stage's axis data (strain rates of the viscosity update).
__device__ __forceinline__ void rk4_uni(const GridView &G, double x, double y, double dt, int markmod, double &vx0,
                                        double &vy0, double &pr, AxisF &X, AxisF &Y, AxisRK &RX, AxisRK &RY)
{
    const int nx = (int)G.nx, ny = (int)G.ny;
    uni_axis1(x, G.xsize, G.gx0, G.wx, G.iwx, G.fiwx, nx, X, RX);
    uni_axis1(y, G.ysize, G.gy0, G.wy, G.iwy, G.fiwy, ny, Y, RY);
    const double vx1 = (double)bilq(G.vxq, ny, X.b, Y.m, X.b1, Y.m1);
    const double vy1 = (double)bilq(G.vyq, ny, X.m, Y.b, X.m1, Y.b1);
    pr = (double)bilq(G.prq, ny, X.m + 1, Y.m + 1, X.m1, Y.m1);
    if (markmod == 1) {
        vx0 = vx1;
        vy0 = vy1;
        return;
    }
    const float h = (float)(dt / 2.0), f = (float)dt;
    if (G.vq4) {
        // the later stages from the quarter-cell forms: one index and one
        // coordinate per axis instead of the basic and the staggered stencil
        const int nhx = 2 * (nx - 1), nhy = 2 * (ny - 1);
        const float hx2 = 2.0f * G.fiwx, hy2 = 2.0f * G.fiwy;
        int qx, qy;
        float fx, fy, v2x, v2y, v3x, v3y, v4x, v4y;
        uni_half(RX, RX.du + h * (float)vx1, hx2, nhx, qx, fx);
        uni_half(RY, RY.du + h * (float)vy1, hy2, nhy, qy, fy);
        quarter_v(G.vq4, nhy, qx, qy, fx, fy, v2x, v2y);
        uni_half(RX, RX.du + h * v2x, hx2, nhx, qx, fx);
        uni_half(RY, RY.du + h * v2y, hy2, nhy, qy, fy);
        quarter_v(G.vq4, nhy, qx, qy, fx, fy, v3x, v3y);
        uni_half(RX, RX.du + f * v3x, hx2, nhx, qx, fx);
        uni_half(RY, RY.du + f * v3y, hy2, nhy, qy, fy);
        quarter_v(G.vq4, nhy, qx, qy, fx, fy, v4x, v4y);
        constexpr double sixth = 1.0 / 6.0;
        vx0 = (vx1 + 2.0 * (double)v2x + 2.0 * (double)v3x + (double)v4x) * sixth;
        vy0 = (vy1 + 2.0 * (double)v2y + 2.0 * (double)v3y + (double)v4y) * sixth;
        return;
    }
    AxisF Xs, Ys;
    uni_stage(RX, RX.du + h * (float)vx1, G.fiwx, nx, Xs);
    uni_stage(RY, RY.du + h * (float)vy1, G.fiwy, ny, Ys);
    const float v2x = bilq(G.vxq, ny, Xs.b, Ys.m, Xs.b1, Ys.m1), v2y = bilq(G.vyq, ny, Xs.m, Ys.b, Xs.m1, Ys.b1);
    uni_stage(RX, RX.du + h * v2x, G.fiwx, nx, Xs);
    uni_stage(RY, RY.du + h * v2y, G.fiwy, ny, Ys);
    const float v3x = bilq(G.vxq, ny, Xs.b, Ys.m, Xs.b1, Ys.m1), v3y = bilq(G.vyq, ny, Xs.m, Ys.b, Xs.m1, Ys.b1);
    uni_stage(RX, RX.du + f * v3x, G.fiwx, nx, Xs);
    uni_stage(RY, RY.du + f * v3y, G.fiwy, ny, Ys);
    const float v4x = bilq(G.vxq, ny, Xs.b, Ys.m, Xs.b1, Ys.m1), v4y = bilq(G.vyq, ny, Xs.m, Ys.b, Xs.m1, Ys.b1);
    constexpr double sixth = 1.0 / 6.0;
    vx0 = (vx1 + 2.0 * (double)v2x + 2.0 * (double)v3x + (double)v4x) * sixth;
    vy0 = (vy1 + 2.0 * (double)v2y + 2.0 * (double)v3y + (double)v4y) * sixth;
}

// ----------------------------------------------------------------- move + record
__device__ __forceinline__ unsigned lane_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// The 16-byte averaging record {x word, y word, T, type word}:
//   x word: w1 of x in [0, 1] as fixed point w1 2^24 (bits 0-24), log-viscosity bits 21-27 (25-31)
//   y word: w1 of y likewise (bits 0-24), log-viscosity bits 28-34 (25-31)
//   T: the marker temperature, FP32
//   type word: type slot (bits 0-1), immobile (bit 2), log-viscosity bits 35-63 (3-31)
// The log-viscosity is rounded to its 43 leading bits (sign, exponent, 31
// fraction bits: 2.3e-10 of itself); the cell sums turn w1 back into an FP64
// number with one FMA, and w0 = 1 - w1 exactly there.
constexpr uint32_t kWeightMask = 0x1FFFFFFu;
__device__ __forceinline__ uint32_t weight_fix(double w)
{
    w = w < 0.0 ? 0.0 : (w > 1.0 ? 1.0 : w);
    // w 2^24 + 2^52 rounds to nearest-even at unit resolution: __double2uint_rn(w 2^24)
    return (uint32_t)__double2loint(fma(w, 0x1p24, 0x1p52));
}
__device__ __forceinline__ double weight_of(uint32_t word)
{
    // (2^52 + n) 2^-24 - 2^28 = n 2^-24, exactly
    return fma(__hiloint2double(0x43300000, (int)(word & kWeightMask)), 0x1p-24, -0x1p28);
}
__device__ __forceinline__ float4 rec_with_lnu(float4 r, double lnu)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(lnu) + (1ull << 20);
    const uint32_t lo = (uint32_t)b, hi = (uint32_t)(b >> 32);
    const uint32_t x = (__float_as_uint(r.x) & kWeightMask) | ((lo >> 21) << 25);
    const uint32_t y = (__float_as_uint(r.y) & kWeightMask) | (((lo >> 28) | (hi << 4)) << 25);
    const uint32_t w = (__float_as_uint(r.w) & 7u) | (hi & ~7u);
    return make_float4(__uint_as_float(x), __uint_as_float(y), r.z, __uint_as_float(w));
}
__device__ __forceinline__ float4 rec_pack(uint32_t wx, uint32_t wy, float tk, uint32_t tinfo, double lnu)
{
    return rec_with_lnu(make_float4(__uint_as_float(wx), __uint_as_float(wy), tk, __uint_as_float(tinfo)), lnu);
}
__device__ __forceinline__ double rec_lnu(float4 r)
{
    const uint32_t x = __float_as_uint(r.x), y = __float_as_uint(r.y), w = __float_as_uint(r.w);
    const uint32_t lo = ((x >> 25) << 21) | (((y >> 25) & 0xFu) << 28);
    const uint32_t hi = (w & ~7u) | (y >> 29);
    return __hiloint2double((int)hi, (int)lo);
}

// the log-viscosity of a record from the marker's viscosity (the radmax override
// first, markmart.c:335-340), in the form viscmod asks for
__device__ __forceinline__ double record_lnu(const GridView &G, const AvgArgsK &V, double x, double y, double mnu)
{
    if (outside_radmax(G, V, x, y)) mnu = 1.000e+22;
    return V.viscmod == 1 ? log_mixed(mnu) : (V.viscmod == 2 ? 1.0 / mnu : mnu);
}

// per-thread maxima of the call's quantisation bounds: largest cell count, |tk|
// and |log-viscosity| (FP32 bit patterns of upper bounds)
struct FusedStat {
    uint32_t cnt, tk, lnu;
};

// One marker (slot i; live = i < n) of the fused step: movemark from its loaded
// x, y, T, eta and type, then the averaging record at the new cell.  Every lane of
// the warp calls it together (the bucket places are claimed per warp).
template <bool VISC, bool UNI>
__device__ __forceinline__ void move_record(const GridView &G, const MarkerView &M, const i2g_types &T,
                                            const MoveArgs &A, const FusedMove &F, int64_t i, bool live, int mt,
                                            double x, double y, const double Tm, double eta, FusedStat &st)
{
    const int lane = threadIdx.x & 31;
    bool ok = false, defer = false;
    int32_t key = 0;
    int bx = 0, by = 0;
    float4 rec = make_float4(0.f, 0.f, 0.f, 0.f);
    double lnu = 0.0;
    if (live) {
        // (movemark changes T only for markers that leave the box, which the
        // averaging skips, and eta only with the viscosity update, which reads it
        // again)
        const bool inbox = (x >= 0 && y >= 0 && x <= G.xsize && y <= G.ysize);
        int hx = -1, hy = -1;
        if ((inbox || A.outgrid != 1) && !T.markim[mt]) {
            double pr, vx0, vy0;
            AxisF X1, Y1;
            if (UNI) {
                AxisRK RX, RY;
                rk4_uni(G, x, y, A.timestep, A.markmod, vx0, vy0, pr, X1, Y1, RX, RY);
                hx = RX.b;
                hy = RY.b;
            } else {
                rk4_mixed(G, x, y, A.timestep, A.markmod, vx0, vy0, &pr, hx, hy, VISC ? &X1 : nullptr,
                          VISC ? &Y1 : nullptr);
            }
            M.p[i] = pr;
            if (VISC) {
                double e[6];
                strain_mixed(G, x, y, X1, Y1, e);
                visc_update(M, T, A, i, mt, pr, e);
                eta = M.eta[i];
            }
            if (A.outgrid == 2) {
                if (x < 0 || x > G.xsize) vy0 = 0;
                if (y < 0 || y > G.ysize) vx0 = 0;
            }
            x = advance(x, A.timestep, vx0, A.f32pos);
            y = advance(y, A.timestep, vy0, A.f32pos);
            M.x[i] = x;
            M.y[i] = y;
            if (x < 0 || y < 0 || x > G.xsize || y > G.ysize) M.T[i] = 0;
        }
        // the averaging's filter at the new position (markmart.c:277)
        const AvgArgsK &V = F.avg;
        ok = x > 0 && y > 0 && x < G.xsize && y < G.ysize && Tm > 0 && mt < kAvgTypes &&
             (V.gridmod <= 1 || (M.id[i] % V.gridmod) == 0);
        if (ok) {
            if (UNI) {
                bx = min(max(floor_dm((x - G.gx0) * G.iwx), 0), (int)G.nx - 2);
                by = min(max(floor_dm((y - G.gy0) * G.iwy), 0), (int)G.ny - 2);
            } else {
                bx = hx >= 0 ? cell_walk(G.gx, (int)G.nx, hx, x) : (int)cell_search(G.gx, G.nx, G.inv_x, x);
                by = hy >= 0 ? cell_walk(G.gy, (int)G.ny, hy, y) : (int)cell_search(G.gy, G.ny, G.inv_y, y);
            }
            key = bx * (int32_t)(G.ny - 1) + by;
        }
    }
    // a place in the cell's bucket: warp-aggregated counting atomics, issued
    // before the record is formed so that their round trip overlaps it
    const unsigned okm = __ballot_sync(0xffffffffu, ok);
    unsigned peers = 0;
    int32_t base = 0;
    if (ok) {
        peers = __match_any_sync(okm, key);
        if (lane == __ffs(peers) - 1) base = atomicAdd(F.count + key, __popc(peers));
        // the record: fixed-point weights at the new position, temperature, type
        // slot, log-viscosity
        const AvgArgsK &V = F.avg;
        double wx1, wy1;
        if (UNI) {
            wx1 = (x - fma(dbl_of(bx), G.wx, G.gx0)) * G.iwx;
            wy1 = (y - fma(dbl_of(by), G.wy, G.gy0)) * G.iwy;
        } else {
            wx1 = (x - __ldg(G.gx + bx)) * (double)__ldg(G.ixb + bx);
            wy1 = (y - __ldg(G.gy + by)) * (double)__ldg(G.iyb + by);
        }
        // sticky air held at the ambient temperature (markmart.c:296-309): the
        // record carries it now, the marker's own T is reset by the averaging call
        double mtk = Tm;
        if (mt < 2) {
            mtk = V.tmp_ambient;
            if (Tm != mtk) F.treset[atomicAdd(&F.ctr->ntreset, 1)] = (int32_t)i;
        }
        // a marker without a viscosity of its own (eta <= 0) gets it from
        // viscalc in k_fused_deferred (a place is kept for it here)
        lnu = eta > 0 ? record_lnu(G, V, x, y, eta) : 0.0;
        defer = !(eta > 0);
        rec = rec_pack(weight_fix(wx1), weight_fix(wy1), (float)mtk, (uint32_t)F.tinfo[mt], lnu);
    }
    uint32_t cnt = 0;
    if (ok) {
        base = __shfl_sync(peers, base, __ffs(peers) - 1);
        const int32_t slot = base + __popc(peers & lane_lt());
        cnt = (uint32_t)slot + 1u;
        int32_t place;  // bucket place, or -(overflow index + 1)
        if (slot < F.cap) {
            const int64_t at = (int64_t)key * F.cap + slot;
            F.ra[at] = rec;
            place = (int32_t)at;
        } else {
            const int32_t o = atomicAdd(&F.ctr->novf, 1);
            OvfRec r;
            r.a = rec;
            r.lnu = lnu;
            r.cell = key;
            r.pad = 0;
            F.ovf[o] = r;
            place = -(o + 1);
        }
        if (defer) F.defer[atomicAdd(&F.ctr->ndefer, 1)] = make_int2((int32_t)i, place);
    }
    // the warp's bounds into its running maxima (lane 0)
    if (okm) {
        const uint32_t m0 = __reduce_max_sync(0xffffffffu, cnt);
        const uint32_t m1 = __reduce_max_sync(0xffffffffu, ok ? __float_as_uint(fabsf(rec.z)) : 0u);
        const uint32_t m2 = __reduce_max_sync(0xffffffffu, ok ? __float_as_uint(__double2float_ru(fabs(lnu))) : 0u);
        if (lane == 0) {
            st.cnt = max(st.cnt, m0);
            st.tk = max(st.tk, m1);
            st.lnu = max(st.lnu, m2);
        }
    }
}

// the warp's bounds (lane 0) into one of kFusedParts slots (an atomic only where
// the value exceeds the slot's)
__device__ __forceinline__ void fused_stat_flush(const FusedStat &st, FusedCounters *ctr)
{
    const uint32_t m0 = st.cnt, m1 = st.tk, m2 = st.lnu;
    if ((threadIdx.x & 31) == 0 && m0 > 0) {
        uint32_t *dst = ctr->part[(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) % kFusedParts];
        if (m0 > *(volatile uint32_t *)(dst + 0)) atomicMax(dst + 0, m0);
        if (m1 > *(volatile uint32_t *)(dst + 1)) atomicMax(dst + 1, m1);
        if (m2 > *(volatile uint32_t *)(dst + 2)) atomicMax(dst + 2, m2);
    }
}

// k_move_fused's tiles: 256 markers, one per thread; x, y, T, eta of the next
// tile are copied into shared memory (cp.async, 8 bytes per field and thread)
// while the current one is computed, the type is loaded a tile ahead into a
// register
constexpr int kMoveTile = 256;
struct MoveStage {
    double v[4][kMoveTile];  // x, y, T, eta
};

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void move_stage_issue(const MarkerView &M, MoveStage &S, int64_t i)
{
    if (i < M.n) {
        const int t = threadIdx.x;
        cp_async8(&S.v[0][t], M.x + i);
        cp_async8(&S.v[1][t], M.y + i);
        cp_async8(&S.v[2][t], M.T + i);
        cp_async8(&S.v[3][t], M.eta + i);
    }
    cp_async_commit();
}

// Persistent: CTA b takes tiles b, b + gridDim.x, ... (the grid is the resident
// CTAs of the device, one wave), so the loads of the next tile are in flight
// while the current tile computes.  Each thread copies and reads only its own
// marker's fields: the cp.async group wait orders them, no CTA barrier.
template <bool VISC, bool UNI>
__global__ void __launch_bounds__(kMoveTile, VISC ? 2 : 4) k_move_fused(const __grid_constant__ GridView G,
                                                    const __grid_constant__ MarkerView M,
                                                    const DevTypes *__restrict__ Ty, const __grid_constant__ MoveArgs A,
                                                    const __grid_constant__ FusedMove F)
{
    __shared__ MoveStage S[2];
    __shared__ FusedStat wst[kMoveTile / 32];
    const i2g_types &T = Ty->t;
    const int tid = threadIdx.x;
    const int ntiles = (int)((M.n + kMoveTile - 1) / kMoveTile);
    FusedStat &st = wst[tid >> 5];
    if ((tid & 31) == 0) st = FusedStat{0u, 0u, 0u};
    int tile = blockIdx.x;
    int64_t i = (int64_t)tile * kMoveTile + tid;
    move_stage_issue(M, S[0], i);
    int mt_next = i < M.n ? M.type[i] : 0;
    for (int b = 0; tile < ntiles; tile += gridDim.x, b ^= 1) {
        i = (int64_t)tile * kMoveTile + tid;
        const int64_t inext = i + (int64_t)gridDim.x * kMoveTile;
        move_stage_issue(M, S[b ^ 1], inext);
        const int mt = mt_next;
        mt_next = inext < M.n ? M.type[inext] : 0;
        cp_async_wait<1>();  // this tile's copies
        const bool live = i < M.n;
        double x = 0.0, y = 0.0, Tm = 0.0, eta = 0.0;
        if (live) {
            x = S[b].v[0][tid];
            y = S[b].v[1][tid];
            Tm = S[b].v[2][tid];
            eta = S[b].v[3][tid];
        }
        move_record<VISC, UNI>(G, M, T, A, F, i, live, mt, x, y, Tm, eta, st);
    }
    cp_async_wait<0>();
    fused_stat_flush(st, F.ctr);
}

// The markers k_move_fused kept a place for: viscosity from the rheology at the
// marker's new position (allintere + viscalc, markmart.c:281, 320-332), then the
// record's log-viscosity and the call's |log-viscosity| bound.
template <bool MIXED>
__global__ void __launch_bounds__(128) k_fused_deferred(const __grid_constant__ GridView G,
                                                        const __grid_constant__ MarkerView M,
                                                        const DevTypes *__restrict__ Ty,
                                                        const __grid_constant__ FusedMove F)
{
    const int32_t m = F.ctr->ndefer;
    if (m == 0) return;
    AvgArgsK V = F.avg;  // viscalc's impact weakening reads timesum (markmart.c:1886-1889)
    if (F.stepc) V.timesum = F.stepc[4 * *F.stepi];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < m; q += stride) {
        const int2 d = F.defer[q];
        const int64_t i = d.x;
        const double x = M.x[i], y = M.y[i];
        const int mt = M.type[i];
        const double mtk = mt < 2 ? V.tmp_ambient : M.T[i];
        double pr = 0.0, mga = 0.0, mnu = 0.0;
        int64_t m10, m20;
        pressure_visc<MIXED>(G, Ty->t, V, x, y, mtk, M.hi ? M.hi[i] : 0.0, mt, false, true, pr, mga, mnu, m10, m20);
        const double lnu = record_lnu(G, V, x, y, mnu);
        if (d.y >= 0) {
            F.ra[d.y] = rec_with_lnu(F.ra[d.y], lnu);
        } else {
            OvfRec &r = F.ovf[-d.y - 1];
            r.a = rec_with_lnu(r.a, lnu);
            r.lnu = lnu;
        }
        atomicMax(&F.ctr->part[q % kFusedParts][2], __float_as_uint(__double2float_ru(fabs(lnu))));
    }
}

// ----------------------------------------------------------------- sums and nodes
// The rounding of one averaging call, derived from the counters.  A term t of a
// sum is replaced by fma(a, b, c) - c = t rounded to the nearest multiple of the
// sum's quantum q = 2^(e - 52), c = 1.5 * 2^e, where 2^e exceeds the largest
// magnitude any node's sum can reach (4 x the largest cell count x the largest
// |term|): every partial sum is then an integer multiple of q below 2^52 q, an
// exact FP64 number, whatever the order of the additions.
struct QConst {
    double cw, ctk, cnu;  // weights, temperature x weight, log-viscosity x weight
    // a node goes to k_node_guard where a weight sum is below thr_w (thr_nuw for
    // the viscosity weights), or |TK| below vtk, or |NU|, |ND| below vnu: there
    // the quanta could move its value by more than 1e-9 of the value
    double thr_w, thr_nuw, vtk, vnu;
};

__device__ __forceinline__ QConst qconst_of(uint32_t cmax, uint32_t tkb, uint32_t lnb, int viscmod)
{
    QConst Q;
    // weights are FP32 in [0, 1] up to a rounding: bound them by 1 + 2^-20
    const double Nn = 4.0 * (double)(cmax > 0 ? cmax : 1u), Sw = Nn * (1.0 + 0x1p-20);
    const double Mtk = (double)__uint_as_float(tkb), Mnu = (double)__uint_as_float(lnb);
    const double Stk = Sw * Mtk, Snu = Sw * Mnu;
    const int ew = ilogb(Sw) + 1, etk = Stk > 0 ? ilogb(Stk) + 1 : 0, enu = Snu > 0 ? ilogb(Snu) + 1 : 0;
    Q.cw = ldexp(1.5, ew);
    Q.ctk = ldexp(1.5, etk);
    Q.cnu = ldexp(1.5, enu);
    // A node sum of up to Nn terms moves by at most Nn q / 2.  A weighted mean
    // S / W then moves by at most (Nn q_S / 2) / |S| + (Nn q_w / 2) / W of
    // itself; keep each part below 1e-9.  For log-viscosity (viscmod 1) the mean
    // is an exponent: its absolute error, (Nn q_S / 2 + |mean| Nn q_w / 2) / W,
    // is the relative error of the node value.
    const double qw = ldexp(1.0, ew - 52), qtk = ldexp(1.0, etk - 52), qnu = ldexp(1.0, enu - 52);
    Q.thr_w = Nn * qw / 2e-9;
    Q.vtk = 4.0 * Nn * qtk / 2e-9;  // a corner's T term combines four quantized sums
    if (viscmod == 1) {
        Q.thr_nuw = Nn * (qnu + qw * Mnu) / 2e-9;
        Q.vnu = 0.0;
    } else {
        Q.thr_nuw = Q.thr_w;
        Q.vnu = Nn * qnu / 2e-9;
    }
    return Q;
}

// the counters' maxima over the kFusedParts slots; every thread of the block
// gets the same QConst (threads 0..63 read, the block reduces in shared memory)
__device__ __forceinline__ QConst block_qconst(const FusedCounters *ctr, int viscmod)
{
    __shared__ uint32_t s[3][2];
    __shared__ QConst sq;
    const int t = threadIdx.x;
    uint32_t a = 0, b = 0, c = 0;
    if (t < kFusedParts) {
        a = ctr->part[t][0];
        b = ctr->part[t][1];
        c = ctr->part[t][2];
    }
    if (t < 64) {
        a = __reduce_max_sync(0xffffffffu, a);
        b = __reduce_max_sync(0xffffffffu, b);
        c = __reduce_max_sync(0xffffffffu, c);
        if ((t & 31) == 0) {
            s[0][t >> 5] = a;
            s[1][t >> 5] = b;
            s[2][t >> 5] = c;
        }
    }
    __syncthreads();
    if (t == 0) sq = qconst_of(max(s[0][0], s[0][1]), max(s[1][0], s[1][1]), max(s[2][0], s[2][1]), viscmod);
    __syncthreads();
    return sq;
}

__device__ __forceinline__ double quant(double a, double b, double c) { return fma(a, b, c) - c; }

// The sums of one cell.  A record's corner weights are the products X0 Y0,
// X0 Y1, X1 Y0, X1 Y1 of its axis weights (X0 = 1 - X1, Y0 = 1 - Y1), so the
// cell keeps, per type slot, the record count and the sums of X1, Y1 and X1 Y1
// (quantized), and for the mobile records T, T X1, T Y1 and T X1 Y1
// (quantized); acc_corners turns them into the four corner sums, exactly.  The
// node viscosity goes to the nearest node with the quadrant weight, the
// cell-centre one with the tent weight.
template <int NT>
struct CellAcc {
    int32_t n[NT];
    double sx[NT], sy[NT], sxy[NT];
    double t0, tx, ty, txy;
    double nu[4], wnu[4];
    double nd, wnd;
};

template <int NT>
__device__ __forceinline__ void acc_zero(CellAcc<NT> &a)
{
#pragma unroll
    for (int k = 0; k < NT; k++) {
        a.n[k] = 0;
        a.sx[k] = a.sy[k] = a.sxy[k] = 0.0;
    }
    a.t0 = a.tx = a.ty = a.txy = 0.0;
#pragma unroll
    for (int q = 0; q < 4; q++) a.nu[q] = a.wnu[q] = 0.0;
    a.nd = a.wnd = 0.0;
}

// One record into its cell's sums (markmart.c:859-913): weights from the
// record's fixed-point X1, Y1 (exact in FP64, as are X1 - 1/2 and 1 - X1);
// every product rounded to its sum's quantum.
template <int NT>
__device__ __forceinline__ void acc_rec(CellAcc<NT> &a, float4 r, const QConst &Q)
{
    const double lnu = rec_lnu(r);
    const double X1 = weight_of(__float_as_uint(r.x)), Y1 = weight_of(__float_as_uint(r.y));
    const double p = quant(X1, Y1, Q.cw);
    const uint32_t tf = __float_as_uint(r.w);
    const int slot = (int)(tf & 3u);
#pragma unroll
    for (int k = 0; k < NT; k++) {
        const double oh = (slot == k) ? 1.0 : 0.0;
        a.n[k] += slot == k ? 1 : 0;
        a.sx[k] = fma(oh, X1, a.sx[k]);
        a.sy[k] = fma(oh, Y1, a.sy[k]);
        a.sxy[k] = fma(oh, p, a.sxy[k]);
    }
    if (!(tf & 4u)) {  // mobile type: temperature
        const double tk = (double)r.z;
        a.t0 += quant(tk, 1.0, Q.ctk);
        a.tx += quant(tk, X1, Q.ctk);
        a.ty += quant(tk, Y1, Q.ctk);
        a.txy += quant(tk * X1, Y1, Q.ctk);
    }
    // the nearest node takes the viscosity with the quadrant weight
    // 4 (wa - 1/2)(wb - 1/2), wa = max(X0, X1) = 1/2 + |X1 - 1/2| (both weights
    // above one half: at most one corner)
    const double ax = X1 - 0.5, ay = Y1 - 0.5, fx = fabs(ax), fy = fabs(ay);
    if (fx > 0.0 && fy > 0.0) {
        const double s2 = 4.0 * fx * fy;
        const double t = quant(lnu, s2, Q.cnu), s2q = quant(s2, 1.0, Q.cw);
        const int qq = (ax > 0.0 ? 2 : 0) | (ay > 0.0 ? 1 : 0);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const double oh = (q == qq) ? 1.0 : 0.0;
            a.nu[q] = fma(oh, t, a.nu[q]);
            a.wnu[q] = fma(oh, s2q, a.wnu[q]);
        }
    }
    // the cell centre takes it with the tent weight 4 (dx - 1/2)(dy - 1/2),
    // dx = 1 - |X0 - 1/2|, so dx - 1/2 = 1/2 - |X1 - 1/2|
    const double cx = 0.5 - fx, cy = 0.5 - fy;
    if (cx > 0.0 && cy > 0.0) {
        const double s2 = 4.0 * cx * cy;
        a.nd += quant(lnu, s2, Q.cnu);
        a.wnd += quant(s2, 1.0, Q.cw);
    }
}

// The corner sums of a cell (corner q = 2a + b at node (m1 + a, m2 + b)): per
// slot X0 Y0 = n - X1 - Y1 + X1 Y1, X0 Y1 = Y1 - X1 Y1, X1 Y0 = X1 - X1 Y1,
// X1 Y1, likewise for T x weight; the mobile weight is the sum over the mobile
// slots (mob: bit k set when slot k's type moves).  Every term is a multiple of
// the sums' quanta and every partial sum stays below the quantum's range (the
// counts are below 2^18), so each is exact.
template <int NT>
__device__ __forceinline__ void acc_corners(const CellAcc<NT> &a, uint32_t mob, double (*wt)[4], double *w1,
                                            double *tk)
{
#pragma unroll
    for (int q = 0; q < 4; q++) w1[q] = 0.0;
#pragma unroll
    for (int k = 0; k < NT; k++) {
        const double n = (double)a.n[k];
        wt[k][3] = a.sxy[k];
        wt[k][2] = a.sx[k] - a.sxy[k];
        wt[k][1] = a.sy[k] - a.sxy[k];
        wt[k][0] = ((n - a.sx[k]) - a.sy[k]) + a.sxy[k];
        if ((mob >> k) & 1u) {
#pragma unroll
            for (int q = 0; q < 4; q++) w1[q] += wt[k][q];
        }
    }
    tk[3] = a.txy;
    tk[2] = a.tx - a.txy;
    tk[1] = a.ty - a.txy;
    tk[0] = ((a.t0 - a.tx) - a.ty) + a.txy;
}

struct CellNodesArgs {
    int32_t nx, ny, nc1, nc2, cap;
    uint32_t mob;  // bit k set when type slot k's type is mobile (its T is averaged)
    int32_t ncol;  // node columns per CTA: 8 * groups - 1
    int32_t ntx;   // CTAs along x
    const int32_t *count;
    const float4 *ra;
    const OvfRec *ovf;
    FusedCounters *ctr;
    double sv[4][4];  // per type slot: ro, cp, kt, ht
    // a step replayed from a CUDA graph: the slots' radiogenic heat from the
    // step's row of a device table (stepc[4 * *stepi + group] x density, group
    // 1..3 = silicate, iron, chondrite, 0 = none) instead of sv[.][3]; NULL otherwise
    const double *stepc;
    const int32_t *stepi;
    double sro[4];
    int32_t sgrp[4];
    int32_t viscmod;
    double nubeg, nuend;
    const double *mu;
    NodeOut O;
    int32_t *guard;
    unsigned long long *navg;  // averaged markers (the records of the cells a CTA owns)
};

// values of a node half (the corner sums of one cell column reaching a node column):
// wt[NT], w1, tk, nu, wnu, then (right halves only) nd, wnd
template <int NT>
struct NodeVals {
    static constexpr int L = NT + 4, R = NT + 6;
};

// uint4 per staged row: 4 records of 16 B.  Record t of row r sits at place
// t ^ cn_swz(r): the 8 rows a quarter warp reads at once then fall on 8
// distinct 16-byte bank groups
constexpr int kCnRS = 4;
__device__ __forceinline__ int cn_swz(int row) { return (row >> 1) & 3; }

struct CnWarpBuf {
    uint4 rec[2][32 * kCnRS];
    int32_t cb[32], cn[32];
};

template <int NT>
struct CnSmem {
    CnWarpBuf w[8];
    double hr[2][8][NodeVals<NT>::R][32];  // right halves, double buffered by group
};

// asynchronous copies of positions [P0, P0 + 4) of the strip's 32 buckets
__device__ __forceinline__ void cn_stage(const CnWarpBuf &B, uint4 *dst, const float4 *__restrict__ ra, int P0,
                                         int lane)
{
#pragma unroll
    for (int it = 0; it < 4; it++) {
        const int e = it * 32 + lane, row = e >> 2, piece = e & 3;
        const int rec = P0 + piece;
        const bool valid = rec < B.cn[row];
        const uint4 *src = reinterpret_cast<const uint4 *>(ra);
        if (valid) src = reinterpret_cast<const uint4 *>(ra + (int64_t)B.cb[row] + rec);
        cp_async16(dst + row * kCnRS + (piece ^ cn_swz(row)), src, valid);
    }
    cp_async_commit();
}

__device__ __forceinline__ unsigned long long okey(double v)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double okey_inv(unsigned long long k)
{
    return __longlong_as_double((long long)((k >> 63) ? (k & 0x7fffffffffffffffull) : ~k));
}

__device__ __forceinline__ double visc_finish(int viscmod, double v)
{
    if (viscmod == 1) v = exp(v);
    if (viscmod == 2) v = 1.0 / v;
    return v;
}

// Node m3 from its sums (markmart.c:917-993), the FP64 node loop: viscosity at
// the node (quadrant sums) and at the cell centre (nd), then the weighted means.
// S: per-slot weights wt[NT], w1, tk, nu, wnu, nd, wnd.
// The type slots' radiogenic heat of this call (sv[.][3]) or, for a step replayed
// from a graph, of the step's row of the device table, in shared memory: the
// block's first threads write it, the block syncs before node_write reads it.
__device__ __forceinline__ double *slot_heat()
{
    __shared__ double h[kFusedSlots];
    return h;
}
__device__ __forceinline__ void slot_heat_init(const CellNodesArgs &P)
{
    if (threadIdx.x < kFusedSlots) {
        const int s = threadIdx.x;
        double v = P.sv[s][3];
        if (P.stepc) {
            const int g = P.sgrp[s];
            const double rad = g ? P.stepc[4 * *P.stepi + g] : 0.0;
            v = rad * P.sro[s];  // rad_of(type) x density, as the host forms sv[.][3]
        }
        slot_heat()[s] = v;
    }
}

template <int NT>
__device__ __forceinline__ void node_write(const CellNodesArgs &P, int64_t m3, const double *S, double &vmin,
                                           double &vmax, int &any)
{
    double W0 = 0.0;
#pragma unroll
    for (int k = 0; k < NT; k++) W0 += S[k];
    const double W1 = S[NT], TK = S[NT + 1], NU = S[NT + 2], WNU = S[NT + 3], ND = S[NT + 4], WND = S[NT + 5];
    const double mu = P.mu ? __ldg(P.mu + m3) : 0.0;
    if (WNU != 0.0) {
        double v = mu ? mu : visc_finish(P.viscmod, NU / WNU);
        if (v < P.nubeg) v = P.nubeg;
        if (v > P.nuend) v = P.nuend;
        if (!any) { vmin = vmax = v; any = 1; }
        else { vmin = fmin(vmin, v); vmax = fmax(vmax, v); }
        P.O.nu[m3] = v;
    }
    if (WND != 0.0) {
        double v = mu ? mu : visc_finish(P.viscmod, ND / WND);
        if (v < P.nubeg) v = P.nubeg;
        if (v > P.nuend) v = P.nuend;
        if (!any) { vmin = vmax = v; any = 1; }
        else { vmin = fmin(vmin, v); vmax = fmax(vmax, v); }
        P.O.nd[m3] = v;
        P.O.po[m3] = 0.0;  // po0[] is never accumulated (markmart.c:968)
    }
    if (W0 != 0.0) {
        double r = 0.0, c = 0.0, k = 0.0, h = 0.0;
#pragma unroll
        for (int s = 0; s < NT; s++) {
            r += P.sv[s][0] * S[s];
            c += P.sv[s][1] * S[s];
            k += P.sv[s][2] * S[s];
            h += slot_heat()[s] * S[s];
        }
        P.O.ro[m3] = r / W0;
        P.O.et[m3] = 0.0 / W0;  // beta is zero on constant-property calls
        P.O.cp[m3] = c / W0;
        P.O.kt[m3] = k / W0;
        P.O.ht[m3] = h / W0;
        if (W1 != 0.0) P.O.tk[m3] = TK / W1;
    }
}

// A node whose sums are so small that the call's quanta would cost more than
// 1e-9 of a value is listed for k_node_guard instead of written.
template <int NT>
__device__ __forceinline__ void node_finish(const CellNodesArgs &P, const QConst &Q, int m1, int m2, const double *S,
                                            double &vmin, double &vmax, int &any)
{
    const int64_t m3 = (int64_t)m1 * P.ny + m2;
    double W0 = 0.0;
#pragma unroll
    for (int k = 0; k < NT; k++) W0 += S[k];
    const double W1 = S[NT], TK = S[NT + 1], NU = S[NT + 2], WNU = S[NT + 3], ND = S[NT + 4], WND = S[NT + 5];
    const bool flag = (W0 > 0 && W0 < Q.thr_w) || (W1 > 0 && (W1 < Q.thr_w || fabs(TK) < Q.vtk)) ||
                      (WNU > 0 && (WNU < Q.thr_nuw || fabs(NU) < Q.vnu)) ||
                      (WND > 0 && (WND < Q.thr_nuw || fabs(ND) < Q.vnu));
    if (flag) P.guard[atomicAdd(&P.ctr->nguard, 1)] = (int32_t)m3;
    else node_write<NT>(P, m3, S, vmin, vmax, any);
}

// {min, max, any} of the CTA into the call's ordered-key atomics
__device__ __forceinline__ void fold_minmax(double vmin, double vmax, int any, FusedCounters *ctr,
                                            unsigned cnt = 0, unsigned long long *navg = nullptr)
{
    __shared__ double smin[32], smax[32];
    __shared__ int sany[32];
    if (navg) {
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(navg, (unsigned long long)cnt);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        const double a2 = __shfl_down_sync(0xffffffffu, vmin, o), b2 = __shfl_down_sync(0xffffffffu, vmax, o);
        const int c2 = __shfl_down_sync(0xffffffffu, any, o);
        if (c2) {
            if (!any) { vmin = a2; vmax = b2; any = 1; }
            else { vmin = fmin(vmin, a2); vmax = fmax(vmax, b2); }
        }
    }
    __syncthreads();
    if (lane == 0) { smin[w] = vmin; smax[w] = vmax; sany[w] = any; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        int c = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
            if (!sany[i]) continue;
            if (!c) { a = smin[i]; b = smax[i]; c = 1; }
            else { a = fmin(a, smin[i]); b = fmax(b, smax[i]); }
        }
        if (c) {
            atomicMin(&ctr->kmin, okey(a));
            atomicMax(&ctr->kmax, okey(b));
            if (!ctr->any) atomicExch(&ctr->any, 1);
        }
    }
}

// One CTA: node rows [d0, d0 + 31) x node columns [cs, cs + ncol).  Warp w of
// group g sums cell column cc = cs - 1 + 8g + w, lane l cell row d0 - 1 + l; the
// node column cc is finished by the same warp from its left half and the right
// half of column cc - 1 (the warp before it, or the previous group's last).
template <int NT>
__global__ void __launch_bounds__(256, NT == 4 ? 2 : 3) k_cellnodes(const __grid_constant__ CellNodesArgs P)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    CnSmem<NT> &S = *reinterpret_cast<CnSmem<NT> *>(smraw);
    constexpr int NL = NodeVals<NT>::L, NR = NodeVals<NT>::R;
    slot_heat_init(P);  // block_qconst syncs the block
    const QConst Q = block_qconst(P.ctr, P.viscmod);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cs = (int)(blockIdx.x % P.ntx) * P.ncol, d0 = (int)(blockIdx.x / P.ntx) * 31;
    const int groups = (P.ncol + 1) / 8;
    CnWarpBuf &B = S.w[warp];
    const int novf = P.ctr->novf;
    double vmin = 0.0, vmax = 0.0;
    int any = 0;
    unsigned owned = 0;
    for (int g = 0; g < groups; g++) {
        const int cc = cs - 1 + 8 * g + warp, cr = d0 - 1 + lane;
        const bool valid = cc >= 0 && cc < P.nc1 && cr >= 0 && cr < P.nc2;
        const int64_t cell = (int64_t)cc * P.nc2 + cr;
        int32_t n = valid ? __ldg(P.count + cell) : 0;
        if (lane >= 1 && !(g == 0 && warp == 0)) owned += (unsigned)n;  // each cell counted by one CTA
        const int32_t nb = min(n, P.cap);
        int maxc = nb;
        for (int o = 16; o > 0; o >>= 1) maxc = max(maxc, __shfl_xor_sync(0xffffffffu, maxc, o));
        __syncwarp();
        B.cb[lane] = valid ? (int32_t)(cell * P.cap) : 0;
        B.cn[lane] = nb;
        __syncwarp();
        CellAcc<NT> a;
        acc_zero(a);
        if (maxc > 0) cn_stage(B, B.rec[0], P.ra, 0, lane);
        for (int P0 = 0, k = 0; P0 < maxc; P0 += 4, k ^= 1) {
            if (P0 + 4 < maxc) {
                cn_stage(B, B.rec[k ^ 1], P.ra, P0 + 4, lane);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncwarp();
            const uint4 *row = B.rec[k] + lane * kCnRS;
            const int m = min(4, nb - P0);
            for (int t = 0; t < m; t++) {
                const uint4 u = row[t ^ cn_swz(lane)];
                acc_rec<NT>(a, make_float4(__uint_as_float(u.x), __uint_as_float(u.y), __uint_as_float(u.z),
                                           __uint_as_float(u.w)),
                            Q);
            }
            __syncwarp();
        }
        if (n > nb) {  // a full bucket: the rest of the cell's records are in the overflow list
            for (int o = 0; o < novf; o++) {
                const OvfRec r = P.ovf[o];
                if (r.cell == (int32_t)cell) acc_rec<NT>(a, r.a, Q);
            }
        }
        // left half (corners 0 and 1 reach node column cc) and right half
        // (corners 2, 3 and the centre reach node column cc + 1) of the node at
        // row cr: corner 0 of this lane, corner 1 of the lane below
        double L[NL];
        double *hr = &S.hr[g & 1][warp][0][0];
        double wt[NT][4], w1[4], tk[4];
        acc_corners<NT>(a, P.mob, wt, w1, tk);
#pragma unroll
        for (int k = 0; k < NT; k++) {
            L[k] = wt[k][0] + __shfl_up_sync(0xffffffffu, wt[k][1], 1);
            hr[k * 32 + lane] = wt[k][2] + __shfl_up_sync(0xffffffffu, wt[k][3], 1);
        }
        L[NT + 0] = w1[0] + __shfl_up_sync(0xffffffffu, w1[1], 1);
        L[NT + 1] = tk[0] + __shfl_up_sync(0xffffffffu, tk[1], 1);
        L[NT + 2] = a.nu[0] + __shfl_up_sync(0xffffffffu, a.nu[1], 1);
        L[NT + 3] = a.wnu[0] + __shfl_up_sync(0xffffffffu, a.wnu[1], 1);
        hr[(NT + 0) * 32 + lane] = w1[2] + __shfl_up_sync(0xffffffffu, w1[3], 1);
        hr[(NT + 1) * 32 + lane] = tk[2] + __shfl_up_sync(0xffffffffu, tk[3], 1);
        hr[(NT + 2) * 32 + lane] = a.nu[2] + __shfl_up_sync(0xffffffffu, a.nu[3], 1);
        hr[(NT + 3) * 32 + lane] = a.wnu[2] + __shfl_up_sync(0xffffffffu, a.wnu[3], 1);
        hr[(NT + 4) * 32 + lane] = __shfl_up_sync(0xffffffffu, a.nd, 1);
        hr[(NT + 5) * 32 + lane] = __shfl_up_sync(0xffffffffu, a.wnd, 1);
        __syncthreads();
        const int m1 = cc, m2 = cr;
        if (lane >= 1 && m1 >= cs && m1 < cs + P.ncol && m1 < P.nx && m2 < P.ny && !(g == 0 && warp == 0)) {
            const double *hp = warp > 0 ? &S.hr[g & 1][warp - 1][0][0] : &S.hr[(g - 1) & 1][7][0][0];
            double Sv[NR];
#pragma unroll
            for (int k = 0; k < NL; k++) Sv[k] = L[k] + hp[k * 32 + lane];
            Sv[NT + 4] = hp[(NT + 4) * 32 + lane];
            Sv[NT + 5] = hp[(NT + 5) * 32 + lane];
            node_finish<NT>(P, Q, m1, m2, Sv, vmin, vmax, any);
        }
        __syncthreads();
    }
    fold_minmax(vmin, vmax, any, P.ctr, owned, P.navg);
}

// Nodes listed by k_cellnodes, a warp each: the records of the node's four cells
// once for the largest terms, once more with quanta fitted to this node (so the
// sums are exact again, at a resolution of 2^-52 of the node's own largest
// terms), then the node as node_write makes it.
template <int NT>
__global__ void __launch_bounds__(128) k_node_guard(const __grid_constant__ CellNodesArgs P)
{
    slot_heat_init(P);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int ng = P.ctr->nguard, novf = P.ctr->novf;
    const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    double vmin = 0.0, vmax = 0.0;
    int any = 0;
    constexpr int NV = NT + 6;
    for (int64_t gi = warp0; gi < ng; gi += nwarps) {
        const int64_t m3 = P.guard[gi];
        const int m1 = (int)(m3 / P.ny), m2 = (int)(m3 - (int64_t)m1 * P.ny);
        // the terms of a record of cell c (c = 0..3: cells (m1-1, m2-1), (m1-1, m2),
        // (m1, m2-1), (m1, m2)), which reaches the node through its corner 3 - c:
        // t[0] weight, t[1] T x weight, t[2] quadrant weight, t[3] its
        // log-viscosity term, t[4] centre weight, t[5] its term
        auto terms = [&](int c, float4 r, double lnu, double *t) {
            const int q = 3 - c;
            const double X1 = weight_of(__float_as_uint(r.x)), Y1 = weight_of(__float_as_uint(r.y));
            const double X0 = 1.0 - X1, Y0 = 1.0 - Y1;
            const double wx = (q >> 1) ? X1 : X0, wy = (q & 1) ? Y1 : Y0;
            t[0] = wx * wy;
            t[1] = (double)r.z * t[0];
            t[2] = t[3] = t[4] = t[5] = 0.0;
            if (wx > 0.5 && wy > 0.5) {
                t[2] = 4.0 * (wx - 0.5) * (wy - 0.5);
                t[3] = lnu * t[2];
            }
            if (c == 0) {
                const double dx = 1.0 - fabs(X0 - 0.5), dy = 1.0 - fabs(Y0 - 0.5);
                if (dx > 0.5 && dy > 0.5) {
                    t[4] = 4.0 * (dx - 0.5) * (dy - 0.5);
                    t[5] = lnu * t[4];
                }
            }
        };
        auto each = [&](auto &&fn) {
            for (int c = 0; c < 4; c++) {
                const int c1 = m1 - 1 + (c >> 1), c2 = m2 - 1 + (c & 1);
                if (c1 < 0 || c2 < 0 || c1 >= P.nc1 || c2 >= P.nc2) continue;
                const int64_t cell = (int64_t)c1 * P.nc2 + c2;
                const int32_t n = P.count[cell], nb = min(n, P.cap);
                for (int t = lane; t < nb; t += 32) {
                    const float4 r = P.ra[cell * P.cap + t];
                    fn(c, r, rec_lnu(r));
                }
                if (n > nb)
                    for (int o = lane; o < novf; o += 32)
                        if (P.ovf[o].cell == (int32_t)cell) fn(c, P.ovf[o].a, rec_lnu(P.ovf[o].a));
            }
        };
        double mx[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int nrec = 0;
        each([&](int c, float4 r, double lnu) {
            double t[6];
            terms(c, r, lnu, t);
            for (int k = 0; k < 6; k++) mx[k] = fmax(mx[k], fabs(t[k]));
            nrec++;
        });
        for (int o = 16; o > 0; o >>= 1) {
            for (int k = 0; k < 6; k++) mx[k] = fmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
            nrec += __shfl_xor_sync(0xffffffffu, nrec, o);
        }
        double cq[6];
        for (int k = 0; k < 6; k++) {
            const double b = (double)(nrec > 0 ? nrec : 1) * mx[k];
            cq[k] = ldexp(1.5, b > 0 ? ilogb(b) + 1 : 0);
        }
        double S[NV];
        for (int k = 0; k < NV; k++) S[k] = 0.0;
        each([&](int c, float4 r, double lnu) {
            double t[6];
            terms(c, r, lnu, t);
            const double wq = (t[0] + cq[0]) - cq[0];
            const uint32_t tf = __float_as_uint(r.w);
            const int slot = (int)(tf & 3u);
            for (int k = 0; k < NT; k++)
                if (slot == k) S[k] += wq;
            if (!(tf & 4u)) {
                S[NT] += wq;
                S[NT + 1] += (t[1] + cq[1]) - cq[1];
            }
            S[NT + 2] += (t[3] + cq[3]) - cq[3];
            S[NT + 3] += (t[2] + cq[2]) - cq[2];
            S[NT + 4] += (t[5] + cq[5]) - cq[5];
            S[NT + 5] += (t[4] + cq[4]) - cq[4];
        });
        for (int o = 16; o > 0; o >>= 1)
            for (int k = 0; k < NV; k++) S[k] += __shfl_xor_sync(0xffffffffu, S[k], o);
        if (lane == 0) node_write<NT>(P, m3, S, vmin, vmax, any);
    }
    fold_minmax(vmin, vmax, any, P.ctr);
}

// Start of a fused averaging call: the call's counters, the markers' averaged
// count, and the sticky-air temperature resets k_move_fused recorded.
static __global__ void k_fused_begin(MarkerView M, FusedCounters *ctr, const int32_t *__restrict__ treset, double tmp_ambient,
                              unsigned long long *navg)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctr->nguard = 0;
        ctr->any = 0;
        ctr->kmin = ~0ull;
        ctr->kmax = 0ull;
        if (navg) *navg = 0ull;  // k_cellnodes counts the averaged markers
    }
    if (!treset) return;  // applied by an earlier call on the same records
    const int32_t m = ctr->ntreset;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x)
        M.T[treset[q]] = tmp_ambient;
}

// marktmax (markmart.c:354-360) on a fused averaging call
static __global__ void k_fused_tmax(const __grid_constant__ GridView G, const __grid_constant__ MarkerView M,
                             const __grid_constant__ AvgArgsK V)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M.n; i += stride) {
        const double x = M.x[i], y = M.y[i], Tm = M.T[i];
        const int mt = M.type[i];
        if (!(x > 0 && y > 0 && x < G.xsize && y < G.ysize && Tm > 0 && mt < kAvgTypes)) continue;
        if (V.gridmod > 1 && (M.id[i] % V.gridmod) != 0) continue;
        if (mt == 0) continue;
        const double mtk = mt < 2 ? V.tmp_ambient : Tm;
        if (M.tmax[i] < mtk) M.tmax[i] = mtk;
    }
}

// the contrast clamp (markmart.c:995-1009) from the call's viscosity range
static __global__ void __launch_bounds__(256) k_fused_clamp(int64_t nn, const FusedCounters *__restrict__ ctr, double nucontr,
                                                     double *__restrict__ nu, double *__restrict__ nd,
                                                     double *__restrict__ stats)
{
    double numin = 0.0, numax = 0.0;
    if (ctr->any) {
        numin = okey_inv(ctr->kmin);
        numax = okey_inv(ctr->kmax);
    }
    if (nucontr >= 1.0) numax = numin * nucontr; else numin = numax * nucontr;
    if (blockIdx.x == 0 && threadIdx.x == 0 && stats) {
        stats[0] = numin;
        stats[1] = numax;
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t m3 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m3 < nn; m3 += stride) {
        double v = nu[m3], u = v;
        if (u < numin) u = numin;
        if (u > numax) u = numax;
        if (u != v) nu[m3] = u;
        v = nd[m3];
        u = v;
        if (u < numin) u = numin;
        if (u > numax) u = numax;
        if (u != v) nd[m3] = u;
    }
}

}  // namespace i2g
