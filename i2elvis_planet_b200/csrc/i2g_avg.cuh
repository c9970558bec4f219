// Marker -> cell averaging (the ronurecalc() marker loop, markmart.c:271-913) in
// two kernels, and the node loop (markmart.c:917-993) in i2g_nodes.cuh.
//
// k_contrib: one thread per slot of the new, cell-sorted device order (cell,
//   then caller index).  It gathers the slot's marker from the current order
//   through the sort permutation (markers move less than a cell per step, so the
//   gathers are nearly local), evaluates the property model and the marker's
//   bilinear weights (marker_contrib), and writes the marker record (the sort's
//   data movement costs no extra pass) and its contribution (the payload) to the
//   slot: coalesced stores.
// k_cellsums: the per-cell corner sums, one warp per column strip of 32 cells
//   (see cellsums_tile): each lane adds its cell's markers in slot order into
//   FP64 registers, a fixed-order segmented reduction.
// No atomics touch a node value; the result does not depend on the tile shape,
// the launch configuration or the device order the markers arrive in.
#pragma once

#include "i2g_kernels.cuh"
#include "i2g_launch.h"

namespace i2g {

template <bool MIXED>
struct AvgCfg {
    using W = typename std::conditional<MIXED, float, double>::type;  // weights, property values
};

// The averaging payload of every marker, in its slot of the sorted order:
// structure of arrays carved from one buffer of payload_bytes(MIXED, cap) bytes.
//   FP64 form: wx0 wx1 wy0 wy1 pv[6] lnu   (double each), meta (byte)
//   mixed:     lnu (double), wx1 wy1 pv[6] (float each),    meta (byte)
//   pv = ro, et (beta), cp, kt, ht, tk: the property values the sums weight;
//   the mixed form's w0 is 1.0f - w1 exactly (fdw32), so it is not stored.
//   meta: bit0 averaged, bit1 immobile type.

template <bool MIXED>
struct PayloadView {
    using W = typename AvgCfg<MIXED>::W;
    W *wx0, *wx1, *wy0, *wy1;  // wx0, wy0: FP64 form only
    W *pv;                     // field f at pv + f * stride
    double *lnu;
    uint8_t *meta;
    int64_t stride;

    __host__ __device__ static PayloadView make(void *base, int64_t cap)
    {
        PayloadView P{};
        const int64_t s = payload_cap(cap);
        P.stride = s;
        if (MIXED) {
            P.lnu = (double *)base;
            P.wx1 = (W *)(P.lnu + s);
            P.wy1 = P.wx1 + s;
            P.pv = P.wy1 + s;
            P.meta = (uint8_t *)(P.pv + 6 * s);
        } else {
            P.wx0 = (W *)base;
            P.wx1 = P.wx0 + s;
            P.wy0 = P.wx1 + s;
            P.wy1 = P.wy0 + s;
            P.pv = P.wy1 + s;
            P.lnu = (double *)(P.pv + 6 * s);
            P.meta = (uint8_t *)(P.lnu + s);
        }
        return P;
    }
};

// Slot j of the sorted order: the marker perm[j] of the current order (j itself
// when perm is NULL: the order is sorted already) -- property model at its cell,
// record and payload into slot j.
template <bool MIXED>
__device__ __forceinline__ void contrib_marker(const GridView &G, const MarkerView &A, const MarkerView &B,
                                               const int32_t *__restrict__ perm, const i2g_types &T,
                                               const AvgArgsK &args, double T0, const PayloadView<MIXED> &P,
                                               int64_t j, int64_t *slot0)
{
    using W = typename AvgCfg<MIXED>::W;
    const bool has_tmax = A.tmax != nullptr, has_por = A.por != nullptr, has_hi = A.hi != nullptr;
    const int64_t i = perm ? (int64_t)__ldg(perm + j) : j;
    MarkerRec r;
    r.x = A.x[i];
    r.y = A.y[i];
    r.T = A.T[i];
    r.eta = A.eta[i];
    r.p = A.p[i];
    r.type = A.type[i];
    r.id = A.id[i];
    r.tmax = has_tmax ? A.tmax[i] : 0.0;
    r.hi = has_hi ? A.hi[i] : 0.0;
    r.por = has_por ? A.por[i] : 0.0;
    // the marker's cell: the cell the sort filed it under (cell_key)
    double xc = r.x, yc = r.y;
    clampxy(G, xc, yc);
    const int64_t m10 = cell_search(G.gx, G.nx, G.inv_x, xc), m20 = cell_search(G.gy, G.ny, G.inv_y, yc);
    MarkerContrib mc;
    const bool ok = (args.gridmod <= 1 || (r.id % args.gridmod) == 0) && r.type >= 0 &&
                    marker_contrib<MIXED>(G, T, args, T0, r, has_tmax && args.track_tmax, has_por, m10, m20, mc);
    B.x[j] = r.x;
    B.y[j] = r.y;
    B.T[j] = r.T;
    B.eta[j] = r.eta;
    B.p[j] = r.p;
    B.type[j] = (int8_t)r.type;
    B.id[j] = r.id;
    if (has_tmax) B.tmax[j] = r.tmax;
    if (has_hi) B.hi[j] = r.hi;
    if (has_por) B.por[j] = r.por;
    if (r.id == 0) *slot0 = j;
    P.meta[j] = (uint8_t)((ok ? 1 : 0) | (ok && mc.immobile ? 2 : 0));
    if (ok) {
        if (!MIXED) {
            P.wx0[j] = (W)mc.wx0;
            P.wy0[j] = (W)mc.wy0;
        }
        P.wx1[j] = (W)mc.wx1;
        P.wy1[j] = (W)mc.wy1;
        const int64_t s = P.stride;
        P.pv[j] = (W)mc.mro;
        P.pv[j + s] = (W)mc.mbb;
        P.pv[j + 2 * s] = (W)mc.mcp;
        P.pv[j + 3 * s] = (W)mc.mkt;
        P.pv[j + 4 * s] = (W)mc.mht;
        P.pv[j + 5 * s] = (W)mc.mtk;
        P.lnu[j] = mc.lnu;
    }
}

template <bool MIXED>
__global__ void __launch_bounds__(256, 4) k_contrib(GridView G, MarkerView A, MarkerView B,
                                                    const int32_t *__restrict__ perm, const DevTypes *__restrict__ Ty,
                                                    AvgArgsK args, const double *__restrict__ T0p, void *payload,
                                                    int64_t pcap, int64_t *slot0)
{
    const PayloadView<MIXED> P = PayloadView<MIXED>::make(payload, pcap);
    const double T0 = *T0p;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < A.n; j += stride)
        contrib_marker<MIXED>(G, A, B, perm, Ty->t, args, T0, P, j, slot0);
}

// k_cellsums: one warp per column strip of 32 cells (lane = cell row); each lane
// keeps all kPart corner sums of its cell in FP64 registers.  The warp stages its
// strip's payload in chunks of PC positions into its own shared buffer, element
// (row, t) at row * RP + t: coalesced global reads (the PC slots of a cell are
// contiguous), conflict-free reads by cell row (RP odd).  Then every lane adds the
// chunk's markers of its cell in position order.  No block-wide barriers.
template <bool MIXED>
struct StripCfg {
    static constexpr int PC = MIXED ? 8 : 2;  // positions per chunk
    static constexpr int RP = PC + 1;         // row pitch (odd)
    static constexpr int N = 32 * RP;
};

template <bool MIXED>
struct StripBuf {
    using W = typename AvgCfg<MIXED>::W;
    static constexpr int N = StripCfg<MIXED>::N, N0 = MIXED ? 1 : StripCfg<MIXED>::N;
    double lnu[N];
    W wx0[N0], wx1[N], wy0[N0], wy1[N];  // w0: FP64 form only (the mixed w0 is 1.0f - w1)
    W pv[6][N];                          // ro, et(beta), cp, kt, ht, tk
    uint8_t flag[N];                     // bit0: averaged, bit1: immobile type
};

// dynamic shared memory of k_cellsums: one strip buffer per warp
template <bool MIXED>
struct AvgSmem {
    StripBuf<MIXED> w[8];
};

// the kPart corner sums of one marker into a cell's accumulators (field-major
// index q * 10 + F_*, then 40, 41 for the cell-centre nd), markmart.c:859-913
template <bool MIXED>
__device__ __forceinline__ void add_marker(double (&a)[kPart], const StripBuf<MIXED> &B, int k)
{
    using W = typename AvgCfg<MIXED>::W;
    const uint8_t fl = B.flag[k];
    if (!(fl & 1)) return;
    const W wx1 = B.wx1[k], wy1 = B.wy1[k];
    const W wx0 = MIXED ? (W)(1.0f - (float)wx1) : B.wx0[k];
    const W wy0 = MIXED ? (W)(1.0f - (float)wy1) : B.wy0[k];
    const W p0 = B.pv[0][k], p1 = B.pv[1][k], p2 = B.pv[2][k], p3 = B.pv[3][k], p4 = B.pv[4][k], p5 = B.pv[5][k];
    const double lnu = B.lnu[k];
    const bool mobile = !(fl & 2);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const W wx = (q >> 1) ? wx1 : wx0;
        const W wy = (q & 1) ? wy1 : wy0;
        double *c = a + q * 10;
        if (!MIXED) {
            const double swt = 1.0 * (double)wx * (double)wy;
            c[F_RO] += (double)p0 * swt;
            c[F_W0] += swt;
            c[F_ET] += (double)p1 * swt;
            c[F_CP] += (double)p2 * swt;
            c[F_KT] += (double)p3 * swt;
            c[F_HT] += (double)p4 * swt;
            if (mobile) {
                c[F_TK] += (double)p5 * swt;
                c[F_W1] += swt;
            }
            if (wx > 0.5 && wy > 0.5) {
                const double swt2 = 1.0 * 4.0 * ((double)wx - 0.5) * ((double)wy - 0.5);
                c[F_NU] += lnu * swt2;
                c[F_WNU] += swt2;
            }
        } else {
            const float swt = (float)wx * (float)wy;
            const double dswt = (double)swt;
            c[F_RO] += (double)((float)p0 * swt);
            c[F_W0] += dswt;
            c[F_ET] += (double)((float)p1 * swt);
            c[F_CP] += (double)((float)p2 * swt);
            c[F_KT] += (double)((float)p3 * swt);
            c[F_HT] += (double)((float)p4 * swt);
            if (mobile) {
                c[F_TK] += (double)((float)p5 * swt);
                c[F_W1] += dswt;
            }
            if (wx > 0.5f && wy > 0.5f) {
                const float swt2 = 4.0f * ((float)wx - 0.5f) * ((float)wy - 0.5f);
                c[F_NU] += lnu * (double)swt2;
                c[F_WNU] += (double)swt2;
            }
        }
    }
    const double ddx = 1.0 - fabs((double)wx0 - 0.5);
    const double ddy = 1.0 - fabs((double)wy0 - 0.5);
    if (ddx > 0.5 && ddy > 0.5) {
        const double swt2 = MIXED ? (double)(4.0f * (float)(ddx - 0.5) * (float)(ddy - 0.5))
                                  : 1.0 * 4.0 * (ddx - 0.5) * (ddy - 0.5);
        a[40] += lnu * swt2;
        a[41] += swt2;
    }
}

// One tile of cells (cell columns [c0, c0+TX) x rows [d0, d0+32)) by the CTA's
// warps, a column strip each at a time.  The grid has nc1 x nc2 cells; the tile
// is column block (tile % ntx), row block (tile / ntx).  Returns the number of
// averaged markers this thread counted.
template <bool MIXED>
__device__ __forceinline__ unsigned cellsums_tile(AvgSmem<MIXED> &S, const PayloadView<MIXED> &P,
                                                  const int32_t *__restrict__ cstart, int64_t nc1, int64_t nc2,
                                                  double *__restrict__ part, int64_t tile, int32_t TX, int32_t ntx)
{
    constexpr int PC = StripCfg<MIXED>::PC;
    constexpr int RP = StripCfg<MIXED>::RP;
    const int64_t ncells = nc1 * nc2;
    const int64_t c0 = (tile % ntx) * TX, c1 = min(c0 + (int64_t)TX, nc1);
    const int64_t d0 = (tile / ntx) * 32;
    const int NR = (int)min((int64_t)32, nc2 - d0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    StripBuf<MIXED> &B = S.w[warp];
    const int64_t s = P.stride;
    unsigned cnt = 0;
    for (int64_t c = c0 + warp; c < c1; c += nwarps) {
        const int64_t cell = c * nc2 + d0 + lane;
        int32_t cb = 0, cn = 0;
        if (lane < NR) {
            cb = __ldg(cstart + cell);
            cn = __ldg(cstart + cell + 1) - cb;
        }
        int maxc = cn;
        for (int o = 16; o > 0; o >>= 1) maxc = max(maxc, __shfl_xor_sync(0xffffffffu, maxc, o));
        double a[kPart];
#pragma unroll
        for (int u = 0; u < kPart; u++) a[u] = 0.0;
        for (int P0 = 0; P0 < maxc; P0 += PC) {
            __syncwarp();  // the previous chunk is consumed
            // stage positions [P0, P0+PC) of the strip's cells: element e = row x PC + t
#pragma unroll
            for (int e0 = 0; e0 < 32 * PC; e0 += 32) {
                const int e = e0 + lane, row = e / PC, t = e % PC;
                const int32_t b = __shfl_sync(0xffffffffu, cb, row), n = __shfl_sync(0xffffffffu, cn, row);
                if (P0 + t >= n) continue;
                const int64_t j = (int64_t)b + P0 + t;
                const int k = row * RP + t;
                const uint8_t meta = __ldg(P.meta + j);
                B.flag[k] = meta & 3;
                cnt += meta & 1;
                if (!MIXED) {
                    B.wx0[k] = __ldg(P.wx0 + j);
                    B.wy0[k] = __ldg(P.wy0 + j);
                }
                B.wx1[k] = __ldg(P.wx1 + j);
                B.wy1[k] = __ldg(P.wy1 + j);
#pragma unroll
                for (int u = 0; u < 6; u++) B.pv[u][k] = __ldg(P.pv + j + u * s);
                B.lnu[k] = __ldg(P.lnu + j);
            }
            __syncwarp();
            const int m = min(PC, cn - P0);
            for (int t = 0; t < m; t++) add_marker<MIXED>(a, B, lane * RP + t);
        }
        if (lane < NR) {
            double *d = part + cell;
#pragma unroll
            for (int u = 0; u < kPart; u++) d[u * ncells] = a[u];
        }
    }
    return cnt;
}

// per-warp sum of the counts into *navg
__device__ __forceinline__ void add_count(unsigned cnt, unsigned long long *navg)
{
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && navg && cnt) atomicAdd(navg, (unsigned long long)cnt);
}

template <bool MIXED>
__global__ void __launch_bounds__(256, 2) k_cellsums(void *payload, int64_t pcap, const int32_t *__restrict__ cstart,
                                                     int64_t nc1, int64_t nc2, double *__restrict__ part, int32_t TX,
                                                     int32_t ntx, unsigned long long *navg)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    AvgSmem<MIXED> &S = *reinterpret_cast<AvgSmem<MIXED> *>(smraw);
    add_count(cellsums_tile<MIXED>(S, PayloadView<MIXED>::make(payload, pcap), cstart, nc1, nc2, part, blockIdx.x,
                                   TX, ntx),
              navg);
}

}  // namespace i2g
