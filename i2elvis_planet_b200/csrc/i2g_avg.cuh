// Marker -> cell averaging (the ronurecalc() marker loop, markmart.c:271-913)
// fused with the application of the cell sort, and the node loop
// (markmart.c:917-993).
//
// k_cellsums: one CTA owns a tile of cells, cell columns [c0, c0+TX) x cell rows
// [d0, d0+32).  It streams the tile column by column; a column's markers are one
// contiguous run of the cell-sorted order (cell, then caller index), reached
// through the permutation of the rank-only sort.
//   A  every thread takes markers of the run in order (gather via the
//      permutation), evaluates the property model and weights (marker_contrib)
//      into a shared-memory payload and writes the marker into its sorted slot of
//      the new device order (the sort's data movement costs no extra pass);
//   B  warp w sums corner (w & 3) of field group (w >> 2) for the column's 32
//      cells at once, one lane per cell, sequentially over that cell's markers: a
//      fixed-order segmented reduction with FP64 accumulators in registers.  The
//      payload is stored position-major with a 33-word row pitch, so the 32 lanes,
//      each at the same position of its own cell, read 32 different banks;
//   the corner sums of each cell go to global memory, field-major.
// k_nodesums: one thread per node adds the corner sums of its four cells in the
// fixed order (m1-1,m2-1), (m1-1,m2), (m1,m2-1), (m1,m2), normalises, takes
// exp()/inverse per viscmod, applies mu[] and the [nubeg, nuend] clamp and folds
// the viscosity range per block.
// No atomics touch a node value; the result does not depend on the tile shape or
// the launch configuration.
#pragma once

#include "i2g_kernels.cuh"

namespace i2g {

template <bool MIXED>
struct AvgCfg {
    using W = typename std::conditional<MIXED, float, double>::type;
    static constexpr int PM = MIXED ? 48 : 32;  // marker positions per cell held per round
    static constexpr int PITCH = 33;            // cells per position row (32 + 1 pad)
    static constexpr int CAP = PM * PITCH;
};

// dynamic shared memory of k_cellsums
template <bool MIXED>
struct AvgSmem {
    using W = typename AvgCfg<MIXED>::W;
    static constexpr int CAP = AvgCfg<MIXED>::CAP;
    W wx0[CAP], wx1[CAP], wy0[CAP], wy1[CAP];
    W pv[6][CAP];  // ro, et(beta), cp, kt, ht, tk
    double lnu[CAP];
    uint8_t flag[CAP];  // bit0: averaged, bit1: immobile type
    int32_t cs[34];     // absolute start of each cell row of the column, plus the end
    int32_t maxcnt;
};

// One tile of cells (see above).  Every thread of the CTA calls it; returns the
// number of markers this thread averaged.
template <bool MIXED>
__device__ __forceinline__ unsigned long long cellsums_tile(AvgSmem<MIXED> &S, const GridView &G, const MarkerView &A,
                                                           const MarkerView &B, const int32_t *__restrict__ perm,
                                                           const int32_t *__restrict__ cstart, const i2g_types &T,
                                                           const AvgArgsK &args, double T0,
                                                           double *__restrict__ part, int64_t tile, int32_t TX,
                                                           int32_t ntx, int64_t *slot0)
{
    using W = typename AvgCfg<MIXED>::W;
    constexpr int PM = AvgCfg<MIXED>::PM;
    constexpr int PITCH = AvgCfg<MIXED>::PITCH;
    const int64_t nc1 = G.nx - 1, nc2 = G.ny - 1, ncells = nc1 * nc2;
    const int64_t c0 = (tile % ntx) * TX, c1 = min(c0 + (int64_t)TX, nc1);
    const int64_t d0 = (tile / ntx) * 32, d1 = min(d0 + 32, nc2);
    const int NR = (int)(d1 - d0);
    __syncthreads();  // the previous tile of a persistent CTA is done with S
    const bool has_tmax = A.tmax != nullptr, has_por = A.por != nullptr, has_hi = A.hi != nullptr;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = warp & 3, grp = warp >> 2;  // corner and field group of phase B
    const int qi = q >> 1, qj = q & 1;
    unsigned long long cnt = 0;

    for (int64_t c = c0; c < c1; c++) {
        if ((int)threadIdx.x <= NR) S.cs[threadIdx.x] = cstart[c * nc2 + d0 + threadIdx.x];
        __syncthreads();
        if (warp == 0) {
            int m = lane < NR ? S.cs[lane + 1] - S.cs[lane] : 0;
            for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0) S.maxcnt = m;
        }
        __syncthreads();
        const int32_t rs = S.cs[0], re = S.cs[NR];
        const int maxcnt = S.maxcnt;
        double a[7] = {0, 0, 0, 0, 0, 0, 0};  // phase-B sums of this warp's fields, lane = cell row
        for (int P0 = 0; P0 < maxcnt; P0 += PM) {
            // ---- phase A: markers at positions [P0, P0+PM) of their cells
            for (int32_t j = rs + threadIdx.x; j < re; j += blockDim.x) {
                int lo = 0, hi = NR;  // cell row of slot j
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (S.cs[mid] <= j) lo = mid; else hi = mid;
                }
                const int p = j - S.cs[lo] - P0;
                if (p < 0 || p >= PM) continue;
                const int32_t i = perm ? __ldg(perm + j) : j;
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
                MarkerContrib mc;
                const bool ok = (args.gridmod <= 1 || (r.id % args.gridmod) == 0) &&
                                marker_contrib<MIXED>(G, T, args, T0, r, has_tmax && args.track_tmax, has_por, c,
                                                      d0 + lo, mc);
                const int t = p * PITCH + lo;
                if (ok) {
                    S.wx0[t] = (W)mc.wx0;
                    S.wx1[t] = (W)mc.wx1;
                    S.wy0[t] = (W)mc.wy0;
                    S.wy1[t] = (W)mc.wy1;
                    S.pv[0][t] = (W)mc.mro;
                    S.pv[1][t] = (W)mc.mbb;
                    S.pv[2][t] = (W)mc.mcp;
                    S.pv[3][t] = (W)mc.mkt;
                    S.pv[4][t] = (W)mc.mht;
                    S.pv[5][t] = (W)mc.mtk;
                    S.lnu[t] = mc.lnu;
                    S.flag[t] = 1 | (mc.immobile ? 2 : 0);
                    cnt++;
                } else {
                    S.flag[t] = 0;
                }
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
            }
            __syncthreads();
            // ---- phase B: lane = cell row, sequential over the cell's positions
            if (lane < NR) {
                const int n = min(S.cs[lane + 1] - S.cs[lane] - P0, PM);
                for (int p = 0; p < n; p++) {
                    const int k = p * PITCH + lane;
                    const uint8_t fl = S.flag[k];
                    if (!(fl & 1)) continue;
                    const W wx = qi ? S.wx1[k] : S.wx0[k];
                    const W wy = qj ? S.wy1[k] : S.wy0[k];
                    if (!MIXED) {
                        const double swt = 1.0 * (double)wx * (double)wy;
                        if (grp == 0) {
                            a[0] += (double)S.pv[0][k] * swt;
                            a[1] += swt;
                            a[2] += (double)S.pv[1][k] * swt;
                            a[3] += (double)S.pv[2][k] * swt;
                            a[4] += (double)S.pv[3][k] * swt;
                        } else {
                            a[0] += (double)S.pv[4][k] * swt;
                            if (!(fl & 2)) {
                                a[1] += (double)S.pv[5][k] * swt;
                                a[2] += swt;
                            }
                            if (wx > 0.5 && wy > 0.5) {
                                const double swt2 = 1.0 * 4.0 * ((double)wx - 0.5) * ((double)wy - 0.5);
                                a[3] += S.lnu[k] * swt2;
                                a[4] += swt2;
                            }
                            if (q == 0) {
                                const double ddx = 1.0 - fabs((double)S.wx0[k] - 0.5);
                                const double ddy = 1.0 - fabs((double)S.wy0[k] - 0.5);
                                if (ddx > 0.5 && ddy > 0.5) {
                                    const double swt2 = 1.0 * 4.0 * (ddx - 0.5) * (ddy - 0.5);
                                    a[5] += S.lnu[k] * swt2;
                                    a[6] += swt2;
                                }
                            }
                        }
                    } else {
                        const float swt = (float)wx * (float)wy;
                        if (grp == 0) {
                            a[0] += (double)((float)S.pv[0][k] * swt);
                            a[1] += (double)swt;
                            a[2] += (double)((float)S.pv[1][k] * swt);
                            a[3] += (double)((float)S.pv[2][k] * swt);
                            a[4] += (double)((float)S.pv[3][k] * swt);
                        } else {
                            a[0] += (double)((float)S.pv[4][k] * swt);
                            if (!(fl & 2)) {
                                a[1] += (double)((float)S.pv[5][k] * swt);
                                a[2] += (double)swt;
                            }
                            if (wx > 0.5f && wy > 0.5f) {
                                const float swt2 = 4.0f * ((float)wx - 0.5f) * ((float)wy - 0.5f);
                                a[3] += S.lnu[k] * (double)swt2;
                                a[4] += (double)swt2;
                            }
                            if (q == 0) {
                                const double ddx = 1.0 - fabs((double)S.wx0[k] - 0.5);
                                const double ddy = 1.0 - fabs((double)S.wy0[k] - 0.5);
                                if (ddx > 0.5 && ddy > 0.5) {
                                    const double swt2 = (double)(4.0f * (float)(ddx - 0.5) * (float)(ddy - 0.5));
                                    a[5] += S.lnu[k] * swt2;
                                    a[6] += swt2;
                                }
                            }
                        }
                    }
                }
            }
            __syncthreads();
        }
        // corner sums of the column's cells, field-major [kPart][ncells]
        if (lane < NR) {
            double *d = part + c * nc2 + d0 + lane;
            if (grp == 0) {
                d[(q * 10 + F_RO) * ncells] = a[0];
                d[(q * 10 + F_W0) * ncells] = a[1];
                d[(q * 10 + F_ET) * ncells] = a[2];
                d[(q * 10 + F_CP) * ncells] = a[3];
                d[(q * 10 + F_KT) * ncells] = a[4];
            } else {
                d[(q * 10 + F_HT) * ncells] = a[0];
                d[(q * 10 + F_TK) * ncells] = a[1];
                d[(q * 10 + F_W1) * ncells] = a[2];
                d[(q * 10 + F_NU) * ncells] = a[3];
                d[(q * 10 + F_WNU) * ncells] = a[4];
                if (q == 0) {
                    d[40 * ncells] = a[5];
                    d[41 * ncells] = a[6];
                }
            }
        }
    }
    return cnt;
}


template <bool MIXED>
__global__ void __launch_bounds__(256, 2) k_cellsums(GridView G, MarkerView A, MarkerView B,
                                                     const int32_t *__restrict__ perm,
                                                     const int32_t *__restrict__ cstart,
                                                     const DevTypes *__restrict__ Ty, AvgArgsK args,
                                                     const double *__restrict__ T0p, double *__restrict__ part,
                                                     int32_t TX, int32_t ntx, unsigned long long *navg,
                                                     int64_t *slot0)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    AvgSmem<MIXED> &S = *reinterpret_cast<AvgSmem<MIXED> *>(smraw);
    unsigned long long cnt =
        cellsums_tile<MIXED>(S, G, A, B, perm, cstart, Ty->t, args, *T0p, part, blockIdx.x, TX, ntx, slot0);
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && navg && cnt) atomicAdd(navg, cnt);
}

}  // namespace i2g
