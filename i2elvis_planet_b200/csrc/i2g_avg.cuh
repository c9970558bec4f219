// Streaming marker -> node averaging (the ronurecalc() marker and node loops,
// markmart.c:271-993) fused with the application of the cell sort.
//
// One CTA owns a tile of nodes: node columns [a0, a1) x node rows [b0, b0+TYN).
// Node (m1, m2) receives from cells (m1-1..m1, m2-1..m2), so the CTA streams the
// cell columns a0-1 .. a1-1 over cell rows b0-1 .. b0+TYN-1 (TYN+1 <= 32 rows):
// the halo column/row is recomputed, never written.  Markers are visited in the
// cell-sorted order (cell, then caller index) through the permutation of the
// rank-only sort; the CTA writes the markers of the cells it owns into that order
// (the new device order), so the sort's data movement costs no extra pass.
//
// Per cell column:
//   A  every thread takes markers (gather via the permutation), evaluates the
//      property model and weights (marker_contrib) into a shared-memory payload,
//      and writes owned markers to their sorted slot;
//   B  warp w sums corner (w & 3) of field group (w >> 2) for 32 cells at once, one
//      lane per cell, sequentially over that cell's markers: a fixed-order
//      (deterministic) segmented reduction with FP64 accumulators in registers;
//   C  once cell columns c-1 and c are summed, node column c adds its four cells'
//      corner sums in the fixed order (c-1,r-1), (c-1,r), (c,r-1), (c,r),
//      normalises and writes the node fields.
// No global atomics touch a node value; the result does not depend on the tile
// shape or the launch configuration.
#pragma once

#include "i2g_kernels.cuh"

namespace i2g {

template <bool MIXED>
struct AvgCfg {
    using W = typename std::conditional<MIXED, float, double>::type;
    static constexpr int CAP = MIXED ? 1536 : 1024;  // payload markers per chunk
};

// dynamic shared memory of k_avg
template <bool MIXED>
struct AvgSmem {
    using W = typename AvgCfg<MIXED>::W;
    static constexpr int CAP = AvgCfg<MIXED>::CAP;
    W wx0[CAP], wx1[CAP], wy0[CAP], wy1[CAP];
    W pv[6][CAP];  // ro, et(beta), cp, kt, ht, tk
    double lnu[CAP];
    uint8_t flag[CAP];  // bit0: averaged, bit1: immobile type
    uint8_t row[CAP];   // cell row of each payload slot
    double acc[2][32][kPart];  // corner sums of two cell columns
    int32_t cs[34];            // run-relative start of each cell row
    double rmin[8], rmax[8];
    int rany[8];
};

__device__ __forceinline__ void mm_fold(double &vmin, double &vmax, int &any, double v)
{
    if (!any) { vmin = vmax = v; any = 1; }
    else { vmin = fmin(vmin, v); vmax = fmax(vmax, v); }
}

template <bool MIXED>
__global__ void __launch_bounds__(256, 2) k_avg(GridView G, MarkerView A, MarkerView B,
                                                const int32_t *__restrict__ perm, const int32_t *__restrict__ cstart,
                                                const DevTypes *__restrict__ Ty, AvgArgsK args,
                                                const double *__restrict__ T0p, NodeOut O, double *__restrict__ mmpart,
                                                int32_t TX, int32_t TYN, int32_t ntx, unsigned long long *navg,
                                                int64_t *slot0)
{
    using W = typename AvgCfg<MIXED>::W;
    constexpr int CAP = AvgCfg<MIXED>::CAP;
    extern __shared__ __align__(16) unsigned char smraw[];
    AvgSmem<MIXED> &S = *reinterpret_cast<AvgSmem<MIXED> *>(smraw);
    const i2g_types &T = Ty->t;
    const int64_t nx = G.nx, ny = G.ny, nc1 = nx - 1, nc2 = ny - 1;
    const int64_t tx = blockIdx.x % ntx, ty = blockIdx.x / ntx;
    const int64_t a0 = tx * TX, a1 = min(a0 + (int64_t)TX, nx);
    const int64_t b0 = ty * TYN, b1 = min(b0 + (int64_t)TYN, ny);
    const int64_t dlo = max(b0 - 1, (int64_t)0), dhi = min(b1 - 1, nc2 - 1);
    const int NR = (int)(dhi - dlo + 1);  // cell rows streamed (<= 32)
    const double T0 = *T0p;
    const bool has_tmax = A.tmax != nullptr, has_por = A.por != nullptr, has_hi = A.hi != nullptr;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = warp & 3, grp = warp >> 2;  // corner and field group handled in phase B
    const int qi = q >> 1, qj = q & 1;
    double vmin = 0, vmax = 0;
    int any = 0;
    unsigned long long cnt = 0;
    const int64_t cfirst = max(a0 - 1, (int64_t)0), clast = min(a1 - 1, nc1 - 1);

    for (int64_t c = cfirst; c <= clast; c++) {
        const int slot = (int)(c & 1);
        for (int r = threadIdx.x; r <= NR; r += blockDim.x) S.cs[r] = cstart[c * nc2 + dlo + r];
        __syncthreads();
        const int32_t rs = S.cs[0], re = S.cs[NR];
        // first slot this CTA owns in the column (owned cells: column >= a0, row >= b0)
        int32_t own_from = re;
        if (c >= a0 && b0 <= dhi) own_from = S.cs[b0 - dlo];
        // phase-B accumulators: lane = cell row, 7 FP64 sums (group 0 uses 5)
        double a[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int32_t base = rs; base < re; base += CAP) {
            const int nch = (int)min((int32_t)CAP, re - base);
            // cell row of every slot of the chunk
            for (int r = warp; r < NR; r += 8) {
                const int32_t k0 = max(S.cs[r], base) - base, k1 = min(S.cs[r + 1], base + nch) - base;
                for (int32_t k = k0 + lane; k < k1; k += 32) S.row[k] = (uint8_t)r;
            }
            __syncthreads();
            // ---- phase A: gather, property model, payload, sorted write-back.
            // The next marker's record is loaded before the current one is
            // processed, so two gathers are in flight per thread.
            auto load_rec = [&](int t, MarkerRec &r) {
                const int32_t j = base + t;
                const int32_t i = perm ? __ldg(perm + j) : j;
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
            };
            MarkerRec nxt;
            if ((int)threadIdx.x < nch) load_rec(threadIdx.x, nxt);
            for (int t = threadIdx.x; t < nch; t += blockDim.x) {
                MarkerRec r = nxt;
                if (t + (int)blockDim.x < nch) load_rec(t + blockDim.x, nxt);
                const int32_t j = base + t;
                const int lo = S.row[t];
                MarkerContrib mc;
                bool ok = (args.gridmod <= 1 || (r.id % args.gridmod) == 0) &&
                          marker_contrib<MIXED>(G, T, args, T0, r, has_tmax && args.track_tmax, has_por, c,
                                                dlo + lo, mc);
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
                if (j >= own_from) {
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
            }
            __syncthreads();
            // ---- phase B: per-cell sequential sums, lane = cell row
            if (lane < NR) {
                const int32_t k0 = max(S.cs[lane], base) - base;
                const int32_t k1 = min(S.cs[lane + 1], base + nch) - base;
                for (int32_t k = k0; k < k1; k++) {
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
        // store this column's cell corner sums (field layout of kPart)
        if (lane < NR) {
            double *d = S.acc[slot][lane];
            if (grp == 0) {
                d[q * 10 + F_RO] = a[0];
                d[q * 10 + F_W0] = a[1];
                d[q * 10 + F_ET] = a[2];
                d[q * 10 + F_CP] = a[3];
                d[q * 10 + F_KT] = a[4];
            } else {
                d[q * 10 + F_HT] = a[0];
                d[q * 10 + F_TK] = a[1];
                d[q * 10 + F_W1] = a[2];
                d[q * 10 + F_NU] = a[3];
                d[q * 10 + F_WNU] = a[4];
                if (q == 0) {
                    d[40] = a[5];
                    d[41] = a[6];
                }
            }
        }
        __syncthreads();
        // ---- phase C: node column c (cells c-1 and c), then node column nx-1 at the edge.
        // One work item per (node, output field): the divisions and exp() of the
        // normalisation run in parallel across the CTA.
        for (int pass = 0; pass < 2; pass++) {
            const int64_t m1 = c + pass;
            if (pass == 0 && c < a0) continue;
            if (pass == 1 && !(c == nc1 - 1 && a1 == nx)) continue;
            const int nrows = (int)(b1 - b0);
            for (int w = threadIdx.x; w < nrows * 8; w += blockDim.x) {
                const int fld = w & 7;
                const int64_t m2 = b0 + (w >> 3);
                const int64_t m3 = m1 * ny + m2;
                if (fld == 7) {
                    // normal viscosity at the centre of cell (m1-1, m2-1) (markmart.c:859-872)
                    double snd = 0.0, swnd = 0.0;
                    if (m1 >= 1 && m2 >= 1) {
                        const double *src = S.acc[(m1 - 1) & 1][m2 - 1 - dlo];
                        snd += src[40];
                        swnd += src[41];
                    }
                    if (swnd) {
                        const double mu = G.mu ? __ldg(G.mu + m3) : 0.0;
                        double v;
                        if (mu) v = mu;
                        else {
                            v = snd / swnd;
                            if (args.viscmod == 1) v = exp(v);
                            if (args.viscmod == 2) v = 1.0 / v;
                        }
                        if (v < args.nubeg) v = args.nubeg;
                        if (v > args.nuend) v = args.nuend;
                        mm_fold(vmin, vmax, any, v);
                        O.nd[m3] = v;
                        O.po[m3] = 0.0; /* po0[] is never accumulated (markmart.c:968) */
                    }
                    continue;
                }
                // numerator / weight fields of this output, summed over the four cells
                // in the fixed order (m1-1,m2-1), (m1-1,m2), (m1,m2-1), (m1,m2)
                const int fn = fld == 5 ? F_TK : (fld == 6 ? F_NU : fld);
                const int fw = fld == 5 ? F_W1 : (fld == 6 ? F_WNU : F_W0);
                double sn = 0.0, sw = 0.0, s0 = 0.0;
#pragma unroll
                for (int qq = 0; qq < 4; qq++) {
                    const int64_t c1 = m1 - 1 + (qq >> 1), c2 = m2 - 1 + (qq & 1);
                    if (c1 < 0 || c2 < 0 || c1 > nc1 - 1 || c2 > nc2 - 1) continue;
                    const double *src = S.acc[c1 & 1][c2 - dlo] + (3 - qq) * 10;
                    sn += src[fn];
                    sw += src[fw];
                    s0 += src[F_W0];
                }
                if (fld == 6) {
                    if (sw) {
                        const double mu = G.mu ? __ldg(G.mu + m3) : 0.0;
                        double v;
                        if (mu) v = mu;
                        else {
                            v = sn / sw;
                            if (args.viscmod == 1) v = exp(v);
                            if (args.viscmod == 2) v = 1.0 / v;
                        }
                        if (v < args.nubeg) v = args.nubeg;
                        if (v > args.nuend) v = args.nuend;
                        mm_fold(vmin, vmax, any, v);
                        O.nu[m3] = v;
                    }
                } else if (s0) {  // node touched by markers (markmart.c:978)
                    if (fld == 5) {
                        if (sw) O.tk[m3] = sn / sw;
                    } else {
                        double *dst = fld == 0 ? O.ro : fld == 1 ? O.et : fld == 2 ? O.cp : fld == 3 ? O.kt : O.ht;
                        dst[m3] = sn / sw;
                    }
                }
            }
        }
        __syncthreads();
    }
    // ---- per-CTA viscosity range and averaged-marker count
    for (int o = 16; o > 0; o >>= 1) {
        const double a2 = __shfl_down_sync(0xffffffffu, vmin, o), b2 = __shfl_down_sync(0xffffffffu, vmax, o);
        const int c2 = __shfl_down_sync(0xffffffffu, any, o);
        if (c2) {
            if (!any) { vmin = a2; vmax = b2; any = 1; }
            else { vmin = fmin(vmin, a2); vmax = fmax(vmax, b2); }
        }
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    if (lane == 0) {
        S.rmin[warp] = vmin;
        S.rmax[warp] = vmax;
        S.rany[warp] = any;
        if (navg && cnt) atomicAdd(navg, cnt);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x0 = 0, x1 = 0;
        int c0 = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            if (!S.rany[w]) continue;
            if (!c0) { x0 = S.rmin[w]; x1 = S.rmax[w]; c0 = 1; }
            else { x0 = fmin(x0, S.rmin[w]); x1 = fmax(x1, S.rmax[w]); }
        }
        mmpart[3 * blockIdx.x + 0] = x0;
        mmpart[3 * blockIdx.x + 1] = x1;
        mmpart[3 * blockIdx.x + 2] = c0;
    }
}

}  // namespace i2g
