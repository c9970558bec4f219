// Node loop of ronurecalc() (markmart.c:917-1009): k_nodesums (fixed-order
// combination of the cell corner sums, normalisation, viscosity limits) and the
// contrast clamp.  Included by one translation unit only (i2g_fp64.cu, built
// with --fmad=false).
#pragma once

#include "i2g_avg.cuh"

namespace i2g {

// ----------------------------------------------------------------- node loop
__device__ __forceinline__ void mm_fold(double &vmin, double &vmax, int &any, double v)
{
    if (!any) { vmin = vmax = v; any = 1; }
    else { vmin = fmin(vmin, v); vmax = fmax(vmax, v); }
}

// One node of the node loop (markmart.c:917-993): its four cells' corner sums in
// the fixed order (m1-1,m2-1), (m1-1,m2), (m1,m2-1), (m1,m2), normalised.
__device__ __forceinline__ void node_finalize(const GridView &G, const double *__restrict__ part,
                                              const AvgArgsK &args, const NodeOut &O, int64_t m3, double &vmin,
                                              double &vmax, int &any)
{
    const int64_t nx = G.nx, ny = G.ny, nc2 = ny - 1, ncells = (nx - 1) * nc2;
    const int64_t m1 = m3 / ny, m2 = m3 - m1 * ny;
    double s[10];
#pragma unroll
    for (int f = 0; f < 10; f++) s[f] = 0.0;
#pragma unroll
    for (int qq = 0; qq < 4; qq++) {
        const int64_t c1 = m1 - 1 + (qq >> 1), c2 = m2 - 1 + (qq & 1);
        if (c1 < 0 || c2 < 0 || c1 > nx - 2 || c2 > ny - 2) continue;
        const double *src = part + (int64_t)((3 - qq) * 10) * ncells + c1 * nc2 + c2;
#pragma unroll
        for (int f = 0; f < 10; f++) s[f] += __ldg(src + (int64_t)f * ncells);
    }
    double snd = 0.0, swnd = 0.0;
    if (m1 >= 1 && m2 >= 1) {
        const int64_t cc = (m1 - 1) * nc2 + (m2 - 1);
        snd += __ldg(part + 40 * ncells + cc);
        swnd += __ldg(part + 41 * ncells + cc);
    }
    const double mu = G.mu ? __ldg(G.mu + m3) : 0.0;
    if (s[F_WNU]) {
        double v;
        if (mu) v = mu;
        else {
            v = s[F_NU] / s[F_WNU];
            if (args.viscmod == 1) v = exp(v);
            if (args.viscmod == 2) v = 1.0 / v;
        }
        if (v < args.nubeg) v = args.nubeg;
        if (v > args.nuend) v = args.nuend;
        mm_fold(vmin, vmax, any, v);
        O.nu[m3] = v;
    }
    if (swnd) {
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
    if (O.w1) O.w1[m3] = s[F_W1];
    if (s[F_W0]) {
        O.ro[m3] = s[F_RO] / s[F_W0];
        O.et[m3] = s[F_ET] / s[F_W0];
        O.cp[m3] = s[F_CP] / s[F_W0];
        O.kt[m3] = s[F_KT] / s[F_W0];
        O.ht[m3] = s[F_HT] / s[F_W0];
        if (s[F_W1]) O.tk[m3] = s[F_TK] / s[F_W1];
    }
}

// {min, max, any} over the CTA; thread 0 writes it to out[0..2]
__device__ __forceinline__ void block_fold(double vmin, double vmax, int any, double *__restrict__ out)
{
    __shared__ double smin[32], smax[32];
    __shared__ int sany[32];
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
        double x0 = 0, x1 = 0;
        int c0 = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
            if (!sany[i]) continue;
            if (!c0) { x0 = smin[i]; x1 = smax[i]; c0 = 1; }
            else { x0 = fmin(x0, smin[i]); x1 = fmax(x1, smax[i]); }
        }
        out[0] = x0;
        out[1] = x1;
        out[2] = c0;
    }
}

static __global__ void __launch_bounds__(256) k_nodesums(const __grid_constant__ GridView G,
                                                         const double *__restrict__ part,
                                                         const __grid_constant__ AvgArgsK args, NodeOut O,
                                                         double *__restrict__ mmpart)
{
    double vmin = 0, vmax = 0;
    int any = 0;
    const int64_t m3 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m3 < G.nx * G.ny) node_finalize(G, part, args, O, m3, vmin, vmax, any);
    block_fold(vmin, vmax, any, mmpart + 3 * blockIdx.x);
}

// Contrast clamp (markmart.c:995-1009): the CTA folds the per-block viscosity
// ranges (exact and order-free), derives {numin, numax} and clamps nodes
// [lo, hi) with the given stride.
__device__ __forceinline__ void clamp_nodes(const double *__restrict__ mmpart, int32_t nparts, double nucontr,
                                            double *__restrict__ nu, double *__restrict__ nd, int64_t lo, int64_t hi,
                                            int64_t stride, double *__restrict__ stats)
{
    __shared__ double smin[32], smax[32], lim[2];
    __shared__ int sany[32];
    double a = 0, b = 0;
    int c = 0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        if (mmpart[3 * i + 2] == 0.0) continue;
        if (!c) { a = mmpart[3 * i]; b = mmpart[3 * i + 1]; c = 1; }
        else { a = fmin(a, mmpart[3 * i]); b = fmax(b, mmpart[3 * i + 1]); }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double a2 = __shfl_down_sync(0xffffffffu, a, o), b2 = __shfl_down_sync(0xffffffffu, b, o);
        const int c2 = __shfl_down_sync(0xffffffffu, c, o);
        if (c2) {
            if (!c) { a = a2; b = b2; c = 1; }
            else { a = fmin(a, a2); b = fmax(b, b2); }
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) { smin[w] = a; smax[w] = b; sany[w] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double numin = 0, numax = 0;
        int any = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
            if (!sany[i]) continue;
            if (!any) { numin = smin[i]; numax = smax[i]; any = 1; }
            else { numin = fmin(numin, smin[i]); numax = fmax(numax, smax[i]); }
        }
        if (nucontr >= 1.0) numax = numin * nucontr; else numin = numax * nucontr;
        lim[0] = numin;
        lim[1] = numax;
        if (stats) { stats[0] = numin; stats[1] = numax; }
    }
    __syncthreads();
    const double numin = lim[0], numax = lim[1];
    for (int64_t m3 = lo; m3 < hi; m3 += stride) {
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

static __global__ void __launch_bounds__(256) k_clamp(int64_t nn, const double *__restrict__ mmpart, int32_t nparts,
                                               double nucontr, double *__restrict__ nu, double *__restrict__ nd,
                                               double *__restrict__ stats)
{
    clamp_nodes(mmpart, nparts, nucontr, nu, nd, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, nn,
                (int64_t)gridDim.x * blockDim.x, blockIdx.x == 0 ? stats : nullptr);
}

}  // namespace i2g
