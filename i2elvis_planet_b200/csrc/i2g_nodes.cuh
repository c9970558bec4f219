// Contrast clamp of ronurecalc() (markmart.c:995-1009).  Included by one
// translation unit only (i2g_fp64.cu).
#pragma once

#include "i2g_kernels.cuh"

namespace i2g {

// ----------------------------------------------------------------- node loop
// contrast clamp: every block folds the per-block ranges (exact, order-free),
// then clamps its nodes; block 0 records {numin, numax}
__global__ void __launch_bounds__(256) k_clamp(int64_t nn, const double *__restrict__ mmpart, int32_t nparts,
                                               double nucontr, double *__restrict__ nu, double *__restrict__ nd,
                                               double *__restrict__ stats)
{
    __shared__ double smin[8], smax[8];
    __shared__ int sany[8];
    double a = 0, b = 0;
    int c = 0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        if (mmpart[3 * i + 2] == 0.0) continue;
        if (!c) { a = mmpart[3 * i]; b = mmpart[3 * i + 1]; c = 1; }
        else { a = fmin(a, mmpart[3 * i]); b = fmax(b, mmpart[3 * i + 1]); }
    }
    for (int o = 16; o > 0; o >>= 1) {
        double a2 = __shfl_down_sync(0xffffffffu, a, o), b2 = __shfl_down_sync(0xffffffffu, b, o);
        int c2 = __shfl_down_sync(0xffffffffu, c, o);
        if (c2) {
            if (!c) { a = a2; b = b2; c = 1; }
            else { a = fmin(a, a2); b = fmax(b, b2); }
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { smin[w] = a; smax[w] = b; sany[w] = c; }
    __syncthreads();
    __shared__ double lim[2];
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
        if (blockIdx.x == 0 && stats) { stats[0] = numin; stats[1] = numax; }
    }
    __syncthreads();
    const double numin = lim[0], numax = lim[1];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t m3 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m3 < nn; m3 += stride) {
        double v = nu[m3], u = v;
        if (u < numin) u = numin;
        if (u > numax) u = numax;
        if (u != v || (v != v)) nu[m3] = u;
        v = nd[m3];
        u = v;
        if (u < numin) u = numin;
        if (u > numax) u = numax;
        if (u != v || (v != v)) nd[m3] = u;
    }
}

}  // namespace i2g
