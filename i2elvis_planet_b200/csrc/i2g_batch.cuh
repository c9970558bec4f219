// Batched marker step: many planetesimal instances, each phase one launch over
// the work of every instance.
//
// An instance is a context (grid, markers, nodes, scratch) described on the
// device by an InstDesc.  The work of a phase is numbered globally -- markers,
// cells, averaging tiles or node blocks of instance 0, then instance 1, ... --
// and a thread finds its instance by bisecting the per-instance offsets.  The
// movemark and averaging phases run as persistent grids (a fixed number of CTAs
// per SM striding over the work), so instances of very different sizes share
// the GPU without a launch per instance.  One step is eleven launches; the host
// captures them once into a CUDA graph and replays the graph per step.
// Per-step scalars (timesum and the radiogenic heating rates derived from it)
// come from a per-instance table indexed by a device step counter, so the graph
// is identical from step to step.
//
// Every instance sees exactly the arithmetic and summation order of the
// single-instance path (same device functions), and none of it depends on the
// tile width or grid sizes the autotuner picks.
#pragma once

#include "i2g_avg.cuh"
#include "i2g_launch.h"
#include "i2g_nodes.cuh"

namespace i2g {

__device__ __forceinline__ int find_inst(const int64_t *__restrict__ off, int n, int64_t g)
{
    int lo = 0, hi = n;  // off[lo] <= g < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(off + mid) <= g) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ unsigned lanemask_lt_b()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// zero counts and cursors of every instance's cells, and the averaged-marker counters
static __global__ void kb_zero(const __grid_constant__ BatchRun R)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < R.tot_cell; g += stride) {
        const int k = find_inst(R.off_cell, R.ninst, g);
        const int64_t c = g - R.off_cell[k];
        R.D[k].sb.count[c] = 0;
        R.D[k].sb.cursor[c] = 0;
    }
    if (blockIdx.x == 0)
        for (int k = threadIdx.x; k < R.ninst; k += blockDim.x) *R.D[k].navg = 0;
}

template <bool MIXED>
__global__ void __launch_bounds__(256) kb_move(const __grid_constant__ BatchRun R)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < R.tot_mark; g += stride) {
        const int k = find_inst(R.off_mark, R.ninst, g);
        const InstDesc &d = R.D[k];
        const int64_t i = g - R.off_mark[k];
        const int32_t key = move_marker<MIXED, false>(d.G, d.buf[d.cur], d.types->t, d.move, d.sb.key, i);
        // count per (instance, cell): a key alone may repeat across instances
        const unsigned long long tag = ((unsigned long long)(unsigned)k << 32) | (unsigned)key;
        const unsigned peers = __match_any_sync(__activemask(), tag);
        if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(d.sb.count + key, __popc(peers));
    }
}

// one CTA per instance: exclusive prefix of the cell counts -> cell starts
static __global__ void __launch_bounds__(1024) kb_scan(const __grid_constant__ BatchRun R)
{
    __shared__ int32_t wsum[32];
    __shared__ int32_t carry_s;
    const InstDesc &d = R.D[blockIdx.x];
    const int64_t n = d.ncells;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    for (int64_t base = 0; base < n; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const int32_t v = i < n ? d.sb.count[i] : 0;
        int32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            int32_t s = lane < nw ? wsum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t t = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += t;
            }
            wsum[lane] = s;
        }
        __syncthreads();
        const int32_t carry = carry_s;
        if (i < n) d.sb.cstart[i] = carry + (w ? wsum[w - 1] : 0) + x - v;
        __syncthreads();
        if (threadIdx.x == 0) carry_s = carry + wsum[nw - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) d.sb.cstart[n] = carry_s;
}

static __global__ void __launch_bounds__(256) kb_scatter(const __grid_constant__ BatchRun R)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = g < R.tot_mark;
    int k = 0;
    int32_t key = -1;
    int64_t i = 0;
    if (valid) {
        k = find_inst(R.off_mark, R.ninst, g);
        i = g - R.off_mark[k];
        key = R.D[k].sb.key[i];
    }
    const unsigned act = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    const InstDesc &d = R.D[k];
    const unsigned long long tag = ((unsigned long long)(unsigned)k << 32) | (unsigned)key;
    const unsigned peers = __match_any_sync(act, tag);
    const int leader = __ffs(peers) - 1;
    int32_t base = 0;
    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(d.sb.cursor + key, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    d.sb.perm1[d.sb.cstart[key] + base + __popc(peers & lanemask_lt_b())] = (int32_t)i;
}

// one warp per cell: order the cell's slots by caller index (the canonical order)
static __global__ void __launch_bounds__(256) kb_fixup(const __grid_constant__ BatchRun R)
{
    __shared__ int32_t sid[8][256];
    const int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (g >= R.tot_cell) return;
    const int k = find_inst(R.off_cell, R.ninst, g);
    const InstDesc &d = R.D[k];
    const int64_t cell = g - R.off_cell[k];
    const int32_t *src = d.sb.perm1, *id = d.buf[d.cur].id;
    int32_t *dst = d.sb.perm2;
    const int32_t s = d.sb.cstart[cell], e = d.sb.cstart[cell + 1], n = e - s;
    if (n <= 64) {
        const int32_t p0 = lane < n ? src[s + lane] : 0, p1 = lane + 32 < n ? src[s + lane + 32] : 0;
        const int32_t v0 = lane < n ? id[p0] : 0x7fffffff, v1 = lane + 32 < n ? id[p1] : 0x7fffffff;
        int r0 = 0, r1 = 0;
        const int n0 = n < 32 ? n : 32;
        for (int j = 0; j < n0; j++) {
            const int32_t u = __shfl_sync(0xffffffffu, v0, j);
            r0 += (u < v0);
            r1 += (u < v1);
        }
        for (int j = 0; j < n - 32; j++) {
            const int32_t u = __shfl_sync(0xffffffffu, v1, j);
            r0 += (u < v0);
            r1 += (u < v1);
        }
        if (lane < n) dst[s + r0] = p0;
        if (lane + 32 < n) dst[s + r1] = p1;
    } else if (n <= 256) {
        for (int32_t a = lane; a < n; a += 32) sid[w][a] = id[src[s + a]];
        __syncwarp();
        for (int32_t a = lane; a < n; a += 32) {
            const int32_t v = sid[w][a];
            int32_t r = 0;
            for (int32_t j = 0; j < n; j++) r += (sid[w][j] < v);
            dst[s + r] = src[s + a];
        }
    } else {
        for (int32_t a = lane; a < n; a += 32) {
            const int32_t p = src[s + a], v = id[p];
            int32_t r = 0;
            for (int32_t j = 0; j < n; j++) r += (id[src[s + j]] < v);
            dst[s + r] = p;
        }
    }
}

// T of each instance's caller marker 0 after its own sticky-air reset (markmart.c:522)
static __global__ void kb_t0(const __grid_constant__ BatchRun R)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R.ninst) return;
    const InstDesc &d = R.D[k];
    const MarkerView &M = d.buf[d.cur];
    const int64_t j = *d.sb.slot0;
    if (j < 0 || j >= M.n) { *d.T0 = 0.0; return; }
    const double x = M.x[j], y = M.y[j], t = M.T[j];
    double v = t;
    if (x > 0 && y > 0 && x < d.G.xsize && y < d.G.ysize && t > 0 && M.type[j] < 2) v = d.avg.tmp_ambient;
    *d.T0 = v;
}

// the instance's averaging constants at the current step
__device__ __forceinline__ AvgArgsK step_args(const InstDesc &d, int step)
{
    AvgArgsK args = d.avg;
    args.timesum = d.stepc[4 * step + 0];
    args.rad_si = d.stepc[4 * step + 1];
    args.rad_fe = d.stepc[4 * step + 2];
    args.rad_ch = d.stepc[4 * step + 3];
    args.track_tmax = d.track_tmax;
    return args;
}

template <bool MIXED>
__global__ void __launch_bounds__(256, 3) kb_contrib(const __grid_constant__ BatchRun R)
{
    const int step = *R.step;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < R.tot_mark; g += stride) {
        const int k = find_inst(R.off_mark, R.ninst, g);
        const InstDesc &d = R.D[k];
        const int cur = d.cur;
        contrib_marker<MIXED>(d.G, d.buf[cur], d.buf[1 - cur], d.sb.perm2, d.types->t, step_args(d, step), *d.T0,
                              reinterpret_cast<uint4 *>(d.payload), g - R.off_mark[k], d.sb.slot0);
    }
}

template <bool MIXED>
__global__ void __launch_bounds__(256, 2) kb_cellsums(const __grid_constant__ BatchRun R)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    AvgSmem<MIXED> &S = *reinterpret_cast<AvgSmem<MIXED> *>(smraw);
    for (int64_t g = blockIdx.x; g < R.tot_tile; g += gridDim.x) {
        const int k = find_inst(R.off_tile, R.ninst, g);
        const InstDesc &d = R.D[k];
        add_count(cellsums_tile<MIXED>(S, reinterpret_cast<const uint4 *>(d.payload), d.sb.cstart, d.G.nx - 1,
                                       d.G.ny - 1, d.part, g - R.off_tile[k], R.TX, d.ntx),
                  d.navg);
    }
}

static __global__ void __launch_bounds__(256) kb_nodesums(const __grid_constant__ BatchRun R)
{
    const int k = find_inst(R.off_nblk, R.ninst, blockIdx.x);
    const InstDesc &d = R.D[k];
    const int64_t b = blockIdx.x - R.off_nblk[k];
    const int64_t m3 = b * blockDim.x + threadIdx.x;
    double vmin = 0, vmax = 0;
    int any = 0;
    if (m3 < d.nn) node_finalize(d.G, d.part, d.avg, d.O, m3, vmin, vmax, any);
    block_fold(vmin, vmax, any, d.mmpart + 3 * b);
}

static __global__ void __launch_bounds__(256) kb_clamp(const __grid_constant__ BatchRun R)
{
    const int k = find_inst(R.off_nblk, R.ninst, blockIdx.x);
    const InstDesc &d = R.D[k];
    const int64_t b = blockIdx.x - R.off_nblk[k];
    const int64_t lo = b * blockDim.x + threadIdx.x, hi = min((b + 1) * (int64_t)blockDim.x, d.nn);
    clamp_nodes(d.mmpart, d.nblk, d.nucontr, d.O.nu, d.O.nd, lo, hi, blockDim.x, b == 0 ? d.stats : nullptr);
}

static __global__ void kb_stepend(const __grid_constant__ BatchRun R)
{
    for (int k = threadIdx.x; k < R.ninst; k += blockDim.x) R.D[k].cur ^= 1;
    if (threadIdx.x == 0) *R.step += 1;
}

template <bool MIXED>
int launch_batch_step_t(cudaStream_t s, const BatchRun &R, int move_ctas, int cell_ctas)
{
    static unsigned long long attr = 0;
    const int smem = (int)sizeof(AvgSmem<MIXED>);
    allow_dynamic_smem((const void *)kb_cellsums<MIXED>, smem, &attr);
    auto nb = [](int64_t n, int t) { return (unsigned)((n + t - 1) / t > 0 ? (n + t - 1) / t : 1); };
    kb_zero<<<(unsigned)std::min<int64_t>(nb(R.tot_cell, 256), 148 * 8), 256, 0, s>>>(R);
    kb_move<MIXED><<<move_ctas, 256, 0, s>>>(R);
    kb_scan<<<R.ninst, 1024, 0, s>>>(R);
    kb_scatter<<<nb(R.tot_mark, 256), 256, 0, s>>>(R);
    kb_fixup<<<nb(R.tot_cell * 32, 256), 256, 0, s>>>(R);
    kb_t0<<<nb(R.ninst, 64), 64, 0, s>>>(R);
    kb_contrib<MIXED><<<move_ctas, 256, 0, s>>>(R);
    kb_cellsums<MIXED><<<cell_ctas, 256, smem, s>>>(R);
    kb_nodesums<<<(unsigned)R.tot_nblk, 256, 0, s>>>(R);
    kb_clamp<<<(unsigned)R.tot_nblk, 256, 0, s>>>(R);
    kb_stepend<<<1, 128, 0, s>>>(R);
    return 11;
}

}  // namespace i2g
