// Cell sort of the marker arrays and the small helper kernels of the context.
//
// Markers live on the device sorted by cell (x-major cell index, the node
// layout of headmart.c:87-99) and, inside a cell, by ascending caller index.
// That canonical order makes every per-cell and per-node sum a fixed-order
// reduction, independent of launch configuration and of earlier history.
//
// Sort = counting sort over cells:
//   k_hist      per-cell counts (warp-aggregated integer atomics: exact)
//   scan        exclusive prefix over cells -> cell start offsets
//   k_scatter   slot reservation per cell (warp-aggregated); after a movemark
//               k_scatter_sub places each marker by the arrival index k_move's
//               counting atomics gave it
//   k_fixup     order each cell's slots by caller index (the canonical order):
//               perm2[slot] = marker and, when asked, rank[marker] = slot
//   k_gather    move every marker field into its slot
#include "i2g_launch.h"

#include <cub/device/device_scan.cuh>

namespace i2g {

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__global__ void __launch_bounds__(256) k_hist(const int32_t *__restrict__ key, int64_t n, int32_t *__restrict__ count)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const int32_t k = valid ? key[i] : -1;
    const unsigned act = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    const unsigned peers = __match_any_sync(act, k);
    const int leader = __ffs(peers) - 1;
    if ((int)(threadIdx.x & 31) == leader) atomicAdd(count + k, __popc(peers));
}

__global__ void __launch_bounds__(256) k_scatter(const int32_t *__restrict__ key, int64_t n,
                                                 const int32_t *__restrict__ cstart, int32_t *__restrict__ cursor,
                                                 int32_t *__restrict__ slot_of)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const int32_t k = valid ? key[i] : -1;
    const unsigned act = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    const unsigned peers = __match_any_sync(act, k);
    const int leader = __ffs(peers) - 1;
    int32_t base = 0;
    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(cursor + k, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    slot_of[cstart[k] + base + __popc(peers & lanemask_lt())] = (int32_t)i;
}

// The slots of markers whose arrival index in their cell k_move recorded.
__global__ void __launch_bounds__(256) k_scatter_sub(const int32_t *__restrict__ key, const int32_t *__restrict__ sub,
                                                     int64_t n, const int32_t *__restrict__ cstart,
                                                     int32_t *__restrict__ slot_of)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) slot_of[__ldg(cstart + __ldg(key + i)) + __ldg(sub + i)] = (int32_t)i;
}

// One warp per cell: rank the cell's entries by caller index (ids are unique).
// Up to 64 entries rank from registers via shuffles, up to kFixSmem from shared
// memory; longer cells (strong compression) rank straight from global memory.
constexpr int kFixSmem = 256;

// One cell by a whole warp (the layout for cells of more than 48 markers).
__device__ __forceinline__ void fix_cell(int64_t cell, int lane, int32_t *__restrict__ sid,
                                         const int32_t *__restrict__ cstart, const int32_t *__restrict__ src,
                                         const int32_t *__restrict__ id, int32_t *__restrict__ dst,
                                         int32_t *__restrict__ rank)
{
    const int32_t s = cstart[cell], e = cstart[cell + 1], n = e - s;
    if (n <= 64) {
        // lanes past the cell hold the largest int32, which no caller index
        // reaches: comparing with them counts nothing, so the loops run in whole
        // groups of 8 without a bound per step
        const int32_t p0 = lane < n ? src[s + lane] : 0, p1 = lane + 32 < n ? src[s + lane + 32] : 0;
        const int32_t v0 = lane < n ? id[p0] : 0x7fffffff, v1 = lane + 32 < n ? id[p1] : 0x7fffffff;
        // u < w exactly when the sign bit of u - w is set (both in [0, 2^31))
        const uint32_t w0 = (uint32_t)v0, w1 = (uint32_t)v1;
        uint32_t r0 = 0, r1 = 0;
        const int n0 = ((n < 32 ? n : 32) + 7) & ~7, n1 = ((n > 32 ? n - 32 : 0) + 7) & ~7;
        for (int j0 = 0; j0 < n0; j0 += 8) {
#pragma unroll
            for (int j = j0; j < j0 + 8; j++) {
                const uint32_t u = (uint32_t)__shfl_sync(0xffffffffu, v0, j);
                r0 += (u - w0) >> 31;
                r1 += (u - w1) >> 31;
            }
        }
        for (int j0 = 0; j0 < n1; j0 += 8) {
#pragma unroll
            for (int j = j0; j < j0 + 8; j++) {
                const uint32_t u = (uint32_t)__shfl_sync(0xffffffffu, v1, j);
                r0 += (u - w0) >> 31;
                r1 += (u - w1) >> 31;
            }
        }
        if (lane < n) {
            dst[s + r0] = p0;
            if (rank) rank[p0] = s + r0;
        }
        if (lane + 32 < n) {
            dst[s + r1] = p1;
            if (rank) rank[p1] = s + r1;
        }
    } else if (n <= kFixSmem) {
        for (int32_t a = lane; a < n; a += 32) sid[a] = id[src[s + a]];
        __syncwarp();
        for (int32_t a = lane; a < n; a += 32) {
            const int32_t v = sid[a];
            int32_t r = 0;
            for (int32_t j = 0; j < n; j++) r += (sid[j] < v);
            const int32_t p = src[s + a];
            dst[s + r] = p;
            if (rank) rank[p] = s + r;
        }
    } else {
        for (int32_t a = lane; a < n; a += 32) {
            const int32_t p = src[s + a], v = id[p];
            int32_t r = 0;
            for (int32_t j = 0; j < n; j++) r += (id[src[s + j]] < v);
            dst[s + r] = p;
            if (rank) rank[p] = s + r;
        }
    }
}

__global__ void __launch_bounds__(256) k_fixup(const int32_t *__restrict__ cstart, int64_t ncells,
                                               const int32_t *__restrict__ src, const int32_t *__restrict__ id,
                                               int32_t *__restrict__ dst, int32_t *__restrict__ rank)
{
    __shared__ int32_t sid[8][kFixSmem];
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (warp >= ncells) return;
    fix_cell(warp, lane, sid[w], cstart, src, id, dst, rank);
}

// the ranks within a half-warp's cell from G registers of up to 16 caller
// indices each (lane j of the half holds indices j, j+16, j+32): every index of
// the cell is broadcast in turn and compared with all of them
template <int G>
__device__ __forceinline__ void rank_half(const uint32_t (&v)[3], uint32_t (&r)[3])
{
#pragma unroll
    for (int g = 0; g < G; g++)
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const uint32_t u = (uint32_t)__shfl_sync(0xffffffffu, v[g], j, 16);
#pragma unroll
            for (int k = 0; k < G; k++) r[k] += (u - v[k]) >> 31;
        }
}

// Two cells per warp, a half-warp each with up to three markers per lane: cells
// of up to 48 markers.  (A warp per cell with two per lane compares a 36-marker
// cell with 28 empty slots at every step.)  A pair with a larger cell is ranked
// a whole warp per cell.
__global__ void __launch_bounds__(256) k_fixup_pairs(const int32_t *__restrict__ cstart, int64_t ncells,
                                                     const int32_t *__restrict__ src, const int32_t *__restrict__ id,
                                                     int32_t *__restrict__ dst, int32_t *__restrict__ rank)
{
    __shared__ int32_t sid[8][kFixSmem];
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, hl = lane & 15;
    const int64_t c0 = 2 * warp;
    if (c0 >= ncells) return;
    const int64_t cell = c0 + (lane >> 4);
    int32_t s = 0, n = 0;
    if (cell < ncells) {
        s = __ldg(cstart + cell);
        n = __ldg(cstart + cell + 1) - s;
    }
    const int nmax = max(n, __shfl_xor_sync(0xffffffffu, n, 16));
    if (nmax > 48) {
        fix_cell(c0, lane, sid[w], cstart, src, id, dst, rank);
        __syncwarp();  // the shared buffer is reused
        if (c0 + 1 < ncells) fix_cell(c0 + 1, lane, sid[w], cstart, src, id, dst, rank);
        return;
    }
    // past the cell: the largest int32, which no caller index reaches (compares
    // with it count nothing); u < w exactly when u - w has its sign bit set
    int32_t p[3];
    uint32_t v[3], r[3] = {0u, 0u, 0u};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int a = hl + 16 * k;
        p[k] = a < n ? src[s + a] : 0;
        v[k] = a < n ? (uint32_t)id[p[k]] : 0x7fffffffu;
    }
    const int groups = (nmax + 15) >> 4;  // the same in both halves
    if (groups == 3) rank_half<3>(v, r);
    else if (groups == 2) rank_half<2>(v, r);
    else if (groups == 1) rank_half<1>(v, r);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (hl + 16 * k < n) {
            dst[s + r[k]] = p[k];
            if (rank) rank[p[k]] = s + (int32_t)r[k];
        }
    }
}

__global__ void __launch_bounds__(256) k_gather(int64_t n, const int32_t *__restrict__ perm, MarkerView src,
                                                MarkerView dst, int64_t *__restrict__ slot0)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const int32_t i = perm[j];
        dst.x[j] = src.x[i];
        dst.y[j] = src.y[i];
        dst.T[j] = src.T[i];
        dst.eta[j] = src.eta[i];
        dst.p[j] = src.p[i];
        dst.type[j] = src.type[i];
        const int32_t id = src.id[i];
        dst.id[j] = id;
        if (dst.tmax) dst.tmax[j] = src.tmax[i];
        if (dst.hi) dst.hi[j] = src.hi[i];
        if (dst.por) dst.por[j] = src.por[i];
        if (dst.mgo) {
            dst.mgo[j] = src.mgo[i];
            dst.mgt[j] = src.mgt[i];
        }
        if (id == 0) *slot0 = j;
    }
}

// ------------------------------------------------------------- exclusive scan
// out[0..n] = exclusive prefix of in[0..n-1]; out[n] = total.  Three passes over
// blocks of kScanTile counts; n <= kScanTile^2.
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int32_t block_exclusive_scan(int32_t v, int32_t *total)
{
    __shared__ int32_t wsum[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int32_t t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int32_t s = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int32_t t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        wsum[lane] = s;
    }
    __syncthreads();
    const int32_t before = (w ? wsum[w - 1] : 0) + x - v;
    *total = wsum[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const int32_t *__restrict__ in, int64_t n,
                                                             int32_t *__restrict__ out, int32_t *__restrict__ tilesum)
{
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems], s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    int32_t total;
    int32_t run = block_exclusive_scan(s, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) tilesum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_top(int32_t *__restrict__ tilesum, int32_t ntiles,
                                                           int32_t *__restrict__ out_total)
{
    const int64_t base = (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems], s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (base + k < ntiles) ? tilesum[base + k] : 0;
        s += v[k];
    }
    int32_t total;
    int32_t run = block_exclusive_scan(s, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < ntiles) tilesum[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) *out_total = total;
}

__global__ void __launch_bounds__(256) k_scan_add(int32_t *__restrict__ out, int64_t n,
                                                  const int32_t *__restrict__ tilesum)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tilesum[i / kScanTile];
}

// ------------------------------------------------------------- small helpers
__global__ void k_iota(int32_t *__restrict__ a, int64_t n)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) a[i] = (int32_t)i;
}

template <bool MIXED>
__global__ void k_keys(GridView G, const double *__restrict__ x, const double *__restrict__ y, int64_t n,
                       int32_t *__restrict__ key)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) key[i] = cell_key(G, x[i], y[i]);
}

// out[id[j]] = in[j]: back to the caller's marker order
__global__ void k_unsort_f64(int64_t n, const int32_t *__restrict__ id, const double *__restrict__ in,
                             double *__restrict__ out)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) out[id[j]] = in[j];
}

// cell keys of markers in the caller's order, from FP64 or FP32 (reference storage)
// coordinates; an FP32 coordinate enters as the double it widens to
template <class R>
__global__ void k_keys_in(GridView G, const R *__restrict__ x, const R *__restrict__ y, int64_t n,
                          int32_t *__restrict__ key)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        key[i] = cell_key(G, (double)x[i], (double)y[i]);
}

// Markers in the caller's order (caller index i) into the sorted device order:
// slot j takes marker perm[j], widened to FP64.  Two passes, so the first can
// run while the second's inputs are still arriving: positions (with the id =
// caller index, the pressure starting at 0 and the slot of caller marker 0),
// then temperature, viscosity and rock type.
template <class R>
__global__ void k_gather_in_xy(int64_t n, const int32_t *__restrict__ perm, const R *__restrict__ x,
                               const R *__restrict__ y, MarkerView dst, int64_t *__restrict__ slot0)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const int32_t i = __ldg(perm + j);
        dst.x[j] = (double)x[i];
        dst.y[j] = (double)y[i];
        dst.id[j] = i;
        dst.p[j] = 0.0;
        if (i == 0) *slot0 = j;
    }
}

template <class R>
__global__ void k_gather_in_rest(int64_t n, const int32_t *__restrict__ perm, const R *__restrict__ T,
                                 const R *__restrict__ eta, const int8_t *__restrict__ type, MarkerView dst)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const int32_t i = __ldg(perm + j);
        dst.T[j] = (double)T[i];
        dst.eta[j] = (double)eta[i];
        dst.type[j] = type[i];
    }
}

// out[id[j]] = (float)in[j]: back to the caller's order, narrowed to its FP32 storage
__global__ void k_unsort_f64_f32(int64_t n, const int32_t *__restrict__ id, const double *__restrict__ in,
                                 float *__restrict__ out)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) out[id[j]] = (float)in[j];
}

__global__ void k_unsort_i8(int64_t n, const int32_t *__restrict__ id, const int8_t *__restrict__ in,
                            int8_t *__restrict__ out)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) out[id[j]] = in[j];
}

__global__ void k_f64_to_f32(int64_t n, const double *__restrict__ in, float *__restrict__ out)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = (float)in[i];
}

__global__ void k_f32_to_f64(int64_t n, const float *__restrict__ in, double *__restrict__ out)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = (double)in[i];
}

// T of caller marker 0 as the molten-material conductivity reads it (markmart.c:522):
// marker 0 is processed first by the reference, so after its own sticky-air reset.
__global__ void k_t0(GridView G, MarkerView M, const int64_t *__restrict__ slot0, double tmp_ambient,
                     double *__restrict__ T0)
{
    if (threadIdx.x || blockIdx.x) return;
    const int64_t j = *slot0;
    if (j < 0 || j >= M.n) { *T0 = 0.0; return; }
    const double x = M.x[j], y = M.y[j], t = M.T[j];
    const int mt = M.type[j];
    double v = t;
    if (x > 0 && y > 0 && x < G.xsize && y < G.ysize && t > 0 && mt < 2) v = tmp_ambient;
    *T0 = v;
}

// ------------------------------------------------------------- adjoint helpers
__global__ void k_combine_modes(int64_t nn, int32_t nm, const double *__restrict__ mvx,
                                const double *__restrict__ mvy, const double *__restrict__ amps,
                                double *__restrict__ vx, double *__restrict__ vy, float *__restrict__ vxf,
                                float *__restrict__ vyf)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += stride) {
        double a = 0.0, b = 0.0;
        for (int m = 0; m < nm; m++) {
            a += amps[m] * mvx[i * nm + m];
            b += amps[m] * mvy[i * nm + m];
        }
        vx[i] = a;
        vy[i] = b;
        if (vxf) vxf[i] = (float)a;
        if (vyf) vyf[i] = (float)b;
    }
}

__global__ void k_ckpt(MarkerView M, double2 *__restrict__ ck)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < M.n; j += stride)
        ck[M.id[j]] = make_double2(M.x[j], M.y[j]);
}

// out[m] = sum over blocks b in order of part[b][m]
__global__ void k_sum_partials(const double *__restrict__ part, int32_t nblk, int32_t nm, double *__restrict__ out)
{
    const int m = threadIdx.x;
    if (m >= nm) return;
    double s = 0.0;
    for (int32_t b = 0; b < nblk; b++) s += part[(int64_t)b * nm + m];
    out[m] = s;
}

// ------------------------------------------------------------- host launchers
static inline unsigned blocks_for(int64_t n, int threads, int64_t cap = 1 << 20)
{
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

int scan_exclusive(cudaStream_t s, const int32_t *in, int64_t n, int32_t *out, int32_t *tilesum)
{
    const int64_t ntiles = (n + kScanTile - 1) / kScanTile;
    k_scan_tiles<<<(unsigned)(ntiles > 0 ? ntiles : 1), kScanThreads, 0, s>>>(in, n, out, tilesum);
    k_scan_top<<<1, kScanThreads, 0, s>>>(tilesum, (int32_t)ntiles, out + n);
    k_scan_add<<<blocks_for(n, 256, INT32_MAX), 256, 0, s>>>(out, n, tilesum);
    return 3;
}

int64_t scan_max_elems() { return (int64_t)kScanTile * kScanTile; }

int sort_markers(cudaStream_t s, const SortBufs &B, int64_t n, int64_t ncells, MarkerView src, MarkerView dst)
{
    int nl = 0;
    cudaMemsetAsync(B.count, 0, sizeof(int32_t) * (size_t)ncells, s);
    cudaMemsetAsync(B.cursor, 0, sizeof(int32_t) * (size_t)ncells, s);
    if (n > 0) k_hist<<<blocks_for(n, 256, INT32_MAX), 256, 0, s>>>(B.key, n, B.count), nl++;
    nl += scan_exclusive(s, B.count, ncells, B.cstart, B.tilesum);
    if (n > 0) {
        k_scatter<<<blocks_for(n, 256, INT32_MAX), 256, 0, s>>>(B.key, n, B.cstart, B.cursor, B.perm1);
        k_fixup_pairs<<<blocks_for((ncells + 1) / 2 * 32, 256, INT32_MAX), 256, 0, s>>>(B.cstart, ncells, B.perm1,
                                                                                        src.id, B.perm2, nullptr);
        k_gather<<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, B.perm2, src, dst, B.slot0);
        nl += 3;
    }
    return nl;
}

int rank_markers(cudaStream_t s, const SortBufs &B, int64_t n, int64_t ncells, const int32_t *id,
                 bool counts_ready)
{
    int nl = 0;
    if (!counts_ready) {
        cudaMemsetAsync(B.count, 0, sizeof(int32_t) * (size_t)ncells, s);
        if (n > 0) k_hist<<<blocks_for(n, 256, INT32_MAX), 256, 0, s>>>(B.key, n, B.count), nl++;
    }
    cudaMemsetAsync(B.cursor, 0, sizeof(int32_t) * (size_t)ncells, s);
    nl += scan_exclusive(s, B.count, ncells, B.cstart, B.tilesum);
    if (n > 0) {
        k_scatter<<<blocks_for(n, 256, INT32_MAX), 256, 0, s>>>(B.key, n, B.cstart, B.cursor, B.perm1);
        k_fixup_pairs<<<blocks_for((ncells + 1) / 2 * 32, 256, INT32_MAX), 256, 0, s>>>(B.cstart, ncells, B.perm1, id,
                                                                                        B.perm2, B.rank);
        nl += 2;
    }
    return nl;
}

int rank_moved(cudaStream_t s, const SortBufs &B, int64_t n, int64_t ncells, const int32_t *id,
               const int32_t *sub)
{
    int nl = scan_exclusive(s, B.count, ncells, B.cstart, B.tilesum);
    if (n > 0) {
        k_scatter_sub<<<blocks_for(n, 256, INT32_MAX), 256, 0, s>>>(B.key, sub, n, B.cstart, B.perm1);
        k_fixup_pairs<<<blocks_for((ncells + 1) / 2 * 32, 256, INT32_MAX), 256, 0, s>>>(B.cstart, ncells, B.perm1, id,
                                                                                        B.perm2, B.rank);
        nl += 2;
    }
    return nl;
}

struct MaxI32 {
    __device__ __forceinline__ int32_t operator()(int32_t a, int32_t b) const { return a > b ? a : b; }
};

int td_prev_scan(cudaStream_t s, void *tmp, size_t *bytes, const int32_t *flag, int32_t *prev, int64_t n)
{
    if (n > INT32_MAX) return -1;
    cudaError_t e = cub::DeviceScan::InclusiveScan(tmp, *bytes, flag, prev, MaxI32(), (int)n, s);
    return e == cudaSuccess ? (tmp ? 1 : 0) : -1;
}

int launch_keys(cudaStream_t s, const GridView &G, const double *x, const double *y, int64_t n, int32_t *key)
{
    if (n <= 0) return 0;
    k_keys<false><<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(G, x, y, n, key);
    return 1;
}

int launch_iota(cudaStream_t s, int32_t *a, int64_t n)
{
    if (n <= 0) return 0;
    k_iota<<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(a, n);
    return 1;
}

int launch_unsort_f64(cudaStream_t s, int64_t n, const int32_t *id, const double *in, double *out)
{
    if (n <= 0) return 0;
    k_unsort_f64<<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, id, in, out);
    return 1;
}

int launch_keys_in(cudaStream_t s, const GridView &G, const void *x, const void *y, int64_t n, bool f32,
                   int32_t *key)
{
    if (n <= 0) return 0;
    if (f32)
        k_keys_in<float><<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(G, (const float *)x, (const float *)y, n, key);
    else
        k_keys_in<double><<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(G, (const double *)x, (const double *)y, n,
                                                                       key);
    return 1;
}

int launch_gather_in_xy(cudaStream_t s, int64_t n, const int32_t *perm, const void *x, const void *y, bool f32,
                        const MarkerView &dst, int64_t *slot0)
{
    if (n <= 0) return 0;
    if (f32)
        k_gather_in_xy<float><<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, perm, (const float *)x,
                                                                           (const float *)y, dst, slot0);
    else
        k_gather_in_xy<double><<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, perm, (const double *)x,
                                                                            (const double *)y, dst, slot0);
    return 1;
}

int launch_gather_in_rest(cudaStream_t s, int64_t n, const int32_t *perm, const void *T, const void *eta,
                          const int8_t *type, bool f32, const MarkerView &dst)
{
    if (n <= 0) return 0;
    if (f32)
        k_gather_in_rest<float><<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, perm, (const float *)T,
                                                                             (const float *)eta, type, dst);
    else
        k_gather_in_rest<double><<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, perm, (const double *)T,
                                                                              (const double *)eta, type, dst);
    return 1;
}

int launch_unsort_f64_f32(cudaStream_t s, int64_t n, const int32_t *id, const double *in, float *out)
{
    if (n <= 0) return 0;
    k_unsort_f64_f32<<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, id, in, out);
    return 1;
}

int launch_unsort_i8(cudaStream_t s, int64_t n, const int32_t *id, const int8_t *in, int8_t *out)
{
    if (n <= 0) return 0;
    k_unsort_i8<<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, id, in, out);
    return 1;
}

int launch_f64_to_f32(cudaStream_t s, int64_t n, const double *in, float *out)
{
    if (n <= 0) return 0;
    k_f64_to_f32<<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, in, out);
    return 1;
}

int launch_f32_to_f64(cudaStream_t s, int64_t n, const float *in, double *out)
{
    if (n <= 0) return 0;
    k_f32_to_f64<<<blocks_for(n, 256, 148 * 16), 256, 0, s>>>(n, in, out);
    return 1;
}

int launch_t0(cudaStream_t s, const GridView &G, const MarkerView &M, const int64_t *slot0, double tmp_ambient,
              double *T0)
{
    k_t0<<<1, 32, 0, s>>>(G, M, slot0, tmp_ambient, T0);
    return 1;
}

// bilinear coefficients of every 2x2 stencil at its lower-left node (GridView.vxq)
__global__ void k_quads(int64_t nx, int64_t ny, const float *__restrict__ f, float4 *__restrict__ q)
{
    const int64_t m3 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m3 >= nx * ny) return;
    const int64_t m1 = m3 / ny, m2 = m3 - m1 * ny;
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
    if (m1 + 1 < nx && m2 + 1 < ny) {
        const float a = f[m3], b = f[m3 + 1], c = f[m3 + ny], d = f[m3 + ny + 1];
        r = make_float4(a, c - a, b - a, (a - b) - (c - d));
    }
    q[m3] = r;
}

int launch_quads(cudaStream_t s, int64_t nx, int64_t ny, const float *f, float4 *q)
{
    const int64_t nn = nx * ny;
    if (nn <= 0) return 0;
    k_quads<<<blocks_for(nn, 256, INT32_MAX), 256, 0, s>>>(nx, ny, f, q);
    return 1;
}

// Per quarter cell of a uniform grid (half a cell along each axis: hx = 2 i + qx,
// hy = 2 j + qy), the bilinear forms of vx and vy in the quarter's coordinates
// fx, fy in [0, 1]: the stencil the mixed RK4 takes there (vx basic in x and
// staggered in y, vy staggered in x and basic in y; the staggered stencil is the
// lower neighbour in a lower half, clamped to [0, n - 3], markmart.c:1403-1437)
// with X = ax + fx / 2, Y = ay + fy / 2 substituted into A + B X + C Y + D X Y,
// in FP64 from the FP32 node values, rounded once.
__global__ void k_quarters(int64_t nx, int64_t ny, const float *__restrict__ vxf, const float *__restrict__ vyf,
                           float4 *__restrict__ q)
{
    const int64_t nhy = 2 * (ny - 1), nq = 2 * (nx - 1) * nhy;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nq) return;
    const int64_t hx = t / nhy, hy = t - hx * nhy;
    const int64_t i = hx >> 1, j = hy >> 1;
    const int qx = (int)(hx & 1), qy = (int)(hy & 1);
    auto stag = [](int64_t b, int q, int64_t n) {
        int64_t m = q ? b : b - 1;
        if (m < 0) m = 0;
        if (m > n - 3) m = n - 3;
        return m;
    };
    auto form = [&](const float *f, int64_t s1, int64_t s2, double ax, double ay) {
        const int64_t m3 = s1 * ny + s2;
        const double a = f[m3], b = f[m3 + 1], c = f[m3 + ny], d = f[m3 + ny + 1];
        const double B = c - a, C = b - a, D = (a - b) - (c - d);
        return make_float4((float)(a + B * ax + C * ay + D * ax * ay), (float)(0.5 * (B + D * ay)),
                           (float)(0.5 * (C + D * ax)), (float)(0.25 * D));
    };
    const int64_t my = stag(j, qy, ny), mx = stag(i, qx, nx);
    q[2 * t] = form(vxf, i, my, 0.5 * qx, (double)(j - my) - 0.5 + 0.5 * qy);
    q[2 * t + 1] = form(vyf, mx, j, (double)(i - mx) - 0.5 + 0.5 * qx, 0.5 * qy);
}

int launch_quarters(cudaStream_t s, int64_t nx, int64_t ny, const float *vxf, const float *vyf, float4 *q)
{
    const int64_t nq = 4 * (nx - 1) * (ny - 1);
    if (nq <= 0) return 0;
    k_quarters<<<blocks_for(nq, 256, INT32_MAX), 256, 0, s>>>(nx, ny, vxf, vyf, q);
    return 1;
}

int launch_combine_modes(cudaStream_t s, int64_t nn, int32_t nm, const double *mvx, const double *mvy,
                         const double *amps, double *vx, double *vy, float *vxf, float *vyf)
{
    k_combine_modes<<<blocks_for(nn, 256, 148 * 16), 256, 0, s>>>(nn, nm, mvx, mvy, amps, vx, vy, vxf, vyf);
    return 1;
}

int launch_ckpt(cudaStream_t s, const MarkerView &M, double2 *ck)
{
    if (M.n <= 0) return 0;
    k_ckpt<<<blocks_for(M.n, 256, 148 * 16), 256, 0, s>>>(M, ck);
    return 1;
}

int launch_sum_partials(cudaStream_t s, const double *part, int32_t nblk, int32_t nm, double *out)
{
    k_sum_partials<<<1, 32, 0, s>>>(part, nblk, nm, out);
    return 1;
}

// the sort's kernels, loaded now rather than at their first launch
void preload_sort()
{
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_hist);
    cudaFuncGetAttributes(&a, k_scatter);
    cudaFuncGetAttributes(&a, k_scatter_sub);
    cudaFuncGetAttributes(&a, k_fixup);
    cudaFuncGetAttributes(&a, k_fixup_pairs);
    cudaFuncGetAttributes(&a, k_gather);
    cudaFuncGetAttributes(&a, k_scan_tiles);
    cudaFuncGetAttributes(&a, k_scan_top);
    cudaFuncGetAttributes(&a, k_scan_add);
    cudaFuncGetAttributes(&a, k_t0);
}

}  // namespace i2g
