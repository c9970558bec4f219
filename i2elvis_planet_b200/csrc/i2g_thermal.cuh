// Marker temperatures after the host's thermal solve: the marker part of
// titerate() (heatmart.c:514-697, intermod = 0).
//
// k_tmark: one thread per marker in storage order.  Inside the box, a fluid
//   marker (type 50..99) takes the new node temperature (heatmart.c:523-533); a
//   rock marker (< 50) is reset to the old node temperature if it has none, gets
//   the subgrid diffusion step toward it when heatdif != 0, then follows the node
//   change (heatmart.c:538-628).  Its diffusion change and weights go to its slot
//   of the cell-sorted order as one averaging payload record.
// k_cellsums (i2g_avg.cuh) sums those records per cell in slot order (weights in
//   the F_W0 sums, change x weight in F_RO), the same fixed-order segmented
//   reduction as the averaging.
// k_tnodes: per node, the four cells' corner sums in the averaging's fixed order,
//   then the averaged change sol1 / sol0 (heatmart.c:638-652).
// k_tanti: per rock marker, the antidiffusion: minus the averaged change of each
//   of its four nodes times its weight, in the reference's node order
//   (heatmart.c:654-693).
// The diffusion term's 1.0/celdx/celdx + 1.0/celdy/celdy (heatmart.c:592) reads
// per-line tables computed on the host with the same operations.
#pragma once

#include "i2g_avg.cuh"

namespace i2g {

// allintert() (markmart.c:1687-1745) at a point strictly inside the box: the
// basic cell by the exact search and its linear weights
__device__ __forceinline__ void tweights(const GridView &G, double x, double y, int64_t &m10, int64_t &m20,
                                         double &wx0, double &wx1, double &wy0, double &wy1)
{
    m10 = cell_search(G.gx, G.nx, G.inv_x, x);
    m20 = cell_search(G.gy, G.ny, G.inv_y, y);
    fdw64(__ldg(G.gx + m10), __ldg(G.gx + m10 + 1), x, wx0, wx1);
    fdw64(__ldg(G.gy + m20), __ldg(G.gy + m20 + 1), y, wy0, wy1);
}

__device__ __forceinline__ bool inside_box(const GridView &G, double x, double y)
{
    return x > 0 && y > 0 && x < G.xsize && y < G.ysize;
}

// FP32 weights of the mixed form at the exact FP64 cell (fdw32)
__device__ __forceinline__ void tweights32(const GridView &G, double x, double y, int64_t &m10, int64_t &m20,
                                           float &wx0, float &wx1, float &wy0, float &wy1)
{
    m10 = cell_search(G.gx, G.nx, G.inv_x, x);
    m20 = cell_search(G.gy, G.ny, G.inv_y, y);
    fdw32(__ldg(G.gx + m10), __ldg(G.ixb + m10), x, wx0, wx1);
    fdw32(__ldg(G.gy + m20), __ldg(G.iyb + m20), y, wy0, wy1);
}

// payload: NULL when heatdif == 0 (no sums); rank: NULL when the storage order is
// the sorted order (slot = index).  The FP64 form follows the reference's
// operations; the mixed form gathers FP32 node copies with FP32 weights and
// keeps the marker temperature itself in FP64.
template <bool MIXED>
__global__ void __launch_bounds__(256) k_tmark(const __grid_constant__ GridView G, const __grid_constant__ MarkerView M,
                                               const int32_t *__restrict__ rank, const __grid_constant__ ThermArgs A,
                                               void *payload)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M.n) return;
    const double x = M.x[i], y = M.y[i];
    const int t = M.type[i];
    PayVec<MIXED> u;
#pragma unroll
    for (int q = 0; q < PayVec<MIXED>::R4; q++) u.v[q] = make_uint4(0u, 0u, 0u, 0u);
    if (inside_box(G, x, y) && t < 100) {
        const int64_t ny = G.ny;
        int64_t m10, m20;
        if constexpr (!MIXED) {
            double wx0, wx1, wy0, wy1;
            tweights(G, x, y, m10, m20, wx0, wx1, wy0, wy1);
            const double tn = bil64(A.tkn, ny, m10, m20, wx0, wx1, wy0, wy1);
            if (t >= 50) {
                M.T[i] = tn;
            } else {
                double T = M.T[i];
                const double to = bil64(A.tko, ny, m10, m20, wx0, wx1, wy0, wy1);
                if (T <= 0) T = to;
                if (A.heatdif != 0) {
                    const double dtk = to - T;
                    const double mkt = bil64(A.kt, ny, m10, m20, wx0, wx1, wy0, wy1);
                    const double mcp = bil64(A.cp, ny, m10, m20, wx0, wx1, wy0, wy1);
                    const double mro = bil64(A.ro, ny, m10, m20, wx0, wx1, wy0, wy1);
                    double dtk1 = -A.heatdif * mkt / mro / mcp * 2.0 * (__ldg(A.idx2 + m10) + __ldg(A.idy2 + m20)) *
                                  A.timestep;
                    if (dtk1 < -150.0) dtk1 = -150.0;
                    dtk1 = dtk * (1.0 - exp(dtk1));
                    T += dtk1;
                    u.r.wx0 = wx0;
                    u.r.wx1 = wx1;
                    u.r.wy0 = wy0;
                    u.r.wy1 = wy1;
                    u.r.pv[0] = dtk1;
                    u.r.flag = 3u;  // summed; "immobile": no temperature-weight sums
                }
                T += tn - to;
                M.T[i] = T;
            }
        } else {
            float wx0, wx1, wy0, wy1;
            tweights32(G, x, y, m10, m20, wx0, wx1, wy0, wy1);
            const int64_t nn = G.nx * ny;
            const int nyi = (int)ny;
            const float tn = bil32(A.f, nyi, m10, m20, wx0, wx1, wy0, wy1);
            if (t >= 50) {
                M.T[i] = (double)tn;
            } else {
                double T = M.T[i];
                const float to = bil32(A.f + nn, nyi, m10, m20, wx0, wx1, wy0, wy1);
                if (T <= 0) T = (double)to;
                if (A.heatdif != 0) {
                    const float dtk = (float)((double)to - T);
                    const float mkt = bil32(A.f + 2 * nn, nyi, m10, m20, wx0, wx1, wy0, wy1);
                    const float mcp = bil32(A.f + 3 * nn, nyi, m10, m20, wx0, wx1, wy0, wy1);
                    const float mro = bil32(A.f + 4 * nn, nyi, m10, m20, wx0, wx1, wy0, wy1);
                    const float k = (float)(-A.heatdif * 2.0 * A.timestep);
                    float e = k * mkt / (mro * mcp) * (float)(__ldg(A.idx2 + m10) + __ldg(A.idy2 + m20));
                    if (e < -150.0f) e = -150.0f;
                    const float d1 = -dtk * expm1f(e);  // dtk (1 - exp(e))
                    T += (double)d1;
                    u.r.wx1 = wx1;
                    u.r.wy1 = wy1;
                    u.r.pv[0] = d1;
                    u.r.flag = 3u;
                }
                T += (double)tn - (double)to;
                M.T[i] = T;
            }
        }
    }
    if (payload) {
        const int64_t slot = rank ? (int64_t)__ldg(rank + i) : i;
        uint4 *d = reinterpret_cast<uint4 *>(payload) + slot * PayVec<MIXED>::R4;
#pragma unroll
        for (int q = 0; q < PayVec<MIXED>::R4; q++) d[q] = u.v[q];
    }
}

// allintert() (markmart.c:1687-1745, intermod = 0) at every marker's position,
// the point clamped to the box first (markmart.c:1697-1698): eps[2] from tk and
// eps[3] from tk2 (NULL: skipped) into out[id], out2[id] (caller order).  FP64,
// in the reference's order of operations.
static __global__ void __launch_bounds__(256) k_interp_tnode(const __grid_constant__ GridView G,
                                                      const __grid_constant__ MarkerView M,
                                                      const double *__restrict__ tk, const double *__restrict__ tk2,
                                                      double *__restrict__ out, double *__restrict__ out2)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= M.n) return;
    double x = M.x[s], y = M.y[s];
    if (x < 0) x = 0;
    else if (x > G.xsize) x = G.xsize;
    if (y < 0) y = 0;
    else if (y > G.ysize) y = G.ysize;
    int64_t m10, m20;
    double wx0, wx1, wy0, wy1;
    tweights(G, x, y, m10, m20, wx0, wx1, wy0, wy1);
    const int32_t id = M.id[s];
    out[id] = bil64(tk, G.ny, m10, m20, wx0, wx1, wy0, wy1);
    if (tk2) out2[id] = bil64(tk2, G.ny, m10, m20, wx0, wx1, wy0, wy1);
}

// sol1 = averaged diffusion change per node: 0 + the corner sums of the cells
// (m1-1,m2-1), (m1-1,m2), (m1,m2-1), (m1,m2), the same order as the node loop
static __global__ void __launch_bounds__(256) k_tnodes(const double *__restrict__ part, int64_t nx, int64_t ny,
                                                       double *__restrict__ sol1)
{
    const int64_t m3 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m3 >= nx * ny) return;
    const int64_t m1 = m3 / ny, m2 = m3 - m1 * ny, nc = (nx - 1) * (ny - 1);
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int qd = 0; qd < 4; qd++) {
        const int64_t c1 = m1 - 1 + (qd >> 1), c2 = m2 - 1 + (qd & 1);
        if (c1 < 0 || c2 < 0 || c1 > nx - 2 || c2 > ny - 2) continue;
        const int64_t cell = c1 * (ny - 1) + c2;
        const int q = 3 - qd;
        s0 += __ldg(part + (int64_t)(q * 10 + F_W0) * nc + cell);
        s1 += __ldg(part + (int64_t)(q * 10 + F_RO) * nc + cell);
    }
    sol1[m3] = s0 != 0.0 ? s1 / s0 : s1;
}

// the antidiffusion of every rock marker inside the box (the mixed form with its
// FP32 weights)
template <bool MIXED>
__global__ void __launch_bounds__(256) k_tanti(const __grid_constant__ GridView G, const __grid_constant__ MarkerView M,
                                               const double *__restrict__ sol1)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M.n) return;
    const double x = M.x[i], y = M.y[i];
    if (!(inside_box(G, x, y) && M.type[i] < 50)) return;
    int64_t m10, m20;
    using W = typename AvgCfg<MIXED>::W;
    W wx0, wx1, wy0, wy1;
    if constexpr (MIXED) tweights32(G, x, y, m10, m20, wx0, wx1, wy0, wy1);
    else tweights(G, x, y, m10, m20, wx0, wx1, wy0, wy1);
    double T = M.T[i];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const double s = __ldg(sol1 + (m10 + a) * G.ny + m20 + b);
            if (s != 0.0) T -= s * (double)((a ? wx1 : wx0) * (b ? wy1 : wy0));
        }
    M.T[i] = T;
}

}  // namespace i2g
