// FP64 instantiation of the step kernels.  Built with --fmad=false: every
// multiply and add is rounded separately, in the reference's order.
#include "i2g_avg.cuh"
#include "i2g_kernels.cuh"
#include "i2g_nodes.cuh"
#include "i2g_launch.h"

namespace i2g {

static inline unsigned grid_for(int64_t n, int threads, int64_t cap)
{
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

int launch_move_fp64(const StepLaunch &L, const MoveArgs &A, int32_t *key, int32_t *count)
{
    if (L.M.n <= 0) return 0;
    if (A.flags & I2G_MOVE_UPDATE_VISC)
        k_move<false, true><<<grid_for(L.M.n, 256, 148 * 32), 256, 0, L.stream>>>(L.G, L.M, L.types, A, key, count);
    else
        k_move<false, false><<<grid_for(L.M.n, 256, 148 * 32), 256, 0, L.stream>>>(L.G, L.M, L.types, A, key, count);
    return 1;
}

int launch_avg_fp64(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V)
{
    static bool attr = false;
    const int smem = (int)sizeof(AvgSmem<false>);
    if (!attr) {
        cudaFuncSetAttribute(k_avg<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        attr = true;
    }
    const int32_t ntx = (int32_t)((L.G.nx + V.TX - 1) / V.TX);
    const int32_t nt = avg_tiles(L.G.nx, L.G.ny, V.TX, V.TYN);
    k_avg<false><<<nt, 256, smem, L.stream>>>(L.G, L.M, V.dst, V.perm, V.cstart, L.types, A, V.T0, V.out, V.mmpart,
                                          V.TX, V.TYN, ntx, V.navg, V.slot0);
    return 1;
}

int32_t avg_tiles(int64_t nx, int64_t ny, int32_t TX, int32_t TYN)
{
    return (int32_t)(((nx + TX - 1) / TX) * ((ny + TYN - 1) / TYN));
}

int launch_clamp(cudaStream_t s, int64_t nn, const double *mmpart, int32_t nparts, double nucontr, double *nu,
                 double *nd, double *stats)
{
    k_clamp<<<grid_for(nn, 256, 148 * 4), 256, 0, s>>>(nn, mmpart, nparts, nucontr, nu, nd, stats);
    return 1;
}

}  // namespace i2g
