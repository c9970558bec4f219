// FP64 instantiation of the step kernels.  Built with --fmad=false: every
// multiply and add is rounded separately, in the reference's order.
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

int launch_move_fp64(const StepLaunch &L, const MoveArgs &A, int32_t *key)
{
    if (L.M.n <= 0) return 0;
    k_move<false><<<grid_for(L.M.n, 256, 148 * 32), 256, 0, L.stream>>>(L.G, L.M, L.types, A, key);
    return 1;
}

int launch_average_fp64(const StepLaunch &L, const AvgArgsK &A, const int32_t *cstart, int64_t ncells,
                         const double *T0, double *part, unsigned long long *navg)
{
    k_cellsum<false><<<grid_for(ncells, 128, 148 * 64), 128, 0, L.stream>>>(L.G, L.M, L.types, A, cstart, ncells,
                                                                           T0, part, navg);
    return 1;
}

int32_t nodesum_blocks(int64_t nn) { return (int32_t)((nn + 255) / 256); }

int launch_nodes(cudaStream_t s, const GridView &G, const double *part, int64_t ncells, const NodeOut &O,
                  double nubeg, double nuend, int32_t viscmod, double nucontr, double *mmpart, double *stats)
{
    const int64_t nn = G.nx * G.ny;
    const int32_t nb = nodesum_blocks(nn);
    k_nodesum<<<nb, 256, 0, s>>>(G, part, ncells, O, nubeg, nuend, viscmod, mmpart);
    k_clamp<<<grid_for(nn, 256, 148 * 4), 256, 0, s>>>(nn, mmpart, nb, nucontr, O.nu, O.nd, stats);
    return 2;
}

}  // namespace i2g
