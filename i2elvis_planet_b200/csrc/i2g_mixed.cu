// Mixed-precision instantiation of the step kernels (FP32 weights, interpolated
// fields and property products; FP64 coordinates, RK4 sum and node sums).
#include "i2g_kernels.cuh"
#include "i2g_launch.h"

namespace i2g {

static inline unsigned grid_for(int64_t n, int threads, int64_t cap)
{
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

int launch_move_mixed(const StepLaunch &L, const MoveArgs &A, int32_t *key)
{
    if (L.M.n <= 0) return 0;
    k_move<true><<<grid_for(L.M.n, 256, 148 * 32), 256, 0, L.stream>>>(L.G, L.M, L.types, A, key);
    return 1;
}

int launch_average_mixed(const StepLaunch &L, const AvgArgsK &A, const int32_t *cstart, int64_t ncells,
                          const double *T0, double *part, unsigned long long *navg)
{
    k_cellsum<true><<<grid_for(ncells, 128, 148 * 64), 128, 0, L.stream>>>(L.G, L.M, L.types, A, cstart, ncells,
                                                                          T0, part, navg);
    return 1;
}

}  // namespace i2g
