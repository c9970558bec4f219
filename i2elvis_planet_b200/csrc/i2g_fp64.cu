// FP64 instantiation of the step kernels.  Built with --fmad=false: every
// multiply and add is rounded separately, in the reference's order.
#include "i2g_adjoint.cuh"
#include "i2g_avg.cuh"
#include "i2g_kernels.cuh"
#include "i2g_nodes.cuh"
#include "i2g_launch.h"
#include "i2g_thermal.cuh"

namespace i2g {

// One thread per element for the marker kernels: the block scheduler balances
// the blocks over the SMs, where a grid-stride loop over a capped grid that is
// not a multiple of the resident blocks leaves a partial last wave running for
// the whole loop.  (Their struct parameters are grid constants, so a block
// starts without copying them to local memory.)
constexpr int64_t kOneEach = INT32_MAX;

static inline unsigned grid_for(int64_t n, int threads, int64_t cap)
{
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

int launch_move_fp64(const StepLaunch &L, const MoveArgs &A, int32_t *key, int32_t *count, int32_t *sub)
{
    if (L.M.n <= 0) return 0;
    if (A.flags & I2G_MOVE_UPDATE_VISC)
        k_move<false, true><<<grid_for(L.M.n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, L.types, A, key, count, sub);
    else
        k_move<false, false><<<grid_for(L.M.n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, L.types, A, key, count, sub);
    return 1;
}

int launch_contrib_fp64(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V)
{
    const int64_t n = L.M.n;
    if (n <= 0) return 0;
    AvgArgsK A2 = A;
    A2.rad2 = radmax_sq_threshold(L.G.xsize);
    k_contrib<false><<<grid_for(n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, V.dst, V.perm, L.types, A2, V.T0,
                                                                 V.payload, V.slot0);
    return 1;
}

int launch_td_melt_fp64(const StepLaunch &L, const TdArgs &D, int32_t gridmod, int32_t *flag, double *si)
{
    if (L.M.n <= 0) return 0;
    k_td_melt<false><<<grid_for(L.M.n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, D, gridmod, flag, si);
    return 1;
}

int launch_contrib_inplace_fp64(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V, const int32_t *rank,
                                const int32_t *key)
{
    const int64_t n = L.M.n;
    if (n <= 0) return 0;
    AvgArgsK A2 = A;
    A2.rad2 = radmax_sq_threshold(L.G.xsize);
    k_contrib_inplace<false><<<grid_for(n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, rank, key, L.types, A2, V.T0,
                                                                         V.payload);
    return 1;
}

int launch_contrib_const_fp64(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V, const int32_t *rank,
                              const int32_t *key, int32_t *deferred, int32_t *ndeferred)
{
    const int64_t n = L.M.n;
    if (n <= 0) return 0;
    AvgArgsK A2 = A;
    A2.rad2 = radmax_sq_threshold(L.G.xsize);
    // a block per 256 markers (one wave of resident blocks, as in the mixed form,
    // measured slower here: 1.07 against 0.96 ms at 36M markers)
    const unsigned nb = grid_for(n, 256, kOneEach);
    k_contrib_const<false><<<nb, 256, 0, L.stream>>>(L.G, L.M, rank, key, L.types, A2, V.payload, deferred, ndeferred,
                                                   static_cast<TypeConst *>(V.tab));
    k_contrib_deferred<false><<<148 * 3, 256, 0, L.stream>>>(L.G, L.M, rank, key, L.types, A2, V.T0, V.payload,
                                                            deferred, ndeferred);
    return 2;
}

template <bool CONST>
static void cellsums_fp64(const StepLaunch &L, const AvgLaunch &V)
{
    static unsigned long long attr = 0;
    const int smem = (int)sizeof(AvgSmem<false, CONST>);
    allow_dynamic_smem((const void *)k_cellsums<false, CONST>, smem, &attr);
    const int64_t nc1 = L.G.nx - 1, nc2 = L.G.ny - 1;
    const int32_t ntx = (int32_t)((nc1 + V.TX - 1) / V.TX), nty = (int32_t)((nc2 + 31) / 32);
    k_cellsums<false, CONST><<<ntx * nty, 256, smem, L.stream>>>(V.payload, V.cstart, nc1, nc2, V.part, V.TX, ntx, V.navg,
                                                            static_cast<const TypeConst *>(V.tab));
}

int launch_cellsums_fp64(const StepLaunch &L, const AvgLaunch &V)
{
    if (V.tab) cellsums_fp64<true>(L, V);
    else cellsums_fp64<false>(L, V);
    return 1;
}

int launch_avg_fp64(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V)
{
    return launch_contrib_fp64(L, A, V) + launch_cellsums_fp64(L, V);
}

int32_t nodesum_blocks(int64_t nn) { return (int32_t)((nn + 255) / 256); }

int launch_nodes(cudaStream_t s, const GridView &G, const double *part, const AvgArgsK &A, const NodeOut &O,
                 double nucontr, double *mmpart, double *stats)
{
    const int64_t nn = G.nx * G.ny;
    const int32_t nb = nodesum_blocks(nn);
    k_nodesums<<<nb, 256, 0, s>>>(G, part, A, O, mmpart);
    k_clamp<<<grid_for(nn, 256, 148 * 4), 256, 0, s>>>(nn, mmpart, nb, nucontr, O.nu, O.nd, stats);
    return 2;
}

int launch_adjoint_fp64(const StepLaunch &L, const MoveArgs &A, const AdjLaunch &J)
{
    const int64_t n = L.M.n;
    if (n <= 0) return 0;
    k_adj_avg<false><<<grid_for(n, 256, 148 * 16), 256, 0, L.stream>>>(L.G, L.M, L.types, J.gridmod, J.tmp_ambient, J.tk,
                                                                  J.w1, J.g, J.T0, J.lam, J.dT);
    AdjView Md{J.mvx, J.mvy, J.nmodes};
    k_adj_rk4<false><<<J.nblk, 128, 0, L.stream>>>(L.G, Md, A, L.types, J.type_by_id, J.ck, n, J.nsteps, J.every,
                                               J.lam, J.dapart);
    return 2;
}

int launch_interp_tnode(const StepLaunch &L, const double *tk, const double *tk2, double *out, double *out2)
{
    if (L.M.n <= 0) return 0;
    k_interp_tnode<<<grid_for(L.M.n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, tk, tk2, out, out2);
    return 1;
}

int launch_titerate_fp64(const StepLaunch &L, const ThermArgs &A, const int32_t *rank, const AvgLaunch &V,
                         double *sol1)
{
    const int64_t n = L.M.n;
    if (n <= 0) return 0;
    const bool sums = A.heatdif != 0;
    k_tmark<false><<<grid_for(n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, rank, A, sums ? V.payload : nullptr);
    if (!sums) return 1;
    return 1 + launch_cellsums_fp64(L, V) + launch_tnodes(L, V.part, sol1) + launch_tanti_fp64(L, sol1);
}

// the node averages of the diffusion changes (both forms)
int launch_tnodes(const StepLaunch &L, const double *part, double *sol1)
{
    const int64_t nn = L.G.nx * L.G.ny;
    k_tnodes<<<grid_for(nn, 256, kOneEach), 256, 0, L.stream>>>(part, L.G.nx, L.G.ny, sol1);
    return 1;
}

int launch_tanti_fp64(const StepLaunch &L, const double *sol1)
{
    k_tanti<false><<<grid_for(L.M.n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, sol1);
    return 1;
}

// Loads the step's kernels of this form now, not at their first launch (lazy
// module loading), so that no step carries a load in its time.
void preload_fp64()
{
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_move<false, true>);
    cudaFuncGetAttributes(&a, k_move<false, false>);
    cudaFuncGetAttributes(&a, k_contrib<false>);
    cudaFuncGetAttributes(&a, k_contrib_inplace<false>);
    cudaFuncGetAttributes(&a, k_contrib_const<false>);
    cudaFuncGetAttributes(&a, k_contrib_deferred<false>);
    cudaFuncGetAttributes(&a, k_cellsums<false, false>);
    cudaFuncGetAttributes(&a, k_cellsums<false, true>);
    cudaFuncGetAttributes(&a, k_tmark<false>);
    cudaFuncGetAttributes(&a, k_tanti<false>);
    cudaFuncGetAttributes(&a, k_tnodes);
    cudaFuncGetAttributes(&a, k_nodesums);
    cudaFuncGetAttributes(&a, k_clamp);
}

}  // namespace i2g
