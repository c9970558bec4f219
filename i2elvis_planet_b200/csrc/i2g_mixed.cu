// Mixed-precision instantiation of the step kernels (FP32 weights, interpolated
// fields and property products; FP64 coordinates, RK4 sum and node sums).
#include "i2g_adjoint.cuh"
#include "i2g_avg.cuh"
#include "i2g_fused.cuh"
#include "i2g_kernels.cuh"
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

int launch_move_mixed(const StepLaunch &L, const MoveArgs &A, int32_t *key, int32_t *count, int32_t *sub)
{
    if (L.M.n <= 0) return 0;
    if (A.flags & I2G_MOVE_UPDATE_VISC)
        k_move<true, true><<<grid_for(L.M.n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, L.types, A, key, count, sub);
    else
        k_move<true, false><<<grid_for(L.M.n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, L.types, A, key, count, sub);
    return 1;
}

int launch_contrib_mixed(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V)
{
    const int64_t n = L.M.n;
    if (n <= 0) return 0;
    AvgArgsK A2 = A;
    A2.rad2 = radmax_sq_threshold(L.G.xsize);
    k_contrib<true><<<grid_for(n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, V.dst, V.perm, L.types, A2, V.T0,
                                                                 V.payload, V.slot0);
    return 1;
}

int launch_td_melt_mixed(const StepLaunch &L, const TdArgs &D, int32_t gridmod, int32_t *flag, double *si)
{
    if (L.M.n <= 0) return 0;
    k_td_melt<true><<<grid_for(L.M.n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, D, gridmod, flag, si);
    return 1;
}

int launch_contrib_inplace_mixed(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V, const int32_t *rank,
                                const int32_t *key)
{
    const int64_t n = L.M.n;
    if (n <= 0) return 0;
    AvgArgsK A2 = A;
    A2.rad2 = radmax_sq_threshold(L.G.xsize);
    k_contrib_inplace<true><<<grid_for(n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, rank, key, L.types, A2, V.T0,
                                                                         V.payload);
    return 1;
}

int launch_contrib_const_mixed(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V, const int32_t *rank,
                              const int32_t *key, int32_t *deferred, int32_t *ndeferred)
{
    const int64_t n = L.M.n;
    if (n <= 0) return 0;
    AvgArgsK A2 = A;
    A2.rad2 = radmax_sq_threshold(L.G.xsize);
    // one wave of resident blocks striding over the markers: every block stages
    // the type table once (36M markers: 0.45 ms against 0.56 ms with a block per
    // 256 markers, which waited at the table's barrier)
    static int64_t wave = 0;
    if (!wave) wave = resident_blocks((const void *)k_contrib_const<true>, 256);
    const unsigned nb = grid_for(n, 256, wave);
    k_contrib_const<true><<<nb, 256, 0, L.stream>>>(L.G, L.M, rank, key, L.types, A2, V.payload, deferred, ndeferred,
                                                   static_cast<TypeConst *>(V.tab));
    k_contrib_deferred<true><<<148 * 3, 256, 0, L.stream>>>(L.G, L.M, rank, key, L.types, A2, V.T0, V.payload,
                                                            deferred, ndeferred);
    return 2;
}

template <bool CONST>
static void cellsums_mixed(const StepLaunch &L, const AvgLaunch &V)
{
    static unsigned long long attr = 0;
    const int smem = (int)sizeof(AvgSmem<true, CONST>);
    allow_dynamic_smem((const void *)k_cellsums<true, CONST>, smem, &attr);
    const int64_t nc1 = L.G.nx - 1, nc2 = L.G.ny - 1;
    const int32_t ntx = (int32_t)((nc1 + V.TX - 1) / V.TX), nty = (int32_t)((nc2 + 31) / 32);
    k_cellsums<true, CONST><<<ntx * nty, 256, smem, L.stream>>>(V.payload, V.cstart, nc1, nc2, V.part, V.TX, ntx, V.navg,
                                                            static_cast<const TypeConst *>(V.tab));
}

int launch_cellsums_mixed(const StepLaunch &L, const AvgLaunch &V)
{
    if (V.tab) cellsums_mixed<true>(L, V);
    else cellsums_mixed<false>(L, V);
    return 1;
}

int launch_avg_mixed(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V)
{
    return launch_contrib_mixed(L, A, V) + launch_cellsums_mixed(L, V);
}

int launch_adjoint_mixed(const StepLaunch &L, const MoveArgs &A, const AdjLaunch &J)
{
    const int64_t n = L.M.n;
    if (n <= 0) return 0;
    k_adj_avg<true><<<grid_for(n, 256, 148 * 16), 256, 0, L.stream>>>(L.G, L.M, L.types, J.gridmod, J.tmp_ambient, J.tk,
                                                                  J.w1, J.g, J.T0, J.lam, J.dT);
    AdjView Md{J.mvx, J.mvy, J.nmodes};
    k_adj_rk4<true><<<J.nblk, 128, 0, L.stream>>>(L.G, Md, A, L.types, J.type_by_id, J.ck, n, J.nsteps, J.every,
                                               J.lam, J.dapart);
    return 2;
}

int launch_titerate_mixed(const StepLaunch &L, const ThermArgs &A, const int32_t *rank, const AvgLaunch &V,
                         double *sol1)
{
    const int64_t n = L.M.n;
    if (n <= 0) return 0;
    const bool sums = A.heatdif != 0;
    k_tmark<true><<<grid_for(n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, rank, A, sums ? V.payload : nullptr);
    if (!sums) return 1;
    return 1 + launch_cellsums_mixed(L, V) + launch_tnodes(L, V.part, sol1) + launch_tanti_mixed(L, sol1);
}

int launch_tanti_mixed(const StepLaunch &L, const double *sol1)
{
    k_tanti<true><<<grid_for(L.M.n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, sol1);
    return 1;
}

// ----------------------------------------------------------------- fused step
size_t fused_counters_bytes() { return sizeof(FusedCounters); }
size_t fused_move_counters_bytes() { return offsetof(FusedCounters, nguard); }
size_t fused_ovf_bytes() { return sizeof(OvfRec); }

void fused_host_stats(const void *counters, int32_t *count_max, int32_t *novf)
{
    const FusedCounters *c = static_cast<const FusedCounters *>(counters);
    uint32_t m = 0;
    for (int k = 0; k < kFusedParts; k++) m = c->part[k][0] > m ? c->part[k][0] : m;
    *count_max = (int32_t)m;
    *novf = c->novf;
}

static FusedMove fused_move_args(const GridView &G, const AvgArgsK &V, const FusedLaunch &F)
{
    FusedMove M{};
    M.avg = V;
    M.avg.rad2 = radmax_sq_threshold(G.xsize);
    for (int t = 0; t < kAvgTypes; t++) M.tinfo[t] = F.tinfo[t];
    M.cap = F.cap;
    M.ra = F.ra;
    M.ovf = F.ovf;
    M.count = F.count;
    M.ctr = F.ctr;
    M.treset = F.treset;
    M.defer = F.defer;
    M.stepc = F.stepc;
    M.stepi = F.stepi;
    return M;
}

// the resident CTAs of a kernel on the current device (one wave of a persistent grid)
static unsigned resident_ctas(const void *fn, int threads, int smem = 0)
{
    int dev = 0, sms = 148, per = 1;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem) != cudaSuccess || per < 1) per = 1;
    return (unsigned)(sms * per);
}

template <bool VISC, bool UNI>
static void move_fused(const StepLaunch &L, const MoveArgs &A, const FusedMove &M)
{
    static unsigned resident = 0;  // per process: the device and kernel do not change
    if (!resident) resident = resident_ctas((const void *)k_move_fused<VISC, UNI>, kMoveTile);
    const int64_t tiles = (L.M.n + kMoveTile - 1) / kMoveTile;
    const unsigned nb = (unsigned)std::min<int64_t>(tiles, resident);
    k_move_fused<VISC, UNI><<<nb, kMoveTile, 0, L.stream>>>(L.G, L.M, L.types, A, M);
}

int launch_move_fused(const StepLaunch &L, const MoveArgs &A, const AvgArgsK &V, const FusedLaunch &F)
{
    if (L.M.n <= 0) return 0;
    const FusedMove M = fused_move_args(L.G, V, F);
    const bool visc = (A.flags & I2G_MOVE_UPDATE_VISC) != 0, uni = L.G.uni != 0;
    if (visc && uni) move_fused<true, true>(L, A, M);
    else if (visc) move_fused<true, false>(L, A, M);
    else if (uni) move_fused<false, true>(L, A, M);
    else move_fused<false, false>(L, A, M);
    k_fused_deferred<true><<<148, 128, 0, L.stream>>>(L.G, L.M, L.types, M);
    return 2;
}

// Cell-column groups per k_cellnodes CTA (node columns 8 per group, less the one
// it repeats): the CTAs of a grid take ceil(CTAs / resident) waves of 8 x groups
// columns each, so the count with the fewest column-waves fills the device best
// (at 1001 x 1001 nodes with 444 resident CTAs, 5 groups: 858 CTAs in 2 waves
// of 40 columns, where 4 groups take 1089 CTAs in 3 waves of 32); ties go to more
// groups (fewer repeated columns).
static int cellnode_groups(int nx, int ny, int resident)
{
    const int64_t nty = (ny + 30) / 31;
    int best = 4;
    int64_t cost = INT64_MAX;
    for (int g = 2; g <= 6; g++) {
        const int64_t ctas = (nx + 8 * g - 2) / (8 * g - 1) * nty;
        const int64_t c = (ctas + resident - 1) / resident * 8 * g;
        if (c <= cost) {
            cost = c;
            best = g;
        }
    }
    return best;
}

template <int NT>
static int cellnodes(const StepLaunch &L, const CellNodesArgs &Pin)
{
    static unsigned long long attr = 0;
    static unsigned resident = 0;
    const int smem = (int)sizeof(CnSmem<NT>);
    allow_dynamic_smem((const void *)k_cellnodes<NT>, smem, &attr);
    if (!resident) {
        // three CTAs of 72 KB per SM: prefer shared memory over L1 (the records are
        // read once, through cp.async)
        cudaFuncSetAttribute((const void *)k_cellnodes<NT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
        resident = resident_ctas((const void *)k_cellnodes<NT>, 256, smem);
    }
    CellNodesArgs P = Pin;
    P.ncol = 8 * cellnode_groups(P.nx, P.ny, (int)resident) - 1;
    P.ntx = (P.nx + P.ncol - 1) / P.ncol;
    const int nty = (P.ny + 30) / 31;
    k_cellnodes<NT><<<(unsigned)(P.ntx * nty), 256, smem, L.stream>>>(P);
    k_node_guard<NT><<<148, 128, 0, L.stream>>>(P);
    return 2;
}

int launch_avg_fused(const StepLaunch &L, const AvgArgsK &V, const FusedLaunch &F, const NodeOut &O)
{
    int nl = 0;
    const int64_t nn = L.G.nx * L.G.ny;
    k_fused_begin<<<148, 256, 0, L.stream>>>(L.M, F.ctr, F.treset, V.tmp_ambient, F.navg);
    nl++;
    if (F.track_tmax && L.M.tmax && L.M.n > 0) {
        AvgArgsK V2 = V;
        k_fused_tmax<<<grid_for(L.M.n, 256, kOneEach), 256, 0, L.stream>>>(L.G, L.M, V2);
        nl++;
    }
    CellNodesArgs P{};
    P.nx = (int32_t)L.G.nx;
    P.ny = (int32_t)L.G.ny;
    P.nc1 = P.nx - 1;
    P.nc2 = P.ny - 1;
    P.cap = F.cap;
    // the mobile slots: every slot but those of immobile types (markim)
    P.mob = (1u << kFusedSlots) - 1u;
    for (int t = 0; t < (int)sizeof(F.tinfo); t++)
        if (F.tinfo[t] & 4u) P.mob &= ~(1u << (F.tinfo[t] & 3u));
    P.count = F.count;
    P.ra = F.ra;
    P.ovf = F.ovf;
    P.ctr = F.ctr;
    for (int s = 0; s < kFusedSlots; s++) {
        for (int k = 0; k < 4; k++) P.sv[s][k] = F.sv[s][k];
        P.sro[s] = F.sro[s];
        P.sgrp[s] = F.sgrp[s];
    }
    P.stepc = F.stepc;
    P.stepi = F.stepi;
    P.viscmod = V.viscmod;
    P.nubeg = V.nubeg;
    P.nuend = V.nuend;
    P.mu = L.G.mu;
    P.O = O;
    P.guard = F.guard;
    P.navg = F.navg;
    switch (F.nt) {
    case 1: nl += cellnodes<1>(L, P); break;
    case 2: nl += cellnodes<2>(L, P); break;
    case 3: nl += cellnodes<3>(L, P); break;
    default: nl += cellnodes<4>(L, P); break;
    }
    // a node per thread: every node's two loads in flight at once
    k_fused_clamp<<<grid_for(nn, 256, kOneEach), 256, 0, L.stream>>>(nn, F.ctr, F.nucontr, O.nu, O.nd, F.stats);
    return nl + 1;
}

__global__ void k_count_max(const int32_t *__restrict__ count, int64_t n, int32_t *out)
{
    int32_t m = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, count[i]);
    m = __reduce_max_sync(0xffffffffu, (unsigned)m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

int launch_count_max(cudaStream_t s, const int32_t *count, int64_t ncells, int32_t *out)
{
    k_count_max<<<grid_for(ncells, 256, 148 * 8), 256, 0, s>>>(count, ncells, out);
    return 1;
}

// Loads the step's kernels of this form now, not at their first launch (lazy
// module loading), so that no step carries a load in its time.
void preload_mixed()
{
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_move<true, true>);
    cudaFuncGetAttributes(&a, k_move<true, false>);
    cudaFuncGetAttributes(&a, k_contrib<true>);
    cudaFuncGetAttributes(&a, k_contrib_inplace<true>);
    cudaFuncGetAttributes(&a, k_contrib_const<true>);
    cudaFuncGetAttributes(&a, k_contrib_deferred<true>);
    cudaFuncGetAttributes(&a, k_cellsums<true, false>);
    cudaFuncGetAttributes(&a, k_cellsums<true, true>);
    cudaFuncGetAttributes(&a, k_tmark<true>);
    cudaFuncGetAttributes(&a, k_tanti<true>);
    cudaFuncGetAttributes(&a, k_move_fused<false, true>);
    cudaFuncGetAttributes(&a, k_move_fused<false, false>);
    cudaFuncGetAttributes(&a, k_move_fused<true, true>);
    cudaFuncGetAttributes(&a, k_move_fused<true, false>);
    cudaFuncGetAttributes(&a, k_cellnodes<1>);
    cudaFuncGetAttributes(&a, k_cellnodes<2>);
    cudaFuncGetAttributes(&a, k_cellnodes<3>);
    cudaFuncGetAttributes(&a, k_cellnodes<4>);
    cudaFuncGetAttributes(&a, k_node_guard<3>);
    cudaFuncGetAttributes(&a, k_fused_deferred<true>);
    cudaFuncGetAttributes(&a, k_fused_begin);
    cudaFuncGetAttributes(&a, k_fused_clamp);
}

}  // namespace i2g
