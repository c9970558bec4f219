// Host-side launcher declarations shared by the translation units of libi2g.
// Every launcher returns the number of kernels it launched.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "i2g_dev.cuh"

namespace i2g {

// AvgArgsK::rad2 for a box of width xsize: the smallest double s with
// pow(s, 0.5) > 0.95 * xsize / 2 in the host's libm -- the reference's own test
// (markmart.c:268, 335-340), whose pow is not correctly rounded, so a search with
// sqrt can land one double off (for about 0.2% of box widths)
inline double radmax_sq_threshold(double xsize)
{
    const double R = xsize / 2.0 * 0.95;
    double s = R * R;
    if (!std::isfinite(s) || !(R > 0)) return s;
    while (s > 0 && std::pow(s, 0.5) > R) s = std::nextafter(s, 0.0);
    while (!(std::pow(s, 0.5) > R)) s = std::nextafter(s, INFINITY);
    return s;
}

// bytes of the averaging payload for n markers (one PayRec each, i2g_avg.cuh)
__host__ __device__ constexpr int64_t payload_bytes(bool mixed, int64_t n) { return n * (mixed ? 48 : 96); }

// scratch of the cell sort
struct SortBufs {
    int32_t *key;     // [cap] cell of every marker (device order)
    int32_t *perm1;   // [cap] slot -> previous slot, cell-grouped
    int32_t *perm2;   // [cap] same, canonical order inside each cell
    int32_t *rank;    // [cap] inverse of perm2 (rank_markers; NULL: not needed)
    int32_t *count;   // [ncells]
    int32_t *cursor;  // [ncells]
    int32_t *cstart;  // [ncells + 1]
    int32_t *tilesum; // scan scratch
    int64_t *slot0;   // slot that holds caller marker 0
};

int scan_exclusive(cudaStream_t s, const int32_t *in, int64_t n, int32_t *out, int32_t *tilesum);
int64_t scan_max_elems();
int sort_markers(cudaStream_t s, const SortBufs &B, int64_t n, int64_t ncells, MarkerView src, MarkerView dst);
// counting sort by key without moving data: perm2[slot] = current index;
// counts_ready: count[] already holds the per-cell counts (k_move computed them)
int rank_markers(cudaStream_t s, const SortBufs &B, int64_t n, int64_t ncells, const int32_t *id,
                 bool counts_ready);
// the same after a movemark: counts and arrival indices (sub) from k_move
int rank_moved(cudaStream_t s, const SortBufs &B, int64_t n, int64_t ncells, const int32_t *id,
               const int32_t *sub);
int launch_keys(cudaStream_t s, const GridView &G, const double *x, const double *y, int64_t n, int32_t *key);
int launch_iota(cudaStream_t s, int32_t *a, int64_t n);
int launch_unsort_f64(cudaStream_t s, int64_t n, const int32_t *id, const double *in, double *out);
int launch_unsort_i8(cudaStream_t s, int64_t n, const int32_t *id, const int8_t *in, int8_t *out);
int launch_unsort_f64_f32(cudaStream_t s, int64_t n, const int32_t *id, const double *in, float *out);
// markers in the caller's order (FP64, or FP32 when f32) -> cell keys; -> sorted device order
int launch_keys_in(cudaStream_t s, const GridView &G, const void *x, const void *y, int64_t n, bool f32,
                   int32_t *key);
int launch_gather_in_xy(cudaStream_t s, int64_t n, const int32_t *perm, const void *x, const void *y, bool f32,
                        const MarkerView &dst, int64_t *slot0);
int launch_gather_in_rest(cudaStream_t s, int64_t n, const int32_t *perm, const void *T, const void *eta,
                          const int8_t *type, bool f32, const MarkerView &dst);
int launch_f64_to_f32(cudaStream_t s, int64_t n, const double *in, float *out);
int launch_f32_to_f64(cudaStream_t s, int64_t n, const float *in, double *out);
int launch_t0(cudaStream_t s, const GridView &G, const MarkerView &M, const int64_t *slot0, double tmp_ambient,
               double *T0);

// precision-specific step kernels (i2g_fp64.cu is built with --fmad=false)
struct StepLaunch {
    cudaStream_t stream;
    GridView G;
    MarkerView M;
    const DevTypes *types;
};
// k_move also counts markers per new cell into count[] (zeroed by the caller)
int launch_move_fp64(const StepLaunch &L, const MoveArgs &A, int32_t *key, int32_t *count, int32_t *sub);
int launch_move_mixed(const StepLaunch &L, const MoveArgs &A, int32_t *key, int32_t *count, int32_t *sub);
// marker contributions + cell sums (i2g_avg.cuh): L.M is the current device
// order, dst receives the sorted order; perm NULL = L.M is sorted already
struct AvgLaunch {
    MarkerView dst;
    const int32_t *perm;
    const int32_t *cstart;
    const double *T0;
    void *payload;  // payload_bytes(precision, markers) bytes
    double *part;  // [kPart][ncells] cell corner sums
    int32_t TX;    // cell columns per tile (tile height is 32 cell rows)
    unsigned long long *navg;
    int64_t *slot0;
    // the per-type table of a constant-property call (the payload holds the
    // compact records then; k_contrib_const writes it), NULL otherwise
    void *tab;
};
constexpr size_t kTypeConstBytes = 2048;  // device bytes of that table

// Blocks of `threads` threads of kernel f resident on the current device at once
// (occupancy x SMs), at least 1.
inline int64_t resident_blocks(const void *f, int threads)
{
    int dev = 0, occ = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, threads, 0);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t r = (int64_t)(occ > 0 ? occ : 1) * (sms > 0 ? sms : 1);
    return r;
}

// Allows `bytes` of dynamic shared memory for kernel f.  The attribute belongs
// to the current device, so it is set once per device (bit d of *done).
inline void allow_dynamic_smem(const void *f, int bytes, unsigned long long *done)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (*done & bit)) return;
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    *done |= bit;
}
int launch_avg_fp64(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V);
int launch_avg_mixed(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V);
// the two halves of launch_avg_*: k_contrib, then k_cellsums
int launch_contrib_fp64(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V);
int launch_contrib_mixed(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V);
int launch_cellsums_fp64(const StepLaunch &L, const AvgLaunch &V);
// k_contrib without moving the markers: L.M stays in its (stale) storage order,
// its cell keys in key[], the payload goes to slot rank[i]; updates T, tmax, por in place
int launch_contrib_inplace_fp64(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V, const int32_t *rank,
                                const int32_t *key);
int launch_contrib_inplace_mixed(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V, const int32_t *rank,
                                 const int32_t *key);
// the same when every averaged type has constant properties (const_properties_call):
// a lean kernel, then the general model for the deferred markers (*ndeferred = 0 first)
int launch_contrib_const_fp64(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V, const int32_t *rank,
                              const int32_t *key, int32_t *deferred, int32_t *ndeferred);
int launch_contrib_const_mixed(const StepLaunch &L, const AvgArgsK &A, const AvgLaunch &V, const int32_t *rank,
                               const int32_t *key, int32_t *deferred, int32_t *ndeferred);
int launch_cellsums_mixed(const StepLaunch &L, const AvgLaunch &V);
// densimod 2: the table markers of the call and the eps[21] each leaves, by caller
// index (k_td_melt), then every caller index's last table marker so far (an
// inclusive max-scan over n; tmp NULL: *bytes = the scratch the scan needs).
// The scan returns -1 on a CUDA error.
int launch_td_melt_fp64(const StepLaunch &L, const TdArgs &D, int32_t gridmod, int32_t *flag, double *si);
int launch_td_melt_mixed(const StepLaunch &L, const TdArgs &D, int32_t gridmod, int32_t *flag, double *si);
int td_prev_scan(cudaStream_t s, void *tmp, size_t *bytes, const int32_t *flag, int32_t *prev, int64_t n);
// node loop over the cell sums + contrast clamp (precision independent: FP64)
int32_t nodesum_blocks(int64_t nn);
// titerate()'s marker temperature update (i2g_thermal.cuh): k_tmark, and when
// heatdif != 0 the cell sums, k_tnodes and k_tanti; returns the launch count
struct ThermArgs {
    const double *tkn, *tko;     // node T after / before the thermal solve
    const double *kt, *cp, *ro;  // node conductivity, heat capacity, density
    const float *f;              // mixed form: FP32 copies of the five, 5 x nodes
    const double *idx2, *idy2;   // per grid line 1.0/d/d, d = g[i+1]-g[i]
    double heatdif, timestep;
};
int launch_titerate_fp64(const StepLaunch &L, const ThermArgs &A, const int32_t *rank, const AvgLaunch &V,
                         double *sol1);
int launch_titerate_mixed(const StepLaunch &L, const ThermArgs &A, const int32_t *rank, const AvgLaunch &V,
                          double *sol1);
int launch_tnodes(const StepLaunch &L, const double *part, double *sol1);
int launch_tanti_fp64(const StepLaunch &L, const double *sol1);
int launch_tanti_mixed(const StepLaunch &L, const double *sol1);
// load the step's kernels into the current context (lazy module loading)
void preload_mixed();
void preload_fp64();
void preload_sort();
int launch_nodes(cudaStream_t s, const GridView &G, const double *part, const AvgArgsK &A, const NodeOut &O,
                 double nucontr, double *mmpart, double *stats);

// ----------------------------------------------------------------- fused mixed step
// movemark with the averaging records (k_move_fused) and the averaging from them
// (i2g_fused.cuh); device state of a context's fused path
struct FusedCounters;
struct OvfRec;
constexpr int kFusedSlots = 4;  // rock types (< 50) a fused call can average
struct FusedLaunch {
    int32_t cap;          // places per cell bucket (even)
    float4 *ra;           // [ncells * cap]
    OvfRec *ovf;          // [markers]
    int32_t *count;       // [ncells]
    FusedCounters *ctr;
    int32_t *treset;      // [markers]
    int2 *defer;          // [markers]
    int32_t *guard;       // [nodes]
    uint8_t tinfo[50];    // per rock type < 50: slot | immobile << 2
    int32_t nt;           // slots in use, 1..kFusedSlots
    double sv[kFusedSlots][4];  // per slot: ro, cp, kt, ht of this call
    // a step replayed from a CUDA graph: timesum and the radiogenic rates from
    // the step's row of a device table {timesum, rad_si, rad_fe, rad_ch}
    // (stepc[4 * *stepi]); per slot the density and rate group (1..3, 0 = none)
    // the heat is formed from; NULL for a step launched directly
    const double *stepc;
    const int32_t *stepi;
    double sro[kFusedSlots];
    int32_t sgrp[kFusedSlots];
    unsigned long long *navg;
    double nucontr;
    double *stats;
    bool track_tmax;
};
size_t fused_counters_bytes();
size_t fused_move_counters_bytes();  // the leading part k_move_fused needs zeroed
size_t fused_ovf_bytes();            // bytes of one overflow record
// largest cell count and overflow count from a host copy of the counters
void fused_host_stats(const void *counters, int32_t *count_max, int32_t *novf);
int launch_move_fused(const StepLaunch &L, const MoveArgs &A, const AvgArgsK &V, const FusedLaunch &F);
int launch_avg_fused(const StepLaunch &L, const AvgArgsK &V, const FusedLaunch &F, const NodeOut &O);
// max over cells of count[] into *out (device int, zeroed by the caller)
int launch_count_max(cudaStream_t s, const int32_t *count, int64_t ncells, int32_t *out);

// ----------------------------------------------------------------- batches
// device description of one instance of a batch (i2g_batch.cuh)
struct InstDesc {
    GridView G;
    MarkerView buf[2];
    int32_t cur;  // current buffer, flipped on the device at the end of each step
    int32_t track_tmax;
    SortBufs sb;
    const DevTypes *types;
    double *part, *mmpart, *stats, *T0;
    unsigned long long *navg;
    NodeOut O;
    void *payload;
    MoveArgs move;
    AvgArgsK avg;
    double nucontr;
    int64_t n, ncells, nn;
    int32_t ntx, nblk;
    const double *stepc;  // [steps][4]: timesum, rad_si, rad_fe, rad_ch
};

struct BatchRun {
    InstDesc *D;
    int32_t ninst;
    const int64_t *off_mark, *off_cell, *off_tile, *off_nblk;  // [ninst + 1] prefix offsets
    int64_t tot_mark, tot_cell, tot_tile, tot_nblk;
    int32_t *step;  // device step index within the current i2g_batch_step call
    int32_t TX;
};

int launch_batch_step_fp64(cudaStream_t s, const BatchRun &R, int move_ctas, int cell_ctas);
int launch_batch_step_mixed(cudaStream_t s, const BatchRun &R, int move_ctas, int cell_ctas);
int avg_smem_bytes(bool mixed);

// ----------------------------------------------------------------- adjoint
struct AdjLaunch {
    const double *mvx, *mvy;  // [nn][nmodes]
    int32_t nmodes;
    const double *tk, *w1, *g, *T0;
    double2 *lam;
    double *dT;
    const int8_t *type_by_id;
    const double2 *ck;
    int32_t nsteps, every;
    double *dapart;
    int32_t nblk;
    int32_t gridmod;
    double tmp_ambient;
};
int launch_adjoint_fp64(const StepLaunch &L, const MoveArgs &A, const AdjLaunch &J);
int launch_adjoint_mixed(const StepLaunch &L, const MoveArgs &A, const AdjLaunch &J);
// vx = sum_m a_m mvx[.][m] (FP64, fixed order), float copies when vxf != NULL
int launch_quads(cudaStream_t s, int64_t nx, int64_t ny, const float *f, float4 *q);
// allintert() at every marker (k_interp_tnode, FP64 in both forms): out[id], out2[id]
int launch_interp_tnode(const StepLaunch &L, const double *tk, const double *tk2, double *out, double *out2);
// the per-quarter-cell forms of vx and vy (GridView.vq4) of a uniform grid
int launch_quarters(cudaStream_t s, int64_t nx, int64_t ny, const float *vxf, const float *vyf, float4 *q);
int launch_combine_modes(cudaStream_t s, int64_t nn, int32_t nm, const double *mvx, const double *mvy,
                         const double *amps, double *vx, double *vy, float *vxf, float *vyf);
int launch_ckpt(cudaStream_t s, const MarkerView &M, double2 *ck);
int launch_sum_partials(cudaStream_t s, const double *part, int32_t nblk, int32_t nm, double *out);

}  // namespace i2g
