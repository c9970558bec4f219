// Marker -> cell averaging (the ronurecalc() marker loop, markmart.c:271-913) in
// two kernels, and the node loop (markmart.c:917-993) in i2g_nodes.cuh.
//
// k_contrib: one thread per slot of the new, cell-sorted device order (cell,
//   then caller index).  It gathers the slot's marker from the current order
//   through the sort permutation (markers move less than a cell per step, so the
//   gathers are nearly local), evaluates the property model and the marker's
//   bilinear weights (marker_contrib), and writes the marker record (the sort's
//   data movement costs no extra pass) and its contribution (one payload record)
//   to the slot: coalesced stores.
// k_contrib_inplace: the same contributions without moving the records: one
//   thread per marker in its storage order (coalesced reads), the payload
//   record scattered to the marker's slot.  The context runs it on all but every
//   reorder_every-th call, so the storage order stays close to cell order.
// k_cellsums: the per-cell corner sums, one warp per column strip of 32 cells
//   (see cellsums_tile): each lane adds its cell's markers in slot order into
//   FP64 registers, a fixed-order segmented reduction.
// No atomics touch a node value; the result does not depend on the tile shape,
// the launch configuration or the device order the markers arrive in.
#pragma once

#include "i2g_kernels.cuh"
#include "i2g_launch.h"

namespace i2g {

template <bool MIXED>
struct AvgCfg {
    using W = typename std::conditional<MIXED, float, double>::type;  // weights, property values
};

// The averaging payload: one record per marker, in its slot of the sorted
// order, 16-byte aligned and moved as uint4 (payload_bytes(MIXED, n) bytes).
//   pv = ro, et (beta), cp, kt, ht, tk: the property values the sums weight;
//   the mixed form's w0 is 1.0f - w1 exactly (fdw32), so it is not stored;
//   flag: bit0 averaged, bit1 immobile type.
template <bool MIXED>
struct PayRec;
template <>
struct __align__(16) PayRec<true> {  // 48 bytes
    double lnu;
    float wx1, wy1;
    float pv[6];
    uint32_t flag, pad;
};
template <>
struct __align__(16) PayRec<false> {  // 96 bytes
    double wx0, wx1, wy0, wy1;
    double pv[6];
    double lnu;
    uint32_t flag, pad;
};
static_assert(sizeof(PayRec<true>) == payload_bytes(true, 1), "mixed payload record size");
static_assert(sizeof(PayRec<false>) == payload_bytes(false, 1), "FP64 payload record size");

// The payload record of a constant-property call (k_contrib_const): density,
// heat capacity, conductivity and heat are functions of the rock type alone
// there, so the record carries the type and k_cellsums reads the values from a
// per-type table (TypeConst); beta (et) is zero.
//   tf: flag (bit0 averaged, bit1 immobile type) | type << 8.
template <bool MIXED>
struct PayConst;
template <>
struct __align__(16) PayConst<true> {  // 32 bytes
    double lnu;
    float wx1, wy1;
    float tk;
    uint32_t tf;
    uint32_t pad[2];
};
template <>
struct __align__(16) PayConst<false> {  // 64 bytes
    double wx0, wx1, wy0, wy1;
    double lnu, tk;
    uint32_t tf, pad[3];
};
static_assert(sizeof(PayConst<true>) == 32 && sizeof(PayConst<false>) == 64, "constant-call record sizes");

template <bool MIXED, bool CONST = false>
union PayVec {
    using Rec = typename std::conditional<CONST, PayConst<MIXED>, PayRec<MIXED>>::type;
    static constexpr int R4 = sizeof(Rec) / 16;  // uint4 per record
    Rec r;
    uint4 v[R4];
};

// Per-type constants of the property model for the types the averaging takes
// (< kAvgTypes), for calls where every such type has constant properties:
// densimod 0, no temperature or pressure term in the conductivity, no molten
// material at this time, porosity not tracked.  Then marker_contrib reduces, for a
// marker with its own viscosity (eta > 0), to these values -- computed with the
// same operations -- plus the marker's temperature, viscosity and weights.
struct TypeConst {
    double ro[kAvgTypes], cp[kAvgTypes], kt[kAvgTypes], ht[kAvgTypes];
    uint8_t im[kAvgTypes];
};

static_assert(sizeof(TypeConst) <= kTypeConstBytes, "type table buffer");

// the same in k_cellsums' shared memory: values rounded to the form's type W
// (as the general record stores them) and widened back, so the sums need no
// conversion per marker
struct TypeTabD {
    double ro[kAvgTypes], cp[kAvgTypes], kt[kAvgTypes], ht[kAvgTypes];
};

// Slot j of the sorted order: the marker perm[j] of the current order (j itself
// when perm is NULL: the order is sorted already) -- property model at its cell,
// record and payload into slot j.
template <bool MIXED>
__device__ __forceinline__ void contrib_marker(const GridView &G, const MarkerView &A, const MarkerView &B,
                                               const int32_t *__restrict__ perm, const i2g_types &T,
                                               const AvgArgsK &args, double T0, uint4 *__restrict__ P, int64_t j,
                                               int64_t *slot0)
{
    using W = typename AvgCfg<MIXED>::W;
    const bool has_tmax = A.tmax != nullptr, has_por = A.por != nullptr, has_hi = A.hi != nullptr;
    const int64_t i = perm ? (int64_t)__ldg(perm + j) : j;
    MarkerRec r;
    r.x = A.x[i];
    r.y = A.y[i];
    r.T = A.T[i];
    r.eta = A.eta[i];
    r.p = A.p[i];
    r.type = A.type[i];
    r.id = A.id[i];
    r.tmax = has_tmax ? A.tmax[i] : 0.0;
    r.hi = has_hi ? A.hi[i] : 0.0;
    r.por = has_por ? A.por[i] : 0.0;
    r.mgo = A.mgo ? A.mgo[i] : 3;
    r.mgt = A.mgo ? A.mgt[i] : -1.0;
    // the marker's cell: the cell the sort filed it under (cell_key)
    double xc = r.x, yc = r.y;
    clampxy(G, xc, yc);
    const int64_t m10 = cell_search(G.gx, G.nx, G.inv_x, xc), m20 = cell_search(G.gy, G.ny, G.inv_y, yc);
    MarkerContrib mc;
    const bool ok = (args.gridmod <= 1 || (r.id % args.gridmod) == 0) && r.type >= 0 &&
                    marker_contrib<MIXED>(G, T, args, T0, r, has_tmax && args.track_tmax, has_por, m10, m20, mc);
    B.x[j] = r.x;
    B.y[j] = r.y;
    B.T[j] = r.T;
    B.eta[j] = r.eta;
    B.p[j] = r.p;
    B.type[j] = (int8_t)r.type;
    B.id[j] = r.id;
    if (has_tmax) B.tmax[j] = r.tmax;
    if (has_hi) B.hi[j] = r.hi;
    if (has_por) B.por[j] = r.por;
    if (A.mgo) {
        B.mgo[j] = (int8_t)r.mgo;
        B.mgt[j] = r.mgt;
    }
    if (r.id == 0) *slot0 = j;
    PayVec<MIXED> u;
#pragma unroll
    for (int k = 0; k < PayVec<MIXED>::R4; k++) u.v[k] = make_uint4(0u, 0u, 0u, 0u);
    if (ok) {
        if constexpr (!MIXED) {
            u.r.wx0 = (W)mc.wx0;
            u.r.wy0 = (W)mc.wy0;
        }
        u.r.wx1 = (W)mc.wx1;
        u.r.wy1 = (W)mc.wy1;
        u.r.pv[0] = (W)mc.mro;
        u.r.pv[1] = (W)mc.mbb;
        u.r.pv[2] = (W)mc.mcp;
        u.r.pv[3] = (W)mc.mkt;
        u.r.pv[4] = (W)mc.mht;
        u.r.pv[5] = (W)mc.mtk;
        u.r.lnu = mc.lnu;
        u.r.flag = 1u | (mc.immobile ? 2u : 0u);
    }
    uint4 *d = P + j * PayVec<MIXED>::R4;
#pragma unroll
    for (int k = 0; k < PayVec<MIXED>::R4; k++) d[k] = u.v[k];
}

// One marker of the averaging in its storage order, without moving it: its cell
// is its key (cell_key, written by movemark for the current position); the
// record's side effects (sticky-air T, tmax, porosity) are written back in
// place and its payload goes to its slot rank[i] of the sorted order.
template <bool MIXED, bool CONST = false>
__device__ __forceinline__ void contrib_inplace(const GridView &G, const MarkerView &A,
                                                const int32_t *__restrict__ rank, const int32_t *__restrict__ key,
                                                const i2g_types &T, const AvgArgsK &args, double T0,
                                                uint4 *__restrict__ P, int64_t i)
{
    using W = typename AvgCfg<MIXED>::W;
    const bool has_tmax = A.tmax != nullptr, has_por = A.por != nullptr, has_hi = A.hi != nullptr;
    MarkerRec r;
    r.x = A.x[i];
    r.y = A.y[i];
    r.T = A.T[i];
    r.eta = A.eta[i];
    r.p = 0.0;
    r.type = A.type[i];
    r.id = A.id[i];
    r.tmax = has_tmax ? A.tmax[i] : 0.0;
    r.hi = has_hi ? A.hi[i] : 0.0;
    r.por = has_por ? A.por[i] : 0.0;
    r.mgo = A.mgo ? A.mgo[i] : 3;
    r.mgt = A.mgo ? A.mgt[i] : -1.0;
    const double T_in = r.T, tmax_in = r.tmax, por_in = r.por;
    const int type_in = r.type;
    const int32_t k = __ldg(key + i);
    const int32_t nc2 = (int32_t)(G.ny - 1);
    const int32_t m10 = k / nc2, m20 = k - m10 * nc2;
    MarkerContrib mc;
    const bool ok = (args.gridmod <= 1 || (r.id % args.gridmod) == 0) && r.type >= 0 &&
                    marker_contrib<MIXED>(G, T, args, T0, r, has_tmax && args.track_tmax, has_por, m10, m20, mc);
    if (r.T != T_in) A.T[i] = r.T;
    if (r.type != type_in) A.type[i] = (int8_t)r.type;  // the table path's melt flip
    if (has_tmax && r.tmax != tmax_in) A.tmax[i] = r.tmax;
    if (has_por && r.por != por_in) A.por[i] = r.por;
    if (A.mgo) {
        A.mgo[i] = (int8_t)r.mgo;
        A.mgt[i] = r.mgt;
    }
    PayVec<MIXED, CONST> u;
#pragma unroll
    for (int q = 0; q < PayVec<MIXED, CONST>::R4; q++) u.v[q] = make_uint4(0u, 0u, 0u, 0u);
    if (ok) {
        if constexpr (!MIXED) {
            u.r.wx0 = (W)mc.wx0;
            u.r.wy0 = (W)mc.wy0;
        }
        u.r.wx1 = (W)mc.wx1;
        u.r.wy1 = (W)mc.wy1;
        u.r.lnu = mc.lnu;
        const uint32_t fl = 1u | (mc.immobile ? 2u : 0u);
        if constexpr (CONST) {
            // the compact record of a constant-property call (the type's values
            // are those the model gave: the same operations on the same inputs)
            u.r.tk = (W)mc.mtk;
            u.r.tf = fl | ((uint32_t)r.type << 8);
        } else {
            u.r.pv[0] = (W)mc.mro;
            u.r.pv[1] = (W)mc.mbb;
            u.r.pv[2] = (W)mc.mcp;
            u.r.pv[3] = (W)mc.mkt;
            u.r.pv[4] = (W)mc.mht;
            u.r.pv[5] = (W)mc.mtk;
            u.r.flag = fl;
        }
    }
    uint4 *d = P + (int64_t)__ldg(rank + i) * PayVec<MIXED, CONST>::R4;
#pragma unroll
    for (int q = 0; q < PayVec<MIXED, CONST>::R4; q++) d[q] = u.v[q];
}

template <bool MIXED>
__global__ void __launch_bounds__(256, 3) k_contrib_inplace(const __grid_constant__ GridView G,
                                                            const __grid_constant__ MarkerView A,
                                                            const int32_t *__restrict__ rank,
                                                            const int32_t *__restrict__ key,
                                                            const DevTypes *__restrict__ Ty,
                                                            const __grid_constant__ AvgArgsK args,
                                                            const double *__restrict__ T0p, void *payload)
{
    uint4 *P = reinterpret_cast<uint4 *>(payload);
    const double T0 = *T0p;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += stride)
        contrib_inplace<MIXED>(G, A, rank, key, Ty->t, args, T0, P, i);
}

// The in-place contributions of such a call (k_contrib_inplace's results): a
// small kernel for the constant-property path; a marker without its own
// viscosity (eta <= 0: viscalc) is appended to `deferred` for k_contrib_deferred.
// Records are the compact PayConst; block 0 also stores the type table for
// k_cellsums.
template <bool MIXED>
__global__ void __launch_bounds__(256) k_contrib_const(const __grid_constant__ GridView G,
                                                       const __grid_constant__ MarkerView A,
                                                       const int32_t *__restrict__ rank,
                                                       const int32_t *__restrict__ key, const DevTypes *__restrict__ Ty,
                                                       const __grid_constant__ AvgArgsK args, void *payload,
                                                       int32_t *__restrict__ deferred, int32_t *__restrict__ ndeferred,
                                                       TypeConst *__restrict__ tab)
{
    using W = typename AvgCfg<MIXED>::W;
    using PV = PayVec<MIXED, true>;
    __shared__ TypeConst S;
    const i2g_types &T = Ty->t;
    for (int t = threadIdx.x; t < kAvgTypes; t += blockDim.x) {
        const double ro = T.markro[t];
        double kt = T.markkt[t];
        if (kt <= 0.0010) kt = 0.0010;
        if (kt >= args.k_cutoff) kt = args.k_cutoff;
        S.ro[t] = ro;
        S.cp[t] = T.markcp[t];
        S.kt[t] = kt;
        S.ht[t] = radcoef(args, t) * ro;
        S.im[t] = T.markim[t] != 0;
    }
    __syncthreads();
    if (blockIdx.x == 0) {  // the table k_cellsums reads
        for (int t = threadIdx.x; t < kAvgTypes; t += blockDim.x) {
            tab->ro[t] = S.ro[t];
            tab->cp[t] = S.cp[t];
            tab->kt[t] = S.kt[t];
            tab->ht[t] = S.ht[t];
            tab->im[t] = S.im[t];
        }
    }
    uint4 *P = reinterpret_cast<uint4 *>(payload);
    const bool has_tmax = A.tmax != nullptr && args.track_tmax;
    const int32_t nc2 = (int32_t)(G.ny - 1);
    // one marker from its loaded fields
    auto one = [&](int64_t i, double x, double y, double Tin, double eta, int mt, int32_t id, int32_t k,
                   int32_t slot) {
        PV u;
#pragma unroll
        for (int q = 0; q < PV::R4; q++) u.v[q] = make_uint4(0u, 0u, 0u, 0u);
        const bool ok = (args.gridmod <= 1 || (id % args.gridmod) == 0) && mt >= 0 && x > 0 && y > 0 &&
                        x < G.xsize && y < G.ysize && Tin > 0 && mt < kAvgTypes;
        if (ok && !(eta > 0)) {  // viscosity from the rheology: the general path
            deferred[atomicAdd(ndeferred, 1)] = (int32_t)i;
            return;
        }
        if (ok) {
            double Tm = Tin;
            if (mt < 2) Tm = args.tmp_ambient;  // sticky air (markmart.c:296-309)
            if (Tm != Tin) A.T[i] = Tm;
            double mnu = eta;
            if (outside_radmax(G, args, x, y)) mnu = 1.000e+22;
            if (has_tmax && mt != 0) {
                const double tm = A.tmax[i];
                if (tm < Tm) A.tmax[i] = Tm;
            }
            const int32_t m10 = k / nc2, m20 = k - m10 * nc2;
            if constexpr (!MIXED) {
                double a0, a1, b0, b1;
                fdw64(__ldg(G.gx + m10), __ldg(G.gx + m10 + 1), x, a0, a1);
                fdw64(__ldg(G.gy + m20), __ldg(G.gy + m20 + 1), y, b0, b1);
                u.r.wx0 = a0;
                u.r.wx1 = a1;
                u.r.wy0 = b0;
                u.r.wy1 = b1;
            } else {
                float a0, a1, b0, b1;
                fdw32(__ldg(G.gx + m10), __ldg(G.ixb + m10), x, a0, a1);
                fdw32(__ldg(G.gy + m20), __ldg(G.iyb + m20), y, b0, b1);
                u.r.wx1 = a1;
                u.r.wy1 = b1;
            }
            u.r.tk = (W)Tm;
            u.r.lnu = args.viscmod == 1 ? (MIXED ? log_mixed(mnu) : log(mnu)) : (args.viscmod == 2 ? 1.0 / mnu : mnu);
            u.r.tf = 1u | (S.im[mt] ? 2u : 0u) | ((uint32_t)mt << 8);
        }
        uint4 *d = P + (int64_t)slot * PV::R4;
#pragma unroll
        for (int q = 0; q < PV::R4; q++) d[q] = u.v[q];
    };
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += (int64_t)gridDim.x * blockDim.x)
        one(i, A.x[i], A.y[i], A.T[i], A.eta[i], A.type[i], args.gridmod > 1 ? A.id[i] : 0, __ldg(key + i),
            __ldg(rank + i));
}

// the markers k_contrib_const deferred, through the general property model
template <bool MIXED>
__global__ void __launch_bounds__(256, 3) k_contrib_deferred(const __grid_constant__ GridView G,
                                                             const __grid_constant__ MarkerView A,
                                                             const int32_t *__restrict__ rank,
                                                             const int32_t *__restrict__ key,
                                                             const DevTypes *__restrict__ Ty,
                                                             const __grid_constant__ AvgArgsK args,
                                                             const double *__restrict__ T0p, void *payload,
                                                             const int32_t *__restrict__ deferred,
                                                             const int32_t *__restrict__ ndeferred)
{
    uint4 *P = reinterpret_cast<uint4 *>(payload);
    const double T0 = *T0p;
    const int64_t m = *ndeferred;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < m; q += stride)
        contrib_inplace<MIXED, true>(G, A, rank, key, Ty->t, args, T0, P, deferred[q]);
}

template <bool MIXED>
__global__ void __launch_bounds__(256, 4) k_contrib(const __grid_constant__ GridView G,
                                                    const __grid_constant__ MarkerView A,
                                                    const __grid_constant__ MarkerView B,
                                                    const int32_t *__restrict__ perm, const DevTypes *__restrict__ Ty,
                                                    const __grid_constant__ AvgArgsK args,
                                                    const double *__restrict__ T0p, void *payload, int64_t *slot0)
{
    uint4 *P = reinterpret_cast<uint4 *>(payload);
    const double T0 = *T0p;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < A.n; j += stride)
        contrib_marker<MIXED>(G, A, B, perm, Ty->t, args, T0, P, j, slot0);
}

// k_cellsums: one warp per column strip of 32 cells (lane = cell row); each lane
// keeps all kPart corner sums of its cell in FP64 registers.  The warp streams its
// strip's records in chunks of PC positions through two shared buffers of its
// own: while the lanes add chunk k (every lane its cell's markers, in position
// order), the asynchronous copies of chunk k+1 are in flight.  Record (row, t)
// sits at uint4 row * RS + t * R4; the PC records of a cell are contiguous in the
// payload, so each chunk is read with coalesced 16-byte copies, and RS (uint4 per
// row) is odd, so the lanes' 16-byte reads by cell row are conflict-free.  No
// block-wide barriers.  CONST: the compact records of a constant-property call
// (PayConst) with the per-type values from a shared table.
template <bool MIXED, bool CONST = false>
struct StripCfg {
    static constexpr int R4 = PayVec<MIXED, CONST>::R4;
    static constexpr int PR = 12;             // uint4 per row per chunk
    static constexpr int PC = PR / R4;        // positions per chunk
    static constexpr int RS = PR + 1;         // row stride (odd)
    static_assert(PC * R4 == PR, "a chunk row holds whole records");
};

template <bool MIXED, bool CONST = false>
struct StripBuf {
    uint4 rec[2][32 * StripCfg<MIXED, CONST>::RS];  // double buffer
    int32_t cb[32], cn[32];  // first slot and marker count of each cell of the strip
};

// dynamic shared memory of k_cellsums: one strip buffer per warp (and the type
// table of a constant-property call)
template <bool MIXED, bool CONST = false>
struct AvgSmem {
    StripBuf<MIXED, CONST> w[8];
};
template <bool MIXED>
struct AvgSmem<MIXED, true> {
    StripBuf<MIXED, true> w[8];
    TypeTabD tab;
};

// 16-byte asynchronous global -> shared copy; zero-fills (reads nothing) when !valid
__device__ __forceinline__ void cp_async16(uint4 *smem, const uint4 *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// the kPart corner sums of one marker into a cell's accumulators (field-major
// index q * 10 + F_*, then 40, 41 for the cell-centre nd), markmart.c:859-913,
// from its flag, FP64 weights and values (the mixed form's FP32 values widened
// exactly), every product and sum in FP64.  ET: whether beta is summed (a
// constant-property call has beta = 0 and skips it: adding +0 changes nothing).
template <bool ET>
__device__ __forceinline__ void add_values(double (&a)[kPart], uint32_t fl, double wx0, double wx1, double wy0,
                                           double wy1, double p0, double p1, double p2, double p3, double p4,
                                           double p5, double lnu)
{
    // the four corner weights, then one field at a time (each accumulator still
    // receives one term per marker), which keeps few widened values live
    double sw[4];
#pragma unroll
    for (int q = 0; q < 4; q++) sw[q] = 1.0 * ((q >> 1) ? wx1 : wx0) * ((q & 1) ? wy1 : wy0);
    const double pv[5] = {p0, p1, p2, p3, p4};
    const int fld[5] = {F_RO, F_ET, F_CP, F_KT, F_HT};
#pragma unroll
    for (int f = 0; f < 5; f++) {
        if (!ET && f == 1) continue;
#pragma unroll
        for (int q = 0; q < 4; q++) a[q * 10 + fld[f]] += pv[f] * sw[q];
    }
#pragma unroll
    for (int q = 0; q < 4; q++) a[q * 10 + F_W0] += sw[q];
    if (!(fl & 2)) {  // mobile type
#pragma unroll
        for (int q = 0; q < 4; q++) {
            a[q * 10 + F_TK] += p5 * sw[q];
            a[q * 10 + F_W1] += sw[q];
        }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double wx = (q >> 1) ? wx1 : wx0;
        const double wy = (q & 1) ? wy1 : wy0;
        if (wx > 0.5 && wy > 0.5) {
            const double swt2 = 1.0 * 4.0 * (wx - 0.5) * (wy - 0.5);
            a[q * 10 + F_NU] += lnu * swt2;
            a[q * 10 + F_WNU] += swt2;
        }
    }
    const double ddx = 1.0 - fabs(wx0 - 0.5);
    const double ddy = 1.0 - fabs(wy0 - 0.5);
    if (ddx > 0.5 && ddy > 0.5) {
        const double swt2 = 1.0 * 4.0 * (ddx - 0.5) * (ddy - 0.5);
        a[40] += lnu * swt2;
        a[41] += swt2;
    }
}

// the mixed form's w0 is 1.0f - w1 exactly (fdw32)
template <bool MIXED>
__device__ __forceinline__ void add_marker(double (&a)[kPart], const PayRec<MIXED> &R)
{
    const uint32_t fl = R.flag;
    if (!(fl & 1)) return;
    double wx0, wy0;
    if constexpr (MIXED) {
        wx0 = (double)(1.0f - R.wx1);
        wy0 = (double)(1.0f - R.wy1);
    } else {
        wx0 = R.wx0;
        wy0 = R.wy0;
    }
    add_values<true>(a, fl, wx0, R.wx1, wy0, R.wy1, R.pv[0], R.pv[1], R.pv[2], R.pv[3], R.pv[4], R.pv[5], R.lnu);
}

template <bool MIXED>
__device__ __forceinline__ void add_marker(double (&a)[kPart], const PayConst<MIXED> &R, const TypeTabD &S)
{
    const uint32_t fl = R.tf & 0xffu;
    if (!(fl & 1)) return;
    const int t = (int)(R.tf >> 8);
    double wx0, wy0;
    if constexpr (MIXED) {
        wx0 = (double)(1.0f - R.wx1);
        wy0 = (double)(1.0f - R.wy1);
    } else {
        wx0 = R.wx0;
        wy0 = R.wy0;
    }
    add_values<false>(a, fl, wx0, R.wx1, wy0, R.wy1, S.ro[t], 0.0, S.cp[t], S.kt[t], S.ht[t], R.tk, R.lnu);
}

// the asynchronous copies of positions [P0, P0+PC) of a strip into buffer dst
template <bool MIXED, bool CONST>
__device__ __forceinline__ void stage_chunk(const StripBuf<MIXED, CONST> &B, uint4 *dst, const uint4 *__restrict__ P,
                                            int P0, int lane)
{
    constexpr int R4 = StripCfg<MIXED, CONST>::R4, PR = StripCfg<MIXED, CONST>::PR, RS = StripCfg<MIXED, CONST>::RS;
#pragma unroll 2
    for (int it = 0; it < PR; it++) {
        const int e = it * 32 + lane, row = e / PR, piece = e - row * PR;
        const bool valid = P0 + piece / R4 < B.cn[row];
        const uint4 *src = valid ? P + (int64_t)(B.cb[row] + P0) * R4 + piece : P;
        cp_async16(dst + row * RS + piece, src, valid);
    }
    cp_async_commit();
}

// One tile of cells (cell columns [c0, c0+TX) x rows [d0, d0+32)) by the CTA's
// warps, a column strip each at a time.  The grid has nc1 x nc2 cells; the tile
// is column block (tile % ntx), row block (tile / ntx).  Returns the number of
// averaged markers this thread counted.
template <bool MIXED, bool CONST = false>
__device__ __forceinline__ unsigned cellsums_tile(AvgSmem<MIXED, CONST> &S, const uint4 *__restrict__ P,
                                                  const int32_t *__restrict__ cstart, int64_t nc1, int64_t nc2,
                                                  double *__restrict__ part, int64_t tile, int32_t TX, int32_t ntx)
{
    using PV = PayVec<MIXED, CONST>;
    constexpr int R4 = StripCfg<MIXED, CONST>::R4, PC = StripCfg<MIXED, CONST>::PC, RS = StripCfg<MIXED, CONST>::RS;
    const int64_t ncells = nc1 * nc2;
    const int64_t c0 = (tile % ntx) * TX, c1 = min(c0 + (int64_t)TX, nc1);
    const int64_t d0 = (tile / ntx) * 32;
    const int NR = (int)min((int64_t)32, nc2 - d0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    StripBuf<MIXED, CONST> &B = S.w[warp];
    unsigned cnt = 0;
    for (int64_t c = c0 + warp; c < c1; c += nwarps) {
        const int64_t cell = c * nc2 + d0 + lane;
        int32_t cb = 0, cn = 0;
        if (lane < NR) {
            cb = __ldg(cstart + cell);
            cn = __ldg(cstart + cell + 1) - cb;
        }
        int maxc = cn;
        for (int o = 16; o > 0; o >>= 1) maxc = max(maxc, __shfl_xor_sync(0xffffffffu, maxc, o));
        __syncwarp();  // the previous strip is done with B
        B.cb[lane] = cb;
        B.cn[lane] = cn;
        __syncwarp();
        double a[kPart];
#pragma unroll
        for (int u = 0; u < kPart; u++) a[u] = 0.0;
        if (maxc > 0) stage_chunk<MIXED, CONST>(B, B.rec[0], P, 0, lane);
        for (int P0 = 0, k = 0; P0 < maxc; P0 += PC, k ^= 1) {
            // chunk P0 is in buffer k; start the next one into the other buffer
            if (P0 + PC < maxc) {
                stage_chunk<MIXED, CONST>(B, B.rec[k ^ 1], P, P0 + PC, lane);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncwarp();  // every lane's copies of chunk P0 are visible
            const uint4 *buf = B.rec[k] + lane * RS;
            const int m = min(PC, cn - P0);
            for (int t = 0; t < m; t++) {
                PV u;
#pragma unroll
                for (int q = 0; q < R4; q++) u.v[q] = buf[t * R4 + q];
                if constexpr (CONST) {
                    cnt += u.r.tf & 1u;
                    add_marker<MIXED>(a, u.r, S.tab);
                } else {
                    cnt += u.r.flag & 1u;
                    add_marker<MIXED>(a, u.r);
                }
            }
            __syncwarp();  // buffer k is free for chunk P0 + 2 PC
        }
        if (lane < NR) {
            double *d = part + cell;
#pragma unroll
            for (int u = 0; u < kPart; u++) d[u * ncells] = a[u];
        }
    }
    return cnt;
}

// per-warp sum of the counts into *navg
__device__ __forceinline__ void add_count(unsigned cnt, unsigned long long *navg)
{
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && navg && cnt) atomicAdd(navg, (unsigned long long)cnt);
}

// tab: the type table of a constant-property call (CONST)
template <bool MIXED, bool CONST = false>
__global__ void __launch_bounds__(256, 2) k_cellsums(const void *payload, const int32_t *__restrict__ cstart,
                                                     int64_t nc1, int64_t nc2, double *__restrict__ part, int32_t TX,
                                                     int32_t ntx, unsigned long long *navg,
                                                     const TypeConst *__restrict__ tab)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    AvgSmem<MIXED, CONST> &S = *reinterpret_cast<AvgSmem<MIXED, CONST> *>(smraw);
    if constexpr (CONST) {
        using W = typename AvgCfg<MIXED>::W;
        for (int t = threadIdx.x; t < kAvgTypes; t += blockDim.x) {
            S.tab.ro[t] = (double)(W)tab->ro[t];
            S.tab.cp[t] = (double)(W)tab->cp[t];
            S.tab.kt[t] = (double)(W)tab->kt[t];
            S.tab.ht[t] = (double)(W)tab->ht[t];
        }
        __syncthreads();
    }
    add_count(cellsums_tile<MIXED, CONST>(S, reinterpret_cast<const uint4 *>(payload), cstart, nc1, nc2, part,
                                          blockIdx.x, TX, ntx),
              navg);
}

}  // namespace i2g
