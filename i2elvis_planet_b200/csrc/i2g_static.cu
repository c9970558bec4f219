// i2g_ronurecalc_static: marker -> node averaging (ronurecalc) that allocates
// nothing, for callers that cannot allocate device memory when they average.
//
// Who those callers are: host codes that keep the markers and nodes in device
// arrays of their own and average inside a region where cudaMalloc is off
// limits -- device memory owned by a pool allocator that must not be bypassed or
// fragmented, a host that has reserved the device's memory for itself, or a
// time loop that must not stall on the implicit device synchronisation that
// cudaMalloc/cudaFree can bring.  The context API (i2g_create) allocates its
// buffers once per instance; this entry point needs no context at all.
//
// All scratch (cell keys, counts and offsets, the sort permutations, the sorted
// marker copy, the per-marker averaging payload, the cell corner sums,
// per-block viscosity ranges, the rock table and the grid lookup tables) is
// carved out of one file-scope device array, g_scratch, of kScratchBytes
// (about 16.7 MB).  Every GPU that loads libi2g.so
// holds that array until the process exits.  Its size sets the limits: at most
// kMaxMarkers markers and kMaxLines grid lines in each direction; larger
// problems get I2G_ECAPACITY.
//
// In host code, g_scratch names a host-side stand-in, not the device array, so
// the host never passes it to a kernel.  The first call on each device, with
// that device current, asks the runtime for the array's device address
// (cudaGetSymbolAddress), checks the result and caches it; make that first call
// before any stream capture.  Every call shares the one array and finds the
// previous call's contents in it: each call zeroes what must start at zero (cell
// counts, cursors, the averaged-marker counter) and seeds the rest itself.
// Calls that overlap on one GPU (two streams, two host threads) race on the
// array: serialise them.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>

#include "../../include/i2g.h"
#include "i2g_launch.h"

using namespace i2g;

namespace {

constexpr int64_t kMaxMarkers = 65536;
constexpr int64_t kMaxLines = 129;  // grid lines per direction
constexpr int64_t kMaxNodes = kMaxLines * kMaxLines;
constexpr int64_t kMaxCells = (kMaxLines - 1) * (kMaxLines - 1);
constexpr int64_t kMaxNodeBlocks = (kMaxNodes + 255) / 256;
constexpr int kPartFields = 42;  // cell corner sums per cell (k_cellsums)

constexpr int64_t al(int64_t b) { return (b + 255) & ~(int64_t)255; }

// byte offsets of the pieces of g_scratch
constexpr int64_t oTypes = 0;
constexpr int64_t oXmid = oTypes + al(sizeof(DevTypes));
constexpr int64_t oYmid = oXmid + al(kMaxLines * 8);
constexpr int64_t oInv = oYmid + al(kMaxLines * 8);  // ixb, iyb, ixm, iym
constexpr int64_t oLx = oInv + 4 * al(kMaxLines * 4);
constexpr int64_t oLy = oLx + al(kMaxLines * 16);
constexpr int64_t oPrf = oLy + al(kMaxLines * 16);
constexpr int64_t oGaf = oPrf + al(kMaxNodes * 4);
constexpr int64_t oKey = oGaf + al(kMaxNodes * 4);
constexpr int64_t oPerm1 = oKey + al(kMaxMarkers * 4);
constexpr int64_t oPerm2 = oPerm1 + al(kMaxMarkers * 4);
constexpr int64_t oCount = oPerm2 + al(kMaxMarkers * 4);
constexpr int64_t oCursor = oCount + al(kMaxCells * 4);
constexpr int64_t oCstart = oCursor + al(kMaxCells * 4);
constexpr int64_t oTile = oCstart + al((kMaxCells + 1) * 4);
constexpr int64_t oSrcId = oTile + al(4096 * 4);          // caller index of each caller marker
constexpr int64_t oSrcP = oSrcId + al(kMaxMarkers * 4);   // stand-in pressure column, never written
constexpr int64_t oDst = oSrcP + al(kMaxMarkers * 8);     // sorted copy: x y T eta p (f64), type, id
constexpr int64_t oPart = oDst + 5 * al(kMaxMarkers * 8) + al(kMaxMarkers) + al(kMaxMarkers * 4);
constexpr int64_t oMm = oPart + al((int64_t)kPartFields * kMaxCells * 8);
constexpr int64_t oPay = oMm + al(3 * kMaxNodeBlocks * 8);  // averaging payload, FP64 size (the larger)
constexpr int64_t oSmall = oPay + al(payload_bytes(false, kMaxMarkers));  // stats[2], T0, navg, slot0
constexpr int64_t kScratchBytes = oSmall + 256;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
// device address of g_scratch per device, looked up once per device: host
// threads making their first call on a device at the same time wait for one
// lookup (std::call_once), and every reader sees the stored address (atomic).
// The address belongs to the device's context as the process first had it: a
// cudaDeviceReset ends that context, and with it every address this cache holds.
std::atomic<void *> g_base[kMaxDevices];
std::once_flag g_once[kMaxDevices];

// xmid, 1/width, 1/mid spacing and the float4 line table {width, 1/width,
// 1/mid spacing} of one axis from its grid lines: the tables i2g_set_grid
// builds on the host, with the same double arithmetic
__global__ void k_line_tables(const double *__restrict__ g, int64_t n, double *__restrict__ mid,
                              float *__restrict__ ib, float *__restrict__ im, float4 *__restrict__ L)
{
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        double m = 0.0, wb = 0.0, imd = 0.0;
        if (i + 1 < n) {
            m = (g[i] + g[i + 1]) / 2.0;
            wb = g[i + 1] - g[i];
        }
        if (i + 2 < n) imd = 1.0 / ((g[i + 1] + g[i + 2]) / 2.0 - m);
        const float ibf = (i + 1 < n) ? (float)(1.0 / wb) : 0.f;
        mid[i] = m;
        ib[i] = ibf;
        im[i] = (float)imd;
        L[i] = make_float4((float)wb, ibf, (float)imd, 0.f);
    }
}

// float copy of a node field (zeros when the field is absent)
__global__ void k_field_f32(int64_t n, const double *__restrict__ a, float *__restrict__ out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a ? (float)a[i] : 0.0f;
}

__global__ void k_caller_ids(int64_t n, int32_t *__restrict__ id)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
        id[j] = (int32_t)j;
}

// the sticky-air temperature reset, made on the sorted copy, back into the
// caller's T (markmart.c:296-309 writes markk[] in place)
__global__ void k_T_to_caller(int64_t n, const int32_t *__restrict__ id, const double *__restrict__ Ts,
                              double *__restrict__ T)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
        T[id[j]] = Ts[j];
}

unsigned blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 4)); }

// radiogenic heating per kg by rock-type group at timesum (markmart.c:749-837),
// on the host with the operation order of the reference, as the context API does
void radiogenic_rates(double timesum, double al26, double fe60, double &rsi, double &rfe, double &rch)
{
    const double tA = timesum / (365.250 * 24.000 * 3600.000);
    const double init_al = 1.89716e+23 * al26 * 4.999e-13 / (3.264e+13);
    const double init_fe = 1.971e+24 * fe60 * 4.3451e-13 / (1.183e+14);
    const double a = init_al * exp(-tA * 9.6673e-7);
    const double u = 2.990e-12 * exp(-tA * 9.8458e-10);
    const double uu = 1.600e-12 * exp(-tA * 1.5541e-10);
    const double th = 1.000e-12 * exp(-tA * 4.9511e-11);
    const double f = init_fe * exp(-tA * 2.6660e-7);
    rsi = a + (0.40689 * 1.430e-11) * exp(-tA * 4.9867e-10) + u + uu + th;
    rfe = f + (0.090625 * 1.430e-11) * exp(-tA * 4.9867e-10);
    rch = a + f + 1.430e-11 * exp(-tA * 4.9867e-10) + u + uu + th;
}

// the device address of g_scratch on the current device (first call per device: look it up)
int scratch_base(unsigned char **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return I2G_ECUDA;
    try {
        // a failed lookup throws, so that call_once lets the next call try again
        std::call_once(g_once[dev], [dev] {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                throw 1;
            }
            g_base[dev].store(p, std::memory_order_release);
        });
    } catch (int) {
        return I2G_ECUDA;
    }
    void *p = g_base[dev].load(std::memory_order_acquire);
    if (!p) return I2G_ECUDA;
    *out = (unsigned char *)p;
    return I2G_OK;
}

}  // namespace

extern "C" int64_t i2g_static_max_markers(void) { return kMaxMarkers; }
extern "C" int64_t i2g_static_max_lines(void) { return kMaxLines; }

extern "C" int i2g_ronurecalc_static(const i2g_params *P, const i2g_types *types, const double *gx,
                                     const double *gy, const double *pr, const double *exx, const double *eyy,
                                     const double *exy, const double *sxx, const double *syy, const double *sxy,
                                     const double *ga, const double *mu, int64_t n, const double *x, const double *y,
                                     double *T, const double *eta, const int8_t *type, double timesum, double *ro,
                                     double *nu, double *nd, double *et, double *cp, double *kt, double *ht,
                                     double *tk, double *po, void *stream)
{
    if (!P || !types || !gx || !gy || !pr || n < 0 || (n > 0 && (!x || !y || !T || !eta || !type))) return I2G_EINVAL;
    if (!ro || !nu || !nd || !et || !cp || !kt || !ht || !tk || !po) return I2G_EINVAL;
    if (P->abi_version != I2G_ABI_VERSION || P->xnumx < 3 || P->ynumy < 3 || !(P->xsize > 0) || !(P->ysize > 0))
        return I2G_EINVAL;
    if (P->precision != I2G_PREC_FP64 && P->precision != I2G_PREC_MIXED) return I2G_EINVAL;
    if (P->gridmod <= 0 || !(P->nubeg > 0)) return I2G_EINVAL;
    if (P->intermod != 0 || P->intermod1 != 0 || (P->densimod != 0 && P->densimod != 1) || P->viscmod < 0 ||
        P->viscmod > 2)
        return I2G_EUNSUPPORTED;
    // problems larger than the static scratch
    if (n > kMaxMarkers || P->xnumx > kMaxLines || P->ynumy > kMaxLines) return I2G_ECAPACITY;
    unsigned char *base = nullptr;
    if (int r = scratch_base(&base)) return r;
    cudaStream_t s = (cudaStream_t)stream;
    const bool mixed = P->precision == I2G_PREC_MIXED;
    const int64_t nx = P->xnumx, ny = P->ynumy, nn = nx * ny, ncells = (nx - 1) * (ny - 1);

    DevTypes *dtypes = (DevTypes *)(base + oTypes);
    double *xmid = (double *)(base + oXmid), *ymid = (double *)(base + oYmid);
    const int64_t invs = al(kMaxLines * 4) / 4;
    float *ixb = (float *)(base + oInv), *iyb = ixb + invs, *ixm = ixb + 2 * invs, *iym = ixb + 3 * invs;
    float4 *lx = (float4 *)(base + oLx), *ly = (float4 *)(base + oLy);
    float *prf = (float *)(base + oPrf), *gaf = (float *)(base + oGaf);
    GridView G{};
    G.nx = nx;
    G.ny = ny;
    G.xsize = P->xsize;
    G.ysize = P->ysize;
    // first guess of the cell search only (the search itself is exact)
    G.inv_x = (double)(nx - 1) / P->xsize;
    G.inv_y = (double)(ny - 1) / P->ysize;
    G.gx = gx;
    G.gy = gy;
    G.xmid = xmid;
    G.ymid = ymid;
    G.pr = pr;
    G.ga = ga;
    G.exx = exx;
    G.eyy = eyy;
    G.exy = exy;
    G.sxx = sxx;
    G.syy = syy;
    G.sxy = sxy;
    G.mu = mu;
    G.prf = mixed ? prf : nullptr;
    G.gaf = mixed ? gaf : nullptr;
    G.ixb = ixb;
    G.iyb = iyb;
    G.ixm = ixm;
    G.iym = iym;
    G.lx = lx;
    G.ly = ly;

    SortBufs sb{};
    sb.key = (int32_t *)(base + oKey);
    sb.perm1 = (int32_t *)(base + oPerm1);
    sb.perm2 = (int32_t *)(base + oPerm2);
    sb.count = (int32_t *)(base + oCount);
    sb.cursor = (int32_t *)(base + oCursor);
    sb.cstart = (int32_t *)(base + oCstart);
    sb.tilesum = (int32_t *)(base + oTile);
    double *small = (double *)(base + oSmall);
    double *stats = small, *T0 = small + 2;
    unsigned long long *navg = (unsigned long long *)(small + 3);
    sb.slot0 = (int64_t *)(small + 4);

    // source: the caller's markers in the caller's order
    MarkerView A{};
    A.n = n;
    A.x = (double *)x;
    A.y = (double *)y;
    A.T = T;
    A.eta = (double *)eta;
    A.p = (double *)(base + oSrcP);
    A.type = (int8_t *)type;
    A.id = (int32_t *)(base + oSrcId);
    // destination of the sort application inside the averaging kernel
    MarkerView B{};
    B.n = n;
    B.x = (double *)(base + oDst);
    B.y = (double *)(base + oDst + al(kMaxMarkers * 8));
    B.T = (double *)(base + oDst + 2 * al(kMaxMarkers * 8));
    B.eta = (double *)(base + oDst + 3 * al(kMaxMarkers * 8));
    B.p = (double *)(base + oDst + 4 * al(kMaxMarkers * 8));
    B.type = (int8_t *)(base + oDst + 5 * al(kMaxMarkers * 8));
    B.id = (int32_t *)(base + oDst + 5 * al(kMaxMarkers * 8) + al(kMaxMarkers));

    // seed the scratch: rock table, line tables, float fields, caller ids; caller
    // marker 0 sits at slot 0 of the source; the averaged-marker counter starts at 0
    if (cudaMemcpyAsync(&dtypes->t, types, sizeof(i2g_types), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return I2G_ECUDA;
    k_line_tables<<<1, 128, 0, s>>>(gx, nx, xmid, ixb, ixm, lx);
    k_line_tables<<<1, 128, 0, s>>>(gy, ny, ymid, iyb, iym, ly);
    if (mixed) {
        k_field_f32<<<blocks(nn), 256, 0, s>>>(nn, pr, prf);
        k_field_f32<<<blocks(nn), 256, 0, s>>>(nn, ga, gaf);
    }
    if (n > 0) k_caller_ids<<<blocks(n), 256, 0, s>>>(n, A.id);
    if (cudaMemsetAsync(sb.slot0, 0, sizeof(int64_t), s) != cudaSuccess) return I2G_ECUDA;
    if (cudaMemsetAsync(navg, 0, sizeof(unsigned long long), s) != cudaSuccess) return I2G_ECUDA;

    // counting sort of the caller's markers into (cell, caller index) order;
    // rank_markers zeroes the counts and cursors it accumulates into
    launch_keys(s, G, x, y, n, sb.key);
    rank_markers(s, sb, n, ncells, A.id, false);

    AvgArgsK args{};
    args.timesum = timesum;
    args.tmp_ambient = P->tmp_ambient;
    args.core_form_time = P->core_form_time;
    args.k_cutoff = P->k_cutoff;
    args.relax_time = P->relax_time;
    args.nubeg = P->nubeg;
    args.nuend = P->nuend;
    args.xmelt_si = P->xmelt_si;
    args.xmelt_fe = P->xmelt_fe;
    args.gridmod = P->gridmod;
    args.densimod = P->densimod;
    args.viscmod = P->viscmod;
    args.track_tmax = 0;
    radiogenic_rates(timesum, P->al2627_init, P->fe6056_init, args.rad_si, args.rad_fe, args.rad_ch);

    StepLaunch L{s, G, A, dtypes};
    AvgLaunch V{};
    V.dst = B;
    V.perm = sb.perm2;
    V.cstart = sb.cstart;
    V.T0 = T0;
    V.payload = base + oPay;
    V.part = (double *)(base + oPart);
    V.TX = 16;
    V.navg = navg;
    V.slot0 = sb.slot0;
    launch_t0(s, G, A, sb.slot0, P->tmp_ambient, T0);
    if (mixed) launch_avg_mixed(L, args, V);
    else launch_avg_fp64(L, args, V);
    NodeOut O{ro, nu, nd, et, cp, kt, ht, tk, po, nullptr};
    launch_nodes(s, G, V.part, args, O, P->nucontr, (double *)(base + oMm), stats);
    if (n > 0) k_T_to_caller<<<blocks(n), 256, 0, s>>>(n, B.id, B.T, T);
    return cudaGetLastError() == cudaSuccess ? I2G_OK : I2G_ECUDA;
}
