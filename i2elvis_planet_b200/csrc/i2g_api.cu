// C ABI of the marker step (include/i2g.h): contexts, host/device transfers and
// the movemark()/ronurecalc() entry points.
//
// Reference boundary replaced here: movemark() (markmart.c:3-188) and
// ronurecalc() (markmart.c:192-1009) over the globals of headmart.c.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/i2g.h"
#include "i2g_kernels.cuh"
#include "i2g_launch.h"
#include "i2g_adjoint.cuh"
#include "i2g_prn.cuh"

using namespace i2g;

namespace {

enum { G_VX = 0, G_VY, G_PR, G_EXX, G_EYY, G_EXY, G_SXX, G_SYY, G_SXY, G_GA, G_MU, G_N };
enum { N_RO = 0, N_NU, N_ND, N_ET, N_CP, N_KT, N_HT, N_TK, N_PO, N_N };

struct MarkerBuf {
    double *x = nullptr, *y = nullptr, *T = nullptr, *eta = nullptr, *p = nullptr;
    double *tmax = nullptr, *hi = nullptr, *por = nullptr;
    int8_t *type = nullptr;
    int32_t *id = nullptr;
    int8_t *mgo = nullptr;  // magnetisation state, time (i2g_set_marker_mag)
    double *mgt = nullptr;
};

}  // namespace

struct i2g_ctx {
    i2g_params P{};
    i2g_types Th{};
    int dev = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int64_t nx = 0, ny = 0, nn = 0, ncells = 0;
    double *gx = nullptr, *gy = nullptr, *xmid = nullptr, *ymid = nullptr;
    float *ixb = nullptr, *iyb = nullptr, *ixm = nullptr, *iym = nullptr;
    float4 *lx = nullptr, *ly = nullptr;
    double *g[G_N] = {};
    bool gpresent[G_N] = {};
    float *vxf = nullptr, *vyf = nullptr, *prf = nullptr, *gaf = nullptr;
    float4 *vxq = nullptr, *vyq = nullptr, *prq = nullptr;  // mixed form: stencil coefficients
    float4 *vq4 = nullptr;  // mixed form, uniform grid: per-quarter-cell forms of vx, vy (8 float4 per cell)
    float *ef[G_N] = {};  // mixed form: FP32 copies of the strain-rate and stress fields (G_EXX..G_SXY)
    double inv_x = 0, inv_y = 0;
    bool grid_set = false;
    double *node[N_N] = {};
    int64_t cap = 0, n = 0;
    MarkerBuf mb[2];
    int cur = 0;
    bool has_tmax = false, has_hi = false, has_por = false, has_mag = false;
    bool markers_set = false, keys_dirty = false;
    // storage order of the markers: canonical (cell, caller index) or left as the
    // last movemark found it; ranks_valid: sb.perm2/rank match storage and positions
    bool order_sorted = false, ranks_valid = false;
    int32_t reorder_every = 32, since_reorder = 0;  // averaging calls between record moves
    SortBufs sb{};
    double *part = nullptr, *mmpart = nullptr, *stats = nullptr, *T0 = nullptr;
    uint8_t *payload = nullptr;  // averaging payload, payload_bytes(precision, cap)
    double *tnode[3] = {};       // titerate marker update: node T after / before the solve, sol1
    float *tnodef = nullptr;     // mixed form: FP32 copies of tk_new, tk_old, kt, cp, ro
    double *idx2 = nullptr, *idy2 = nullptr;  // per grid line 1.0/d/d (the diffusion term)
    cudaStream_t copy_stream = nullptr;  // host transfers of set/get, overlapped with their kernels
    cudaEvent_t xev[4] = {};             // ordering events between stream and copy_stream
    int *typecheck = nullptr;       // device: {bad-type bits, first bad marker}
    int32_t *ndeferred = nullptr;   // device: markers deferred to the general property model
    uint8_t *tconst = nullptr;      // device: per-type table of a constant-property averaging call
    int *typecheck_host = nullptr;  // pinned mirror, read after the set call's final sync
    int32_t TX = 16;  // averaging tile: cell columns (x 32 cell rows)
    unsigned long long *navg = nullptr;
    DevTypes *dtypes = nullptr;
    int64_t nsorts = 0;
    int64_t launches = 0;
    int64_t nallocs = 0, fail_alloc_at = 0;  // test hook I2G_FAIL_ALLOC_AT (see env_long)
    // phase timing (i2g_profile_*)
    bool prof = false;
    struct Pending {
        int phase;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> evpool;
    double prof_ms[I2G_PHASES] = {};
    int64_t prof_calls[I2G_PHASES] = {};
    // adjoint state (i2g_adjoint_*)
    struct Adj {
        double *mvx = nullptr, *mvy = nullptr, *amps = nullptr;
        int32_t nm = 0;
        double2 *ck = nullptr;
        int64_t ck_segs = 0;
        int32_t nsteps = 0, every = 0;
        double dt = 0.0;
        double *T0 = nullptr, *w1 = nullptr, *g = nullptr, *dT = nullptr, *dapart = nullptr, *da = nullptr;
        int8_t *type_by_id = nullptr;
        double2 *lam = nullptr;
        int32_t nblk = 0;
        bool ready = false;
    } adj;
    // fused mixed step (k_move_fused + k_cellnodes, i2g_fused.cuh)
    struct Fused {
        bool enabled = true;         // i2g_set_fused
        int32_t cap = 0;             // places per cell bucket; 0 = buckets not allocated
        float4 *ra = nullptr;        // [ncells * cap] 16-byte records
        OvfRec *ovf = nullptr;       // [max_markers]
        FusedCounters *ctr = nullptr;
        int32_t *treset = nullptr;   // [max_markers]
        int2 *defer = nullptr;       // [max_markers]
        int32_t *guard = nullptr;    // [nodes]
        int32_t *cmax = nullptr;     // device scratch: largest cell count
        int32_t *count = nullptr;    // [ncells] records per cell
        bool resets_done = false;    // the sticky-air resets of the records are applied
        void *host = nullptr;        // pinned copy of the counters of the last fused movemark
        cudaEvent_t host_ev = nullptr;
        bool host_pending = false;
        bool ready = false;          // the buckets hold the records of the markers as they are
        double timesum = 0.0;        // the movemark's timesum
        int32_t nt = 0;              // type slots in use (averaged types present); 0 = none
        uint8_t tinfo[kAvgTypes] = {};
        uint8_t slot_type[kFusedSlots] = {};  // the rock type of each slot
        int64_t calls = 0, overflows = 0;
    } fz;
    // densimod 2 (i2g_set_td_table, i2g_td.cuh)
    struct Td {
        double2 *rh = nullptr;       // [2][tknum][pbnum] density, enthalpy in SI units
        int32_t *flag = nullptr;     // [max_markers] by caller index
        int32_t *prev = nullptr;     // [max_markers] by caller index
        double *si = nullptr;        // [max_markers] by caller index
        void *scan = nullptr;        // scratch of the max-scan
        size_t scan_bytes = 0;
        double *melt = nullptr;      // [12]: the eps[] state in use and the one the next call writes
        int cur = 0;                 // which half of melt is current
        TdArgs a{};                  // table geometry and switches
        int64_t rh_cap = 0;
        bool set = false;
    } td;
    // magnetisation (i2g_mag.cuh): the carried time's scan by caller index
    struct Mag {
        int32_t *flag = nullptr, *prev = nullptr;
        double *val = nullptr;
        void *scan = nullptr;
        size_t scan_bytes = 0;
        double *state = nullptr;  // [4]: the carried time in use and the one the next call writes
        int cur = 0;
    } mag;
    // output-file marker section (i2g_prn.cuh), allocated at the first use
    struct Prn {
        uint8_t *buf = nullptr;  // [39 cap] records
        int32_t *pos = nullptr;  // [cap] caller index -> slot
        float *f = nullptr;      // [9][cap] caller-order float fields
        int8_t *b = nullptr;     // [2][cap] type, magnetisation state
        double *mgt = nullptr;   // [cap] magnetisation time
    } prn;
    // a step captured into a batch's CUDA graph: per-step constants from the
    // batch's device table, no host decisions that the replays could not repeat
    const double *g_stepc = nullptr;
    const int32_t *g_stepi = nullptr;
    bool in_graph = false;
    double timestep = 0.0;                 // the global timestep the averaging reads (porosity sintering)
    unsigned int *sinter_stuck = nullptr;  // device: grain-size searches that gave up this call
    bool keys_stale = true;  // sb.key does not hold the device-order cells of the positions
    bool f32_storage = false;  // markers came in the reference's single-precision storage
    bool uni = false;        // uniform grid (GridView.uni)
    double ux0 = 0, uy0 = 0, uwx = 0, uwy = 0;
    std::vector<void *> allocs;
    std::string err;
};

namespace {

int fail(i2g_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(c, (e_ == cudaErrorMemoryAllocation) ? I2G_ENOMEM : I2G_ECUDA,           \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

#define CKL()                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = cudaGetLastError();                                                     \
        if (e_ != cudaSuccess) return fail(c, I2G_ECUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
    } while (0)

// Failure hooks for tests, host only: I2G_FAIL_ALLOC_AT=k makes the k-th device
// allocation of a context fail as an exhausted cudaMalloc would (I2G_ENOMEM);
// I2G_FAIL_CUDA=1 makes the entry points' first CUDA call report a failure
// (I2G_ECUDA).  Neither touches the device.
long env_long(const char *name)
{
    const char *v = getenv(name);
    return v ? atol(v) : 0;
}

bool alloc_injected(i2g_ctx *c) { return c->fail_alloc_at > 0 && ++c->nallocs == c->fail_alloc_at; }

template <class T>
int dalloc(i2g_ctx *c, T **p, int64_t count)
{
    *p = nullptr;
    if (count <= 0) count = 1;
    if (alloc_injected(c))
        return fail(c, I2G_ENOMEM, "cudaMalloc: injected failure (I2G_FAIL_ALLOC_AT)");
    cudaError_t e = cudaMalloc((void **)p, sizeof(T) * (size_t)count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(c, I2G_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    c->allocs.push_back((void *)*p);
    return I2G_OK;
}

#define TRY(x)                   \
    do {                         \
        int r_ = (x);            \
        if (r_ != I2G_OK) return r_; \
    } while (0)

cudaEvent_t event_get(i2g_ctx *c)
{
    cudaEvent_t e = nullptr;
    if (!c->evpool.empty()) {
        e = c->evpool.back();
        c->evpool.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        e = nullptr;
    }
    return e;
}

// events around one phase on the context's stream (only when profiling is on)
struct PhaseTimer {
    i2g_ctx *c;
    int phase;
    cudaEvent_t a = nullptr;
    PhaseTimer(i2g_ctx *c_, int ph) : c(c_), phase(ph)
    {
        if (c->prof && (a = event_get(c))) cudaEventRecord(a, c->stream);
    }
    ~PhaseTimer()
    {
        if (!a) return;
        cudaEvent_t b = event_get(c);
        if (!b) { c->evpool.push_back(a); return; }
        cudaEventRecord(b, c->stream);
        c->pending.push_back({phase, a, b});
    }
};

GridView grid_view(const i2g_ctx *c)
{
    GridView G{};
    G.nx = c->nx;
    G.ny = c->ny;
    G.xsize = c->P.xsize;
    G.ysize = c->P.ysize;
    G.inv_x = c->inv_x;
    G.inv_y = c->inv_y;
    G.gx = c->gx;
    G.gy = c->gy;
    G.xmid = c->xmid;
    G.ymid = c->ymid;
    G.vx = c->g[G_VX];
    G.vy = c->g[G_VY];
    G.pr = c->g[G_PR];
    G.ga = c->g[G_GA];
    G.exx = c->gpresent[G_EXX] ? c->g[G_EXX] : nullptr;
    G.eyy = c->gpresent[G_EYY] ? c->g[G_EYY] : nullptr;
    G.exy = c->gpresent[G_EXY] ? c->g[G_EXY] : nullptr;
    G.sxx = c->gpresent[G_SXX] ? c->g[G_SXX] : nullptr;
    G.syy = c->gpresent[G_SYY] ? c->g[G_SYY] : nullptr;
    G.sxy = c->gpresent[G_SXY] ? c->g[G_SXY] : nullptr;
    G.mu = c->gpresent[G_MU] ? c->g[G_MU] : nullptr;
    G.vxf = c->vxf;
    G.vyf = c->vyf;
    G.prf = c->prf;
    G.vxq = c->vxq;
    G.vyq = c->vyq;
    G.prq = c->prq;
    G.vq4 = c->uni ? c->vq4 : nullptr;
    G.gaf = c->gaf;
    G.exxf = c->gpresent[G_EXX] ? c->ef[G_EXX] : nullptr;
    G.eyyf = c->gpresent[G_EYY] ? c->ef[G_EYY] : nullptr;
    G.exyf = c->gpresent[G_EXY] ? c->ef[G_EXY] : nullptr;
    G.sxxf = c->gpresent[G_SXX] ? c->ef[G_SXX] : nullptr;
    G.syyf = c->gpresent[G_SYY] ? c->ef[G_SYY] : nullptr;
    G.sxyf = c->gpresent[G_SXY] ? c->ef[G_SXY] : nullptr;
    G.ixb = c->ixb;
    G.iyb = c->iyb;
    G.ixm = c->ixm;
    G.iym = c->iym;
    G.lx = c->lx;
    G.ly = c->ly;
    G.uni = c->uni ? 1 : 0;
    G.gx0 = c->ux0;
    G.gy0 = c->uy0;
    G.wx = c->uwx;
    G.wy = c->uwy;
    G.iwx = c->uwx > 0 ? 1.0 / c->uwx : 0.0;
    G.iwy = c->uwy > 0 ? 1.0 / c->uwy : 0.0;
    G.fwx = (float)G.wx;
    G.fwy = (float)G.wy;
    G.fiwx = (float)G.iwx;
    G.fiwy = (float)G.iwy;
    return G;
}

MarkerView marker_view(const i2g_ctx *c, int which, bool with_tmax = true)
{
    const MarkerBuf &b = c->mb[which];
    MarkerView M{};
    M.n = c->n;
    M.x = b.x;
    M.y = b.y;
    M.T = b.T;
    M.eta = b.eta;
    M.p = b.p;
    M.tmax = (c->has_tmax && with_tmax) ? b.tmax : nullptr;
    M.hi = c->has_hi ? b.hi : nullptr;
    M.por = c->has_por ? b.por : nullptr;
    M.type = b.type;
    M.id = b.id;
    M.mgo = c->has_mag ? b.mgo : nullptr;
    M.mgt = c->has_mag ? b.mgt : nullptr;
    return M;
}

// sort the current buffer into the other one (cell order, caller index inside a cell)
// sb.key from the current positions (device order), when k_move_fused left it stale
int refresh_keys(i2g_ctx *c)
{
    if (!c->keys_stale) return I2G_OK;
    const MarkerBuf &b = c->mb[c->cur];
    c->launches += launch_keys(c->stream, grid_view(c), b.x, b.y, c->n, c->sb.key);
    CKL();
    c->keys_stale = false;
    return I2G_OK;
}

// per rock type < 50: the fused path's slot of the type and its immobile bit
void fused_tinfo(i2g_ctx *c, uint64_t present)
{
    c->fz.nt = 0;
    for (int t = 0; t < kAvgTypes; t++) c->fz.tinfo[t] = 0;
    int nt = 0;
    for (int t = 0; t < kAvgTypes; t++) {
        if (!((present >> t) & 1ull)) continue;
        if (nt == kFusedSlots) { nt = -1; break; }
        c->fz.slot_type[nt] = (uint8_t)t;
        c->fz.tinfo[t] = (uint8_t)(nt | (c->Th.markim[t] ? 4 : 0));
        nt++;
    }
    c->fz.nt = nt > 0 ? nt : 0;
}

// Buckets for the fused path, sized from the largest cell count: the average
// room of a bucket is 1.5 x that count (at least 8 more places), an even number
// of 16-byte records.
int fused_buckets(i2g_ctx *c, int32_t count_max)
{
    int64_t cap = (int64_t)count_max + std::max<int64_t>(8, count_max / 2);
    cap = (cap + 1) & ~(int64_t)1;
    if (cap <= c->fz.cap) return I2G_OK;
    if (c->fz.ra) cudaFree(c->fz.ra);
    c->fz.ra = nullptr;
    c->fz.cap = 0;
    // too large for the fused path: the places must fit an int32, and the cell
    // sums are exact only for fewer than 2^19 records in a cell (k_cellnodes)
    if (c->ncells * cap >= (int64_t)INT32_MAX || count_max >= (1 << 18)) return I2G_OK;
    if (alloc_injected(c)) return fail(c, I2G_ENOMEM, "fused buckets: injected failure (I2G_FAIL_ALLOC_AT)");
    cudaError_t e = cudaMalloc((void **)&c->fz.ra, sizeof(float4) * (size_t)(c->ncells * cap) + 64);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c->fz.ra = nullptr;
        return fail(c, I2G_ENOMEM, std::string("fused buckets: ") + cudaGetErrorString(e));
    }
    c->fz.cap = (int32_t)cap;
    return I2G_OK;
}

// record moves of the fused step: four times the general path's interval
int32_t fused_reorder_every(const i2g_ctx *c) { return 4 * c->reorder_every; }

int resort(i2g_ctx *c)
{
    TRY(refresh_keys(c));
    MarkerView src = marker_view(c, c->cur), dst = marker_view(c, 1 - c->cur);
    PhaseTimer t(c, 1);
    c->launches += sort_markers(c->stream, c->sb, c->n, c->ncells, src, dst);
    CKL();
    c->cur = 1 - c->cur;
    c->nsorts++;
    c->keys_dirty = false;
    c->order_sorted = true;
    c->ranks_valid = false;
    c->since_reorder = 0;
    return I2G_OK;
}

// resort, then the sorted records copied back into the buffer the markers were
// in, so that device addresses captured in a graph stay valid
int resort_in_place(i2g_ctx *c)
{
    const int was = c->cur;
    TRY(resort(c));
    if (c->cur == was) return I2G_OK;
    const MarkerBuf &src = c->mb[c->cur];
    MarkerBuf &dst = c->mb[was];
    const size_t n = (size_t)c->n, d = sizeof(double) * n;
    CK(cudaMemcpyAsync(dst.x, src.x, d, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(dst.y, src.y, d, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(dst.T, src.T, d, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(dst.eta, src.eta, d, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(dst.p, src.p, d, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(dst.type, src.type, n, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(dst.id, src.id, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, c->stream));
    if (c->has_tmax) CK(cudaMemcpyAsync(dst.tmax, src.tmax, d, cudaMemcpyDeviceToDevice, c->stream));
    if (c->has_hi) CK(cudaMemcpyAsync(dst.hi, src.hi, d, cudaMemcpyDeviceToDevice, c->stream));
    if (c->has_por) CK(cudaMemcpyAsync(dst.por, src.por, d, cudaMemcpyDeviceToDevice, c->stream));
    if (c->has_mag) {
        CK(cudaMemcpyAsync(dst.mgo, src.mgo, n, cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaMemcpyAsync(dst.mgt, src.mgt, d, cudaMemcpyDeviceToDevice, c->stream));
    }
    c->cur = was;
    return I2G_OK;
}

int check_ctx(i2g_ctx *c, bool need_markers)
{
    if (!c) return I2G_EINVAL;
    if (!c->grid_set) return fail(c, I2G_ESTATE, "grid not set (call i2g_set_grid first)");
    if (need_markers && !c->markers_set) return fail(c, I2G_ESTATE, "markers not set (call i2g_set_markers first)");
    if (env_long("I2G_FAIL_CUDA")) return fail(c, I2G_ECUDA, "cudaSetDevice: injected failure (I2G_FAIL_CUDA)");
    CK(cudaSetDevice(c->dev));
    return I2G_OK;
}

// radiogenic heating per kg by rock-type group at timesum (markmart.c:749-837),
// computed on the host with the same libm the reference uses
void radiogenic(double timesum, double al, double fe, double &rsi, double &rfe, double &rch)
{
    double timesumA = timesum / (365.250 * 24.000 * 3600.000);
    {
        double init_al = 1.89716e+23 * al * 4.999e-13 / (3.264e+13);
        double init_k = 0.40689 * 1.430e-11, init_u = 2.990e-12, init_uu = 1.600e-12, init_th = 1.000e-12;
        double a = init_al * exp(-timesumA * 9.6673e-7);
        double k = init_k * exp(-timesumA * 4.9867e-10);
        double u = init_u * exp(-timesumA * 9.8458e-10);
        double uu = init_uu * exp(-timesumA * 1.5541e-10);
        double th = init_th * exp(-timesumA * 4.9511e-11);
        rsi = a + k + u + uu + th;
    }
    {
        double init_fe = 1.971e+24 * fe * 4.3451e-13 / (1.183e+14);
        double init_ka = 0.090625 * 1.430e-11;
        rfe = init_fe * exp(-timesumA * 2.6660e-7) + init_ka * exp(-timesumA * 4.9867e-10);
    }
    {
        double init_al = 1.89716e+23 * al * 4.999e-13 / (3.264e+13);
        double init_u = 2.990e-12, init_uu = 1.600e-12, init_th = 1.000e-12;
        double init_fe = 1.971e+24 * fe * 4.3451e-13 / (1.183e+14);
        double init_k = 1.430e-11;
        double a = init_al * exp(-timesumA * 9.6673e-7);
        double u = init_u * exp(-timesumA * 9.8458e-10);
        double uu = init_uu * exp(-timesumA * 1.5541e-10);
        double th = init_th * exp(-timesumA * 4.9511e-11);
        double f = init_fe * exp(-timesumA * 2.6660e-7);
        double k = init_k * exp(-timesumA * 4.9867e-10);
        rch = a + f + k + u + uu + th;
    }
}

}  // namespace

// ====================================================================== ABI
extern "C" {

const char *i2g_strerror(int s)
{
    switch (s) {
    case I2G_OK: return "ok";
    case I2G_EINVAL: return "invalid argument";
    case I2G_ECAPACITY: return "capacity exceeded";
    case I2G_ECUDA: return "CUDA error";
    case I2G_ETIMEOUT: return "device wait timed out";
    case I2G_EUNSUPPORTED: return "unsupported reference mode";
    case I2G_ENOMEM: return "out of device memory";
    case I2G_ESTATE: return "invalid call order";
    default: return "unknown status";
    }
}

const char *i2g_last_error(const i2g_ctx *c) { return c ? c->err.c_str() : ""; }

int i2g_abi_version(void) { return I2G_ABI_VERSION; }

int i2g_destroy(i2g_ctx *c)
{
    if (!c) return I2G_OK;
    cudaSetDevice(c->dev);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (void *p : c->allocs) cudaFree(p);
    if (c->fz.ra) cudaFree(c->fz.ra);
    if (c->fz.host) cudaFreeHost(c->fz.host);
    if (c->fz.host_ev) cudaEventDestroy(c->fz.host_ev);
    if (c->typecheck_host) cudaFreeHost(c->typecheck_host);
    for (auto &p : c->pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    for (cudaEvent_t e : c->xev)
        if (e) cudaEventDestroy(e);
    delete c;
    return I2G_OK;
}

int i2g_create(i2g_ctx **out, const i2g_params *P, const i2g_types *T)
{
    if (!out || !P || !T) return I2G_EINVAL;
    *out = nullptr;
    if (P->abi_version != I2G_ABI_VERSION) return I2G_EINVAL;
    if (P->xnumx < 3 || P->ynumy < 3) return I2G_EINVAL;
    if (P->max_markers < 0 || P->max_markers >= (int64_t)INT32_MAX) return I2G_EINVAL;
    if ((P->xnumx - 1) * (P->ynumy - 1) > scan_max_elems()) return I2G_EINVAL;
    if (!(P->xsize > 0) || !(P->ysize > 0)) return I2G_EINVAL;
    if (P->precision != I2G_PREC_FP64 && P->precision != I2G_PREC_MIXED) return I2G_EINVAL;
    if (P->gridmod < 0 || !(P->nubeg > 0)) return I2G_EINVAL;
    if (P->intermod != 0 || P->intermod1 != 0) return I2G_EUNSUPPORTED;
    if (P->densimod < 0 || P->densimod > 2) return I2G_EUNSUPPORTED;
    if (P->viscmod < 0 || P->viscmod > 2) return I2G_EUNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return I2G_ECUDA;
    }
    if (P->device < 0 || P->device >= ndev) return I2G_EINVAL;
    i2g_ctx *c = new i2g_ctx();
    c->P = *P;
    c->Th = *T;
    c->dev = P->device;
    c->nx = P->xnumx;
    c->ny = P->ynumy;
    c->nn = c->nx * c->ny;
    c->ncells = (c->nx - 1) * (c->ny - 1);
    c->cap = P->max_markers;
    c->fail_alloc_at = env_long("I2G_FAIL_ALLOC_AT");
    auto bail = [&](int r) {
        std::string m = c->err;
        i2g_destroy(c);
        return r;
    };
    if (cudaSetDevice(c->dev) != cudaSuccess) return bail(I2G_ECUDA);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(I2G_ECUDA);
    c->own_stream = true;
    if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess) return bail(I2G_ECUDA);
    for (cudaEvent_t &e : c->xev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return bail(I2G_ECUDA);
    int r = I2G_OK;
#define A(p, n) if ((r = dalloc(c, &(p), (n))) != I2G_OK) return bail(r)
    A(c->gx, c->nx); A(c->gy, c->ny); A(c->xmid, c->nx); A(c->ymid, c->ny);
    A(c->ixb, c->nx); A(c->iyb, c->ny); A(c->ixm, c->nx); A(c->iym, c->ny);
    A(c->lx, c->nx); A(c->ly, c->ny);
    for (int k = 0; k < G_N; k++) A(c->g[k], c->nn);
    if (P->precision == I2G_PREC_MIXED) {
        A(c->vxf, c->nn); A(c->vyf, c->nn); A(c->prf, c->nn); A(c->gaf, c->nn);
        A(c->vxq, c->nn); A(c->vyq, c->nn); A(c->prq, c->nn);
        for (int k = G_EXX; k <= G_SXY; k++) A(c->ef[k], c->nn);
    }
    for (int k = 0; k < N_N; k++) A(c->node[k], c->nn);
    for (int b = 0; b < 2; b++) {
        MarkerBuf &m = c->mb[b];
        A(m.x, c->cap); A(m.y, c->cap); A(m.T, c->cap); A(m.eta, c->cap); A(m.p, c->cap);
        A(m.type, c->cap); A(m.id, c->cap);
    }
    A(c->sb.key, c->cap); A(c->sb.perm1, c->cap); A(c->sb.perm2, c->cap); A(c->sb.rank, c->cap);
    A(c->payload, payload_bytes(P->precision == I2G_PREC_MIXED, c->cap));
    A(c->sb.count, c->ncells); A(c->sb.cursor, c->ncells); A(c->sb.cstart, c->ncells + 1);
    A(c->sb.tilesum, 4096); A(c->sb.slot0, 1);
    A(c->part, (int64_t)kPart * c->ncells);
    A(c->mmpart, 3 * (int64_t)nodesum_blocks(c->nn));
    A(c->stats, 4); A(c->T0, 1); A(c->navg, 1);
    A(c->dtypes, 1);
    A(c->typecheck, 8);
    A(c->ndeferred, 1);
    if (P->precision == I2G_PREC_MIXED) {
        uint8_t *ovf = nullptr, *ctr = nullptr;
        A(ovf, (int64_t)fused_ovf_bytes() * (c->cap > 0 ? c->cap : 1));
        A(ctr, (int64_t)fused_counters_bytes());
        c->fz.ovf = reinterpret_cast<OvfRec *>(ovf);
        c->fz.ctr = reinterpret_cast<FusedCounters *>(ctr);
        A(c->fz.treset, c->cap);
        A(c->fz.defer, c->cap);
        A(c->fz.guard, c->nn);
        A(c->fz.cmax, 1);
        A(c->fz.count, c->ncells);
    }
    A(c->tconst, (int64_t)kTypeConstBytes);
    for (double *&p : c->tnode) A(p, c->nn);
    if (P->precision == I2G_PREC_MIXED) A(c->tnodef, 5 * c->nn);
    A(c->idx2, c->nx); A(c->idy2, c->ny);
    A(c->td.melt, 12);
    A(c->sinter_stuck, 1);
#undef A
    if (cudaHostAlloc((void **)&c->typecheck_host, 8 * sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        c->typecheck_host = nullptr;
        return bail(I2G_ENOMEM);
    }
    if (P->precision == I2G_PREC_MIXED) {
        if (cudaHostAlloc(&c->fz.host, fused_counters_bytes(), cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            c->fz.host = nullptr;
            return bail(I2G_ENOMEM);
        }
        if (cudaEventCreateWithFlags(&c->fz.host_ev, cudaEventDisableTiming) != cudaSuccess) return bail(I2G_ECUDA);
    }
    for (int k = 0; k < N_N; k++)
        if (cudaMemsetAsync(c->node[k], 0, sizeof(double) * (size_t)c->nn, c->stream) != cudaSuccess) return bail(I2G_ECUDA);
    if (cudaMemcpyAsync(&c->dtypes->t, T, sizeof(i2g_types), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
        return bail(I2G_ECUDA);
    if (cudaMemsetAsync(c->stats, 0, 4 * sizeof(double), c->stream) != cudaSuccess) return bail(I2G_ECUDA);
    if (cudaMemsetAsync(c->sinter_stuck, 0, sizeof(unsigned int), c->stream) != cudaSuccess) return bail(I2G_ECUDA);
    const double melt0[6] = {P->xmelt_si, 0.0, P->xmelt_fe, 0.0, P->xmelt_ice, 0.0};
    if (cudaMemcpyAsync(c->td.melt, melt0, sizeof melt0, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
        return bail(I2G_ECUDA);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(I2G_ECUDA);
    preload_sort();
    preload_fp64();
    if (P->precision == I2G_PREC_MIXED) preload_mixed();
    cudaGetLastError();
    *out = c;
    return I2G_OK;
}

int i2g_set_types(i2g_ctx *c, const i2g_types *T)
{
    if (!c || !T) return I2G_EINVAL;
    CK(cudaSetDevice(c->dev));
    c->Th = *T;
    CK(cudaMemcpyAsync(&c->dtypes->t, &c->Th, sizeof(i2g_types), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    uint64_t present = 0;
    for (int k = 0; k < c->fz.nt; k++) present |= 1ull << c->fz.slot_type[k];
    if (c->fz.nt) fused_tinfo(c, present);
    c->fz.ready = false;
    return I2G_OK;
}

int i2g_set_grid(i2g_ctx *c, const double *gx, const double *gy, const double *vx, const double *vy,
                 const double *pr, const double *exx, const double *eyy, const double *exy, const double *sxx,
                 const double *syy, const double *sxy, const double *ga, const double *mu)
{
    if (!c || !gx || !gy) return fail(c, I2G_EINVAL, "gx and gy are required");
    CK(cudaSetDevice(c->dev));
    const int64_t nx = c->nx, ny = c->ny, nn = c->nn;
    for (int64_t i = 1; i < nx; i++)
        if (!(gx[i] > gx[i - 1])) return fail(c, I2G_EINVAL, "gx must be strictly increasing");
    for (int64_t i = 1; i < ny; i++)
        if (!(gy[i] > gy[i - 1])) return fail(c, I2G_EINVAL, "gy must be strictly increasing");
    std::vector<double> xm(nx, 0.0), ym(ny, 0.0);
    std::vector<float> ixb(nx, 0.f), iyb(ny, 0.f), ixm(nx, 0.f), iym(ny, 0.f);
    for (int64_t i = 0; i + 1 < nx; i++) xm[i] = (gx[i] + gx[i + 1]) / 2.0;
    for (int64_t i = 0; i + 1 < ny; i++) ym[i] = (gy[i] + gy[i + 1]) / 2.0;
    for (int64_t i = 0; i + 1 < nx; i++) ixb[i] = (float)(1.0 / (gx[i + 1] - gx[i]));
    for (int64_t i = 0; i + 1 < ny; i++) iyb[i] = (float)(1.0 / (gy[i + 1] - gy[i]));
    for (int64_t i = 0; i + 2 < nx; i++) ixm[i] = (float)(1.0 / (xm[i + 1] - xm[i]));
    for (int64_t i = 0; i + 2 < ny; i++) iym[i] = (float)(1.0 / (ym[i + 1] - ym[i]));
    // 1.0/celdx/celdx of the diffusion term (heatmart.c:592), the same operations
    std::vector<double> idx2(nx, 0.0), idy2(ny, 0.0);
    for (int64_t i = 0; i + 1 < nx; i++) idx2[i] = 1.0 / (gx[i + 1] - gx[i]) / (gx[i + 1] - gx[i]);
    for (int64_t i = 0; i + 1 < ny; i++) idy2[i] = 1.0 / (gy[i + 1] - gy[i]) / (gy[i + 1] - gy[i]);
    std::vector<float4> lx(nx, make_float4(0.f, 0.f, 0.f, 0.f)), ly(ny, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int64_t i = 0; i + 1 < nx; i++) lx[i] = make_float4((float)(gx[i + 1] - gx[i]), ixb[i], ixm[i], 0.f);
    for (int64_t i = 0; i + 1 < ny; i++) ly[i] = make_float4((float)(gy[i + 1] - gy[i]), iyb[i], iym[i], 0.f);
    c->inv_x = (double)(nx - 1) / (gx[nx - 1] - gx[0]);
    c->inv_y = (double)(ny - 1) / (gy[ny - 1] - gy[0]);
    // uniform axes: every line within 1e-9 of a width of g[0] + i w
    auto uniform = [](const double *g, int64_t n, double &w) {
        w = (g[n - 1] - g[0]) / (double)(n - 1);
        for (int64_t i = 0; i < n; i++)
            if (!(std::fabs(g[i] - (g[0] + (double)i * w)) <= 1e-9 * w)) return false;
        return true;
    };
    double uwx = 0, uwy = 0;
    const bool ux = uniform(gx, nx, uwx), uy = uniform(gy, ny, uwy);
    c->uni = ux && uy;
    c->ux0 = gx[0];
    c->uy0 = gy[0];
    c->uwx = uwx;
    c->uwy = uwy;
    c->fz.ready = false;
    CK(cudaMemcpyAsync(c->gx, gx, sizeof(double) * nx, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->gy, gy, sizeof(double) * ny, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->xmid, xm.data(), sizeof(double) * nx, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->ymid, ym.data(), sizeof(double) * ny, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->ixb, ixb.data(), sizeof(float) * nx, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->iyb, iyb.data(), sizeof(float) * ny, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->ixm, ixm.data(), sizeof(float) * nx, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->iym, iym.data(), sizeof(float) * ny, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->lx, lx.data(), sizeof(float4) * nx, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->ly, ly.data(), sizeof(float4) * ny, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->idx2, idx2.data(), sizeof(double) * nx, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->idy2, idy2.data(), sizeof(double) * ny, cudaMemcpyHostToDevice, c->stream));
    const double *src[G_N] = {vx, vy, pr, exx, eyy, exy, sxx, syy, sxy, ga, mu};
    for (int k = 0; k < G_N; k++) {
        c->gpresent[k] = src[k] != nullptr;
        if (src[k]) CK(cudaMemcpyAsync(c->g[k], src[k], sizeof(double) * nn, cudaMemcpyHostToDevice, c->stream));
        else CK(cudaMemsetAsync(c->g[k], 0, sizeof(double) * nn, c->stream));
    }
    if (c->P.precision == I2G_PREC_MIXED) {
        launch_f64_to_f32(c->stream, nn, c->g[G_VX], c->vxf);
        launch_f64_to_f32(c->stream, nn, c->g[G_VY], c->vyf);
        launch_f64_to_f32(c->stream, nn, c->g[G_PR], c->prf);
        launch_quads(c->stream, c->nx, c->ny, c->vxf, c->vxq);
        launch_quads(c->stream, c->nx, c->ny, c->vyf, c->vyq);
        launch_quads(c->stream, c->nx, c->ny, c->prf, c->prq);
        // a uniform grid's quarter-cell forms (indexed in int32 by the kernels)
        if (c->uni && 8 * (c->nx - 1) * (c->ny - 1) < (int64_t)INT32_MAX) {
            if (!c->vq4) TRY(dalloc(c, &c->vq4, 8 * (c->nx - 1) * (c->ny - 1)));
            launch_quarters(c->stream, c->nx, c->ny, c->vxf, c->vyf, c->vq4);
        }
        launch_f64_to_f32(c->stream, nn, c->g[G_GA], c->gaf);
        for (int k = G_EXX; k <= G_SXY; k++)
            if (c->gpresent[k]) launch_f64_to_f32(c->stream, nn, c->g[k], c->ef[k]);
        CKL();
    }
    CK(cudaStreamSynchronize(c->stream));
    c->grid_set = true;
    return I2G_OK;
}

static int set_nodes_impl(i2g_ctx *c, const double *const *f, cudaMemcpyKind kind)
{
    if (!c) return I2G_EINVAL;
    CK(cudaSetDevice(c->dev));
    for (int k = 0; k < N_N; k++)
        if (f[k]) CK(cudaMemcpyAsync(c->node[k], f[k], sizeof(double) * (size_t)c->nn, kind, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

int i2g_set_nodes(i2g_ctx *c, const double *ro, const double *nu, const double *nd, const double *et,
                  const double *cp, const double *kt, const double *ht, const double *tk, const double *po)
{
    const double *f[N_N] = {ro, nu, nd, et, cp, kt, ht, tk, po};
    return set_nodes_impl(c, f, cudaMemcpyHostToDevice);
}

static int get_nodes_impl(i2g_ctx *c, double *const *f, cudaMemcpyKind kind)
{
    if (!c) return I2G_EINVAL;
    CK(cudaSetDevice(c->dev));
    for (int k = 0; k < N_N; k++)
        if (f[k]) CK(cudaMemcpyAsync(f[k], c->node[k], sizeof(double) * (size_t)c->nn, kind, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

int i2g_get_nodes(i2g_ctx *c, double *ro, double *nu, double *nd, double *et, double *cp, double *kt, double *ht,
                  double *tk, double *po)
{
    double *f[N_N] = {ro, nu, nd, et, cp, kt, ht, tk, po};
    return get_nodes_impl(c, f, cudaMemcpyDeviceToHost);
}

int i2g_get_nodes_dev(i2g_ctx *c, double *ro, double *nu, double *nd, double *et, double *cp, double *kt,
                      double *ht, double *tk, double *po)
{
    double *f[N_N] = {ro, nu, nd, et, cp, kt, ht, tk, po};
    return get_nodes_impl(c, f, cudaMemcpyDeviceToDevice);
}

// bad[0]: bit0 a negative type, bit1 an immobile type (>= 100); bad[1]: first such marker
__global__ void k_check_types(int64_t n, const int8_t *__restrict__ type, int *__restrict__ bad)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned lo = 0, hi = 0;  // rock types < 50 present (the averaged ones)
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int t = type[i];
        if (t < 0 || t >= 100) {
            atomicOr(bad, t < 0 ? 1 : 2);
            atomicMin(bad + 1, (int)i);
        }
        if (t >= 0 && t < 32) lo |= 1u << t;
        else if (t >= 32 && t < 50) hi |= 1u << (t - 32);
    }
    lo = __reduce_or_sync(0xffffffffu, lo);
    hi = __reduce_or_sync(0xffffffffu, hi);
    if ((threadIdx.x & 31) == 0) {
        if (lo) atomicOr((unsigned *)bad + 2, lo);
        if (hi) atomicOr((unsigned *)bad + 3, hi);
    }
}

// Markers in the caller's order -> the current buffer in the canonical sorted
// order.  host: the arrays are host memory (FP64, or FP32 when f32); they are
// staged in the idle buffer by the copy stream, x and y first, so the cell keys
// and the ranking run while T, eta and type are still in flight.  !host: FP64
// device arrays, read in place.  One gather then widens and moves every field
// into its slot.  Rock types are checked on the device and read after the one
// final synchronisation; a bad type leaves the context without markers.
static int set_markers_impl(i2g_ctx *c, int64_t n, const void *x, const void *y, const void *T, const void *eta,
                            const int8_t *type, bool host, bool f32)
{
    if (!c || n < 0 || (n > 0 && (!x || !y || !T || !eta || !type))) return fail(c, I2G_EINVAL, "bad marker arrays");
    int r = check_ctx(c, false);
    if (r) return r;
    if (n > c->cap) return fail(c, I2G_ECAPACITY, "more markers than max_markers");
    c->markers_set = false;
    c->n = n;
    c->has_tmax = c->has_hi = c->has_por = c->has_mag = false;
    c->f32_storage = f32;
    MarkerBuf &s = c->mb[1 - c->cur];
    cudaStream_t cs = c->copy_stream;
    c->typecheck_host[0] = 0;
    c->typecheck_host[1] = INT32_MAX;
    c->typecheck_host[2] = c->typecheck_host[3] = c->typecheck_host[4] = 0;
    c->fz.ready = false;
    c->keys_stale = true;
    const void *sx = x, *sy = y, *sT = T, *se = eta;
    const int8_t *st = type;
    if (host && n > 0) {
        const size_t es = f32 ? sizeof(float) : sizeof(double);
        void *px = s.x, *py = s.y, *pT = s.T, *pe = s.eta;
        if (f32) {  // two float arrays in each idle double array
            py = (float *)s.x + c->cap;
            pT = s.y;
            pe = (float *)s.y + c->cap;
        }
        CK(cudaEventRecord(c->xev[0], c->stream));  // earlier work on the idle buffer is done
        CK(cudaStreamWaitEvent(cs, c->xev[0], 0));
        CK(cudaMemcpyAsync(px, x, es * n, cudaMemcpyHostToDevice, cs));
        CK(cudaMemcpyAsync(py, y, es * n, cudaMemcpyHostToDevice, cs));
        CK(cudaEventRecord(c->xev[1], cs));
        CK(cudaMemcpyAsync(pT, T, es * n, cudaMemcpyHostToDevice, cs));
        CK(cudaMemcpyAsync(pe, eta, es * n, cudaMemcpyHostToDevice, cs));
        CK(cudaMemcpyAsync(s.type, type, (size_t)n, cudaMemcpyHostToDevice, cs));
        CK(cudaEventRecord(c->xev[2], cs));
        sx = px;
        sy = py;
        sT = pT;
        se = pe;
        st = s.type;
        CK(cudaStreamWaitEvent(c->stream, c->xev[1], 0));
    }
    const GridView G = grid_view(c);
    c->launches += launch_keys_in(c->stream, G, sx, sy, n, f32, c->sb.key);
    c->launches += launch_iota(c->stream, s.id, n);  // caller index of each caller-order marker
    c->launches += rank_markers(c->stream, c->sb, n, c->ncells, s.id, false);
    CK(cudaMemsetAsync(c->sb.slot0, 0xff, sizeof(int64_t), c->stream));
    const MarkerView B = marker_view(c, c->cur, false);
    c->launches += launch_gather_in_xy(c->stream, n, c->sb.perm2, sx, sy, f32, B, c->sb.slot0);
    CKL();
    if (host && n > 0) CK(cudaStreamWaitEvent(c->stream, c->xev[2], 0));
    if (n > 0) {
        CK(cudaMemcpyAsync(c->typecheck, c->typecheck_host, 5 * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        k_check_types<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16), 256, 0, c->stream>>>(n, st,
                                                                                                  c->typecheck);
        CKL();
        // the largest cell count of the initial sort sizes the fused path's buckets
        if (c->fz.cmax) c->launches += launch_count_max(c->stream, c->sb.count, c->ncells, c->typecheck + 4);
        CKL();
        CK(cudaMemcpyAsync(c->typecheck_host, c->typecheck, 5 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    }
    c->launches += launch_gather_in_rest(c->stream, n, c->sb.perm2, sT, se, st, f32, B);
    CKL();
    c->keys_dirty = false;
    c->order_sorted = true;
    c->ranks_valid = false;
    c->since_reorder = 0;
    c->nsorts++;
    CK(cudaStreamSynchronize(c->stream));
    const int bad = c->typecheck_host[0], first = c->typecheck_host[1];
    if (bad & 1) return fail(c, I2G_EINVAL, "negative rock type at marker " + std::to_string(first));
    if (bad & 2)
        return fail(c, I2G_EUNSUPPORTED,
                    "immobile marker (type >= 100, markmart.c:30-41) at marker " + std::to_string(first));
    if (c->fz.cmax) {
        const uint64_t present = (uint64_t)(uint32_t)c->typecheck_host[2] | ((uint64_t)(uint32_t)c->typecheck_host[3] << 32);
        fused_tinfo(c, present);
        TRY(fused_buckets(c, c->typecheck_host[4]));
    }
    c->markers_set = true;
    return I2G_OK;
}

int i2g_set_markers(i2g_ctx *c, int64_t n, const double *x, const double *y, const double *T, const double *eta,
                    const int8_t *type)
{
    return set_markers_impl(c, n, x, y, T, eta, type, true, false);
}

int i2g_set_markers_dev(i2g_ctx *c, int64_t n, const double *x, const double *y, const double *T, const double *eta,
                        const int8_t *type)
{
    return set_markers_impl(c, n, x, y, T, eta, type, false, false);
}

// caller-order host array -> device-order field (dst[j] = src[id[j]])
__global__ void k_sortin_f64(int64_t n, const int32_t *__restrict__ id, const double *__restrict__ src,
                             double *__restrict__ dst)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) dst[j] = src[id[j]];
}

__global__ void k_sortin_i8(int64_t n, const int32_t *__restrict__ id, const int8_t *__restrict__ src,
                            int8_t *__restrict__ dst)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) dst[j] = src[id[j]];
}

// The markers of the averaging call that assign the magnetisation time
// (markmart.c:651-744): flag[id] = id and val[id] = the value, else flag[id] = -1.
// The filter of markmart.c:277 and the sticky-air temperature of markmart.c:301.
__global__ void __launch_bounds__(256) k_mag_flags(const __grid_constant__ GridView G,
                                                   const __grid_constant__ MarkerView M,
                                                   const DevTypes *__restrict__ Ty,
                                                   const __grid_constant__ AvgArgsK A, int32_t *__restrict__ flag,
                                                   double *__restrict__ val)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M.n) return;
    const int32_t id = M.id[i];
    const int mt = M.type[i];
    const double x = M.x[i], y = M.y[i], Tm = M.T[i];
    bool as = false;
    double v = 0.0;
    if ((A.gridmod <= 1 || (id % A.gridmod) == 0) && mt >= 0 && x > 0 && y > 0 && x < G.xsize && y < G.ysize &&
        Tm > 0 && mt < kAvgTypes) {
        const double mtk = mt < 2 ? A.tmp_ambient : Tm;
        mag_state(A.dynamo, mt, mtk, M.mgo[i], A.timesum, as, v);
    }
    flag[id] = as ? id : -1;
    if (as) val[id] = v;
}

static int sortin(i2g_ctx *c, const double *host, double *dst)
{
    double *stage = c->mb[1 - c->cur].x;  // free between sorts
    CK(cudaMemcpyAsync(stage, host, sizeof(double) * (size_t)c->n, cudaMemcpyHostToDevice, c->stream));
    if (c->n > 0) k_sortin_f64<<<(unsigned)std::min<int64_t>((c->n + 255) / 256, 148 * 16), 256, 0, c->stream>>>(
        c->n, c->mb[c->cur].id, stage, dst);
    CKL();
    return I2G_OK;
}

int i2g_set_marker_extras(i2g_ctx *c, const double *tmax, const double *hi, const double *por)
{
    int r = check_ctx(c, true);
    if (r) return r;
    c->fz.ready = false;
    const double *src[3] = {tmax, hi, por};
    bool *flag[3] = {&c->has_tmax, &c->has_hi, &c->has_por};
    for (int k = 0; k < 3; k++) {
        if (!src[k]) { *flag[k] = false; continue; }
        for (int b = 0; b < 2; b++) {
            double **f = k == 0 ? &c->mb[b].tmax : (k == 1 ? &c->mb[b].hi : &c->mb[b].por);
            if (!*f) TRY(dalloc(c, f, c->cap));
        }
        double *dst = k == 0 ? c->mb[c->cur].tmax : (k == 1 ? c->mb[c->cur].hi : c->mb[c->cur].por);
        TRY(sortin(c, src[k], dst));
        *flag[k] = true;
    }
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

// Device order -> caller order: each field is unsorted on the context stream
// into a staging array of the idle buffer; host copies run on the copy stream,
// each as soon as its field is staged, so they overlap the next unsort.
static int get_markers_impl(i2g_ctx *c, int64_t n, double *x, double *y, double *T, double *eta, double *p,
                            double *tmax, int8_t *type, cudaMemcpyKind kind)
{
    int r = check_ctx(c, true);
    if (r) return r;
    if (n != c->n) return fail(c, I2G_EINVAL, "marker count differs from the count set");
    if (tmax && !c->has_tmax) return fail(c, I2G_ESTATE, "tmax not tracked");
    const MarkerBuf &b = c->mb[c->cur];
    MarkerBuf &s = c->mb[1 - c->cur];  // staging in caller order
    const bool host = kind == cudaMemcpyDeviceToHost;
    cudaStream_t cs = host ? c->copy_stream : c->stream;
    double *outs[6] = {x, y, T, eta, p, tmax};
    double *ins[6] = {b.x, b.y, b.T, b.eta, b.p, b.tmax};
    double *stage[6] = {s.x, s.y, s.T, s.eta, s.p, s.tmax};
    for (int k = 0; k < 6; k++) {
        if (!outs[k] || n <= 0) continue;
        c->launches += launch_unsort_f64(c->stream, n, b.id, ins[k], stage[k]);
        CKL();
        if (host) {
            CK(cudaEventRecord(c->xev[0], c->stream));
            CK(cudaStreamWaitEvent(cs, c->xev[0], 0));
        }
        CK(cudaMemcpyAsync(outs[k], stage[k], sizeof(double) * n, kind, cs));
    }
    if (type && n > 0) {
        c->launches += launch_unsort_i8(c->stream, n, b.id, b.type, s.type);
        CKL();
        if (host) {
            CK(cudaEventRecord(c->xev[0], c->stream));
            CK(cudaStreamWaitEvent(cs, c->xev[0], 0));
        }
        CK(cudaMemcpyAsync(type, s.type, (size_t)n, kind, cs));
    }
    CK(cudaStreamSynchronize(cs));
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

int i2g_get_markers(i2g_ctx *c, int64_t n, double *x, double *y, double *T, double *eta, double *p, double *tmax,
                    int8_t *type)
{
    return get_markers_impl(c, n, x, y, T, eta, p, tmax, type, cudaMemcpyDeviceToHost);
}

int i2g_get_marker_extras(i2g_ctx *c, int64_t n, double *tmax, double *hi, double *por)
{
    int r = check_ctx(c, true);
    if (r) return r;
    if (n != c->n) return fail(c, I2G_EINVAL, "marker count differs from the count set");
    const bool has[3] = {c->has_tmax, c->has_hi, c->has_por};
    double *outs[3] = {tmax, hi, por};
    for (int k = 0; k < 3; k++)
        if (outs[k] && !has[k]) return fail(c, I2G_ESTATE, "field not tracked (i2g_set_marker_extras)");
    const MarkerBuf &b = c->mb[c->cur];
    double *ins[3] = {b.tmax, b.hi, b.por};
    double *stage = c->mb[1 - c->cur].x;  // free between sorts
    for (int k = 0; k < 3; k++) {
        if (!outs[k] || n <= 0) continue;
        c->launches += launch_unsort_f64(c->stream, n, b.id, ins[k], stage);
        CKL();
        CK(cudaMemcpyAsync(outs[k], stage, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return I2G_OK;
}

int i2g_get_markers_dev(i2g_ctx *c, int64_t n, double *x, double *y, double *T, double *eta, double *p)
{
    return get_markers_impl(c, n, x, y, T, eta, p, nullptr, nullptr, cudaMemcpyDeviceToDevice);
}

int i2g_set_markers_f32(i2g_ctx *c, int64_t n, const float *x, const float *y, const float *T, const float *eta,
                        const char *type)
{
    return set_markers_impl(c, n, x, y, T, eta, (const int8_t *)type, true, true);
}

int i2g_get_markers_f32(i2g_ctx *c, int64_t n, float *x, float *y, float *T, float *eta, float *p)
{
    int r = check_ctx(c, true);
    if (r) return r;
    if (n != c->n) return fail(c, I2G_EINVAL, "marker count differs from the count set");
    // caller order and narrowing in one pass on the device, into two alternating
    // float staging arrays (the idle buffer's x holds both); each host copy runs
    // on the copy stream while the next field is unsorted
    const MarkerBuf &b = c->mb[c->cur];
    float *stage[2] = {(float *)c->mb[1 - c->cur].x, (float *)c->mb[1 - c->cur].x + c->cap};
    cudaEvent_t freed[2] = {c->xev[1], c->xev[2]};
    cudaStream_t cs = c->copy_stream;
    float *outs[5] = {x, y, T, eta, p};
    const double *ins[5] = {b.x, b.y, b.T, b.eta, b.p};
    int m = 0;
    for (int k = 0; k < 5 && n > 0; k++) {
        if (!outs[k]) continue;
        const int q = m & 1;
        if (m >= 2) CK(cudaStreamWaitEvent(c->stream, freed[q], 0));  // its previous copy is done
        c->launches += launch_unsort_f64_f32(c->stream, n, b.id, ins[k], stage[q]);
        CKL();
        CK(cudaEventRecord(c->xev[0], c->stream));
        CK(cudaStreamWaitEvent(cs, c->xev[0], 0));
        CK(cudaMemcpyAsync(outs[k], stage[q], sizeof(float) * n, cudaMemcpyDeviceToHost, cs));
        CK(cudaEventRecord(freed[q], cs));
        m++;
    }
    CK(cudaStreamSynchronize(cs));
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

static bool const_properties_call(const i2g_ctx *c, double timesum);
static AvgArgsK avg_args(const i2g_ctx *c, double timesum, uint32_t flags);

// The fused mixed step applies: mixed form, at most kFusedSlots averaged rock
// types, constant-property averaging at this time, buckets allocated, no
// adjoint recording the temperature weights.
static bool fused_call(const i2g_ctx *c, double timesum)
{
    return c->P.precision == I2G_PREC_MIXED && c->fz.enabled && c->fz.nt > 0 && c->fz.cap > 0 && !c->adj.w1 &&
           const_properties_call(c, timesum);
}

// the host copy of the last fused movemark's counters: grow the buckets when a
// cell overflowed its bucket (the overflow list kept the results exact)
static int fused_check_overflow(i2g_ctx *c)
{
    if (!c->fz.host_pending || c->in_graph) return I2G_OK;
    if (cudaEventQuery(c->fz.host_ev) != cudaSuccess) {
        cudaGetLastError();
        return I2G_OK;
    }
    c->fz.host_pending = false;
    int32_t cmax = 0, novf = 0;
    fused_host_stats(c->fz.host, &cmax, &novf);
    if (novf > 0 && cmax > c->fz.cap) {
        c->fz.overflows++;
        CK(cudaStreamSynchronize(c->stream));
        TRY(fused_buckets(c, cmax));
    }
    return I2G_OK;
}

int i2g_movemark(i2g_ctx *c, double timestep, double timesum, uint32_t flags)
{
    int r = check_ctx(c, true);
    if (r) return r;
    if (flags & ~(uint32_t)I2G_MOVE_UPDATE_VISC) return fail(c, I2G_EINVAL, "unknown movemark flag");
    if (c->P.precision == I2G_PREC_MIXED) TRY(fused_check_overflow(c));
    c->fz.ready = false;
    c->timestep = timestep;  // the global the next averaging's sintering reads
    MoveArgs A{};
    A.timestep = timestep;
    A.timesum = timesum;
    A.relax_time = c->P.relax_time;
    A.nubeg = c->P.nubeg;
    A.nuend = c->P.nuend;
    A.markmod = c->P.markmod;
    A.outgrid = c->P.outgrid;
    A.flags = flags;
    A.f32pos = c->f32_storage ? 1 : 0;
    StepLaunch L{c->stream, grid_view(c), marker_view(c, c->cur), c->dtypes};
    if (fused_call(c, timesum)) {
        // movemark with every marker's averaging record, into the cell buckets
        FusedLaunch F{};
        F.cap = c->fz.cap;
        F.ra = c->fz.ra;
        F.ovf = c->fz.ovf;
        F.count = c->fz.count;
        F.ctr = c->fz.ctr;
        F.treset = c->fz.treset;
        F.defer = c->fz.defer;
        F.stepc = c->g_stepc;
        F.stepi = c->g_stepi;
        for (int t = 0; t < kAvgTypes; t++) F.tinfo[t] = c->fz.tinfo[t];
        const AvgArgsK V = avg_args(c, timesum, 0);
        {
            PhaseTimer t(c, 0);
            CK(cudaMemsetAsync(c->fz.count, 0, sizeof(int32_t) * (size_t)c->ncells, c->stream));
            CK(cudaMemsetAsync(c->fz.ctr, 0, fused_move_counters_bytes(), c->stream));
            c->launches += launch_move_fused(L, A, V, F);
        }
        CKL();
        if (!c->fz.host_pending) {
            CK(cudaMemcpyAsync(c->fz.host, c->fz.ctr, fused_counters_bytes(), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaEventRecord(c->fz.host_ev, c->stream));
            c->fz.host_pending = true;
        }
        c->fz.ready = true;
        c->fz.resets_done = false;
        c->fz.timesum = timesum;
        c->fz.calls++;
        c->keys_stale = true;
        c->keys_dirty = false;
        c->order_sorted = false;
        c->ranks_valid = false;
        return I2G_OK;
    }
    {
        PhaseTimer t(c, 0);
        CK(cudaMemsetAsync(c->sb.count, 0, sizeof(int32_t) * (size_t)c->ncells, c->stream));
        // sb.rank holds the arrival indices until the next ranking overwrites it
        c->launches += (c->P.precision == I2G_PREC_MIXED)
                           ? launch_move_mixed(L, A, c->sb.key, c->sb.count, c->sb.rank)
                           : launch_move_fp64(L, A, c->sb.key, c->sb.count, c->sb.rank);
    }
    CKL();
    c->keys_dirty = true;
    c->keys_stale = false;
    c->order_sorted = false;
    c->ranks_valid = false;
    return I2G_OK;
}

// Every rock type the averaging takes (< 50) has constant properties in this
// call: density without P-T dependence, conductivity without temperature or
// pressure terms, no molten material yet (markmart.c:509-610), porosity not
// tracked.  Then k_contrib_const evaluates the property model from per-type
// constants.
static bool const_properties_call(const i2g_ctx *c, double timesum)
{
    if (c->P.densimod != 0 || timesum > c->P.core_form_time || c->has_por || c->has_mag) return false;
    for (int t = 0; t < kAvgTypes; t++)
        if (c->Th.markkf[t] != 0.0 || c->Th.markkp[t] != 0.0) return false;
    return true;
}

static AvgArgsK avg_args(const i2g_ctx *c, double timesum, uint32_t flags)
{
    AvgArgsK A{};
    A.timesum = timesum;
    // mtk = markk[] = (float)(tmp_ambient) (markmart.c:301): in single-precision
    // storage the reset temperature is the FP32 value
    A.tmp_ambient = c->f32_storage ? (double)(float)c->P.tmp_ambient : c->P.tmp_ambient;
    A.core_form_time = c->P.core_form_time;
    A.k_cutoff = c->P.k_cutoff;
    A.relax_time = c->P.relax_time;
    A.nubeg = c->P.nubeg;
    A.nuend = c->P.nuend;
    A.xmelt_si = c->P.xmelt_si;
    A.xmelt_fe = c->P.xmelt_fe;
    A.gridmod = c->P.gridmod;
    A.densimod = c->P.densimod;
    A.viscmod = c->P.viscmod;
    radiogenic(timesum, c->P.al2627_init, c->P.fe6056_init, A.rad_si, A.rad_fe, A.rad_ch);
    A.track_tmax = (flags & I2G_AVG_TRACK_TMAX) != 0;
    A.dynamo = c->P.dynamo;
    A.timestep = c->timestep;
    A.por_init = c->P.por_init;
    A.f32por = c->f32_storage ? 1 : 0;
    A.sinter_stuck = c->has_por ? c->sinter_stuck : nullptr;
    return A;
}

// radiogenic heat per kg of rock type t (markmart.c:749-837 groups)
// radiogenic group of rock type t (markmart.c:749-837): 1 silicate, 2 iron,
// 3 chondrite, 0 none
static int rad_group(int t)
{
    if (t == 5 || t == 6 || t == 25 || t == 26) return 1;
    if (t == 7 || t == 8 || t == 9 || t == 10 || t == 17 || t == 18 || t == 19) return 2;
    if (t == 15) return 3;
    return 0;
}

// radiogenic heat per kg of rock type t
static double rad_of(const AvgArgsK &A, int t)
{
    switch (rad_group(t)) {
    case 1: return A.rad_si;
    case 2: return A.rad_fe;
    case 3: return A.rad_ch;
    default: return 0.0;
    }
}

// The averaging from the records of a fused movemark: the sticky-air resets,
// marktmax when tracked, cell sums and nodes, the contrast clamp.  The per-type
// values (density, heat capacity, clamped conductivity, heat) are those the
// constant-property model gives (markmart.c:475-478, 639-650, 749-837).
static int fused_ronurecalc(i2g_ctx *c, double timesum, uint32_t flags)
{
    const AvgArgsK A = avg_args(c, timesum, flags);
    FusedLaunch F{};
    F.cap = c->fz.cap;
    F.ra = c->fz.ra;
    F.ovf = c->fz.ovf;
    F.count = c->fz.count;
    F.ctr = c->fz.ctr;
    F.treset = c->fz.resets_done ? nullptr : c->fz.treset;  // marker indices of the storage at movemark
    F.guard = c->fz.guard;
    F.nt = c->fz.nt;
    for (int t = 0; t < kAvgTypes; t++) F.tinfo[t] = c->fz.tinfo[t];  // slots and immobile bits
    for (int k = 0; k < c->fz.nt; k++) {
        const int t = c->fz.slot_type[k];
        double kt = c->Th.markkt[t];
        if (kt <= 0.0010) kt = 0.0010;
        if (kt >= A.k_cutoff) kt = A.k_cutoff;
        F.sv[k][0] = c->Th.markro[t];
        F.sv[k][1] = c->Th.markcp[t];
        F.sv[k][2] = kt;
        F.sv[k][3] = rad_of(A, t) * c->Th.markro[t];
        F.sro[k] = c->Th.markro[t];
        F.sgrp[k] = rad_group(t);
    }
    F.stepc = c->g_stepc;
    F.stepi = c->g_stepi;
    F.navg = c->navg;
    F.nucontr = c->P.nucontr;
    F.stats = c->stats;
    F.track_tmax = A.track_tmax;
    const GridView G = grid_view(c);
    StepLaunch L{c->stream, G, marker_view(c, c->cur), c->dtypes};
    NodeOut O{c->node[N_RO], c->node[N_NU], c->node[N_ND], c->node[N_ET], c->node[N_CP],
              c->node[N_KT], c->node[N_HT], c->node[N_TK], c->node[N_PO], nullptr};
    {
        PhaseTimer t(c, 3);
        c->launches += launch_avg_fused(L, A, F, O);
    }
    CKL();
    c->fz.resets_done = true;
    // keep the storage near cell order: every 4 x reorder_every-th fused call
    // moves the records into the canonical order (the sums do not depend on it;
    // the fused step only reads the grid near each marker, whose locality decays
    // slowly: at C3 an interval of 128 steps costs less than 32); a step captured
    // into a graph leaves that to the batch, between replays
    if (!c->in_graph && ++c->since_reorder >= fused_reorder_every(c)) TRY(resort(c));
    return I2G_OK;
}

int i2g_ronurecalc(i2g_ctx *c, double timesum, uint32_t flags)
{
    int r = check_ctx(c, true);
    if (r) return r;
    if (flags & ~(uint32_t)I2G_AVG_TRACK_TMAX) return fail(c, I2G_EINVAL, "unknown ronurecalc flag");
    if (c->P.gridmod <= 0) return fail(c, I2G_EINVAL, "gridmod must be positive (the reference loops forever)");
    if ((flags & I2G_AVG_TRACK_TMAX) && !c->has_tmax) return fail(c, I2G_ESTATE, "tmax tracking needs marker extras");
    if (c->P.densimod == 2 && !c->td.set) return fail(c, I2G_ESTATE, "densimod 2 needs the table (i2g_set_td_table)");
    if (c->fz.ready && timesum == c->fz.timesum && fused_call(c, timesum)) return fused_ronurecalc(c, timesum, flags);
    c->fz.ready = false;
    TRY(refresh_keys(c));
    // Markers sorted already: the contributions pass copies them through.  Else,
    // after ranking them by (cell, caller index), every reorder_every-th call moves
    // the records into that order; the calls between leave them in place and only
    // scatter their payload to their slots (the order the sums see is the same).
    const bool dirty = c->keys_dirty;
    if (!c->order_sorted && !c->ranks_valid) {
        PhaseTimer t(c, 1);
        c->launches += dirty ? rank_moved(c->stream, c->sb, c->n, c->ncells, c->mb[c->cur].id, c->sb.rank)
                             : rank_markers(c->stream, c->sb, c->n, c->ncells, c->mb[c->cur].id, false);
        c->ranks_valid = true;
        c->nsorts++;
    }
    CKL();
    const bool inplace = !c->order_sorted && c->since_reorder + 1 < c->reorder_every;
    AvgArgsK A = avg_args(c, timesum, flags);
    const GridView G = grid_view(c);
    const MarkerView M = marker_view(c, c->cur);
    const bool mixed = c->P.precision == I2G_PREC_MIXED;
    const bool td = c->P.densimod == 2 && c->n > 0;
    if (td) {
        // the table markers and the melt fraction each passes on, then every
        // marker's predecessor among them in the caller's order (i2g_td.cuh)
        PhaseTimer t(c, 2);
        TdArgs &D = A.td;
        D = c->td.a;
        D.prev = c->td.prev;
        D.last = c->td.prev + (c->n - 1);
        D.si = c->td.si;
        D.melt_in = c->td.melt + 6 * c->td.cur;
        D.melt_out = c->td.melt + 6 * (1 - c->td.cur);
        CK(cudaMemcpyAsync(D.melt_out, D.melt_in, 6 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        const StepLaunch L0{c->stream, G, M, c->dtypes};
        c->launches += mixed ? launch_td_melt_mixed(L0, D, c->P.gridmod, c->td.flag, c->td.si)
                             : launch_td_melt_fp64(L0, D, c->P.gridmod, c->td.flag, c->td.si);
        size_t bytes = c->td.scan_bytes;
        const int rs = td_prev_scan(c->stream, c->td.scan, &bytes, c->td.flag, c->td.prev, c->n);
        if (rs < 0) return fail(c, I2G_ECUDA, "melt-state scan");
        c->launches += rs;
        CKL();
    }
    const bool mag = c->has_mag && c->n > 0;
    if (mag) {
        // the markers that assign the magnetisation time and their values, then
        // every marker's last assigning predecessor in the caller's order (i2g_mag.cuh)
        PhaseTimer t(c, 2);
        A.mag_prev = c->mag.prev;
        A.mag_val = c->mag.val;
        A.mag_last = c->mag.prev + (c->n - 1);
        A.mag_in = c->mag.state + 2 * c->mag.cur;
        A.mag_out = c->mag.state + 2 * (1 - c->mag.cur);
        CK(cudaMemcpyAsync(A.mag_out, A.mag_in, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        k_mag_flags<<<(unsigned)((c->n + 255) / 256), 256, 0, c->stream>>>(G, M, c->dtypes, A, c->mag.flag,
                                                                            c->mag.val);
        c->launches++;
        size_t bytes = c->mag.scan_bytes;
        const int rs = td_prev_scan(c->stream, c->mag.scan, &bytes, c->mag.flag, c->mag.prev, c->n);
        if (rs < 0) return fail(c, I2G_ECUDA, "magnetisation-time scan");
        c->launches += rs;
        CKL();
    }
    AvgLaunch V{};
    V.dst = marker_view(c, 1 - c->cur);
    V.perm = c->order_sorted ? nullptr : c->sb.perm2;
    V.cstart = c->sb.cstart;
    V.T0 = c->T0;
    V.payload = c->payload;
    V.part = c->part;
    V.TX = c->TX;
    V.navg = c->navg;
    V.slot0 = c->sb.slot0;
    StepLaunch L{c->stream, G, M, c->dtypes};
    {
        PhaseTimer t(c, 2);
        c->launches += launch_t0(c->stream, G, M, c->sb.slot0, A.tmp_ambient, c->T0);
        if (inplace && const_properties_call(c, timesum)) {
            // sb.perm1 is free once the ranking is done: the deferred-marker list
            CK(cudaMemsetAsync(c->ndeferred, 0, sizeof(int32_t), c->stream));
            V.tab = c->tconst;
            c->launches += mixed ? launch_contrib_const_mixed(L, A, V, c->sb.rank, c->sb.key, c->sb.perm1, c->ndeferred)
                                 : launch_contrib_const_fp64(L, A, V, c->sb.rank, c->sb.key, c->sb.perm1, c->ndeferred);
        } else if (inplace) {
            c->launches += mixed ? launch_contrib_inplace_mixed(L, A, V, c->sb.rank, c->sb.key)
                                 : launch_contrib_inplace_fp64(L, A, V, c->sb.rank, c->sb.key);
        }
        else
            c->launches += mixed ? launch_contrib_mixed(L, A, V) : launch_contrib_fp64(L, A, V);
    }
    CKL();
    if (td) c->td.cur = 1 - c->td.cur;  // the state the call's last table marker left
    if (mag) c->mag.cur = 1 - c->mag.cur;  // the time the call's last assigning marker left
    {
        PhaseTimer t(c, 3);
        CK(cudaMemsetAsync(c->navg, 0, sizeof(unsigned long long), c->stream));
        c->launches += mixed ? launch_cellsums_mixed(L, V) : launch_cellsums_fp64(L, V);
    }
    CKL();
    {
        PhaseTimer t(c, 4);
        NodeOut O{c->node[N_RO], c->node[N_NU], c->node[N_ND], c->node[N_ET], c->node[N_CP],
                  c->node[N_KT], c->node[N_HT], c->node[N_TK], c->node[N_PO], c->adj.w1};
        c->launches += launch_nodes(c->stream, G, c->part, A, O, c->P.nucontr, c->mmpart, c->stats);
    }
    CKL();
    if (c->has_por) {
        // the sintering's grain-size search gave up for some marker (the reference
        // would repeat it forever, markmart.c:426-432)
        unsigned int stuck = 0;
        CK(cudaMemcpyAsync(&stuck, c->sinter_stuck, sizeof stuck, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemsetAsync(c->sinter_stuck, 0, sizeof stuck, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (stuck)
            return fail(c, I2G_ETIMEOUT, std::to_string(stuck) +
                                              " porous markers: the sintering grain-size search did not settle");
    }
    c->keys_dirty = false;
    if (inplace) {
        c->since_reorder++;
    } else {
        c->cur = 1 - c->cur;
        c->order_sorted = true;
        c->ranks_valid = false;
        c->since_reorder = 0;
    }
    return I2G_OK;
}

int i2g_set_fused(i2g_ctx *c, int enable)
{
    if (!c) return I2G_EINVAL;
    c->fz.enabled = enable != 0;
    c->fz.ready = false;
    return I2G_OK;
}

int i2g_set_timestep(i2g_ctx *c, double timestep)
{
    if (!c) return I2G_EINVAL;
    if (!std::isfinite(timestep)) return fail(c, I2G_EINVAL, "timestep not finite");
    c->timestep = timestep;
    return I2G_OK;
}

int i2g_set_td_table(i2g_ctx *c, const i2g_td_table *t)
{
    if (!c) return I2G_EINVAL;
    if (!t || !t->td) return fail(c, I2G_EINVAL, "table required");
    if (t->tknum < 2 || t->pbnum < 2 || t->tknum > t->tkdim || t->pbnum > t->pbdim)
        return fail(c, I2G_EINVAL, "table sizes: 2 <= tknum <= tkdim, 2 <= pbnum <= pbdim");
    if (!(t->tkstp > 0) || !(t->pbstp > 0) || !std::isfinite(t->tkmin) || !std::isfinite(t->pbmin) ||
        !std::isfinite(t->tkstp) || !std::isfinite(t->pbstp))
        return fail(c, I2G_EINVAL, "table grid: finite origin, positive steps");
    if (t->si_melting < 0 || t->si_melting > 1 || t->ice_melting < 0 || t->ice_melting > 1 || t->fe_melting < 0 ||
        t->fe_melting > 1)
        return fail(c, I2G_EINVAL, "melting switches are 0 or 1");
    CK(cudaSetDevice(c->dev));
    // density (kg/m^3) and enthalpy (J/kg) per node, formed as tdbasecalc forms
    // them (markmart.c:2147-2154): td * 1000.0, then td * 1000.0 * 4.1837
    const int64_t nodes = 2 * (int64_t)t->tknum * t->pbnum;
    std::vector<double2> h((size_t)nodes);
    for (int db = 0; db < 2; db++)
        for (int64_t n1 = 0; n1 < t->tknum; n1++)
            for (int64_t n2 = 0; n2 < t->pbnum; n2++) {
                const double *q = t->td + ((n1 * t->pbdim + n2) * 2 + db) * 5;
                h[(size_t)(((int64_t)db * t->tknum + n1) * t->pbnum + n2)] =
                    make_double2(q[0] * 1000.0, q[1] * 1000.0 * 4.1837);
            }
    if (nodes > c->td.rh_cap) {
        TRY(dalloc(c, &c->td.rh, nodes));
        c->td.rh_cap = nodes;
    }
    if (!c->td.flag) {
        TRY(dalloc(c, &c->td.flag, c->cap));
        TRY(dalloc(c, &c->td.prev, c->cap));
        TRY(dalloc(c, &c->td.si, c->cap));
        size_t bytes = 0;
        if (td_prev_scan(c->stream, nullptr, &bytes, nullptr, nullptr, c->cap > 0 ? c->cap : 1) < 0)
            return fail(c, I2G_ECUDA, "scan scratch size");
        uint8_t *scan = nullptr;
        TRY(dalloc(c, &scan, (int64_t)bytes));
        c->td.scan = scan;
        c->td.scan_bytes = bytes;
    }
    CK(cudaMemcpyAsync(c->td.rh, h.data(), sizeof(double2) * h.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    TdArgs &a = c->td.a;
    a = TdArgs{};
    a.rh = c->td.rh;
    a.tkmin = t->tkmin;
    a.pbmin = t->pbmin;
    a.tkstp = t->tkstp;
    a.pbstp = t->pbstp;
    a.tknum = t->tknum;
    a.pbnum = t->pbnum;
    a.si_melting = t->si_melting;
    a.exact = c->P.precision == I2G_PREC_FP64 ? 1 : 0;
    a.ice_melting = t->ice_melting;
    c->td.set = true;
    return I2G_OK;
}

int i2g_set_melt_state(i2g_ctx *c, const double *eps6)
{
    if (!c) return I2G_EINVAL;
    if (!eps6) return fail(c, I2G_EINVAL, "six values required");
    CK(cudaSetDevice(c->dev));
    CK(cudaMemcpyAsync(c->td.melt + 6 * c->td.cur, eps6, 6 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->P.xmelt_si = eps6[0];
    c->P.xmelt_fe = eps6[2];
    c->P.xmelt_ice = eps6[4];
    return I2G_OK;
}

int i2g_get_melt_state(i2g_ctx *c, double *eps6)
{
    if (!c) return I2G_EINVAL;
    if (!eps6) return fail(c, I2G_EINVAL, "room for six values required");
    CK(cudaSetDevice(c->dev));
    CK(cudaMemcpyAsync(eps6, c->td.melt + 6 * c->td.cur, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->P.xmelt_si = eps6[0];
    c->P.xmelt_fe = eps6[2];
    c->P.xmelt_ice = eps6[4];
    return I2G_OK;
}

int i2g_set_marker_mag(i2g_ctx *c, const int8_t *mg_old, const double *mg_time)
{
    int r = check_ctx(c, true);
    if (r) return r;
    if (!mg_old || !mg_time) return fail(c, I2G_EINVAL, "state and time arrays required");
    c->fz.ready = false;
    for (int b = 0; b < 2; b++) {
        if (!c->mb[b].mgo) TRY(dalloc(c, &c->mb[b].mgo, c->cap));
        if (!c->mb[b].mgt) TRY(dalloc(c, &c->mb[b].mgt, c->cap));
    }
    if (!c->mag.flag) {
        TRY(dalloc(c, &c->mag.flag, c->cap));
        TRY(dalloc(c, &c->mag.prev, c->cap));
        TRY(dalloc(c, &c->mag.val, c->cap));
        TRY(dalloc(c, &c->mag.state, 4));
        size_t bytes = 0;
        if (td_prev_scan(c->stream, nullptr, &bytes, nullptr, nullptr, c->cap > 0 ? c->cap : 1) < 0)
            return fail(c, I2G_ECUDA, "scan scratch size");
        uint8_t *scan = nullptr;
        TRY(dalloc(c, &scan, (int64_t)bytes));
        c->mag.scan = scan;
        c->mag.scan_bytes = bytes;
    }
    // ronurecalc's mag_time before the first assignment: the reference leaves the
    // local uninitialised; here it starts at -1 (demagnetised)
    const double m1 = -1.0;
    CK(cudaMemcpyAsync(c->mag.state + 2 * c->mag.cur, &m1, sizeof m1, cudaMemcpyHostToDevice, c->stream));
    const MarkerBuf &b = c->mb[c->cur];
    double *stage = c->mb[1 - c->cur].x;  // free between sorts
    if (c->n > 0) {
        int8_t *stage8 = c->mb[1 - c->cur].type;
        CK(cudaMemcpyAsync(stage8, mg_old, (size_t)c->n, cudaMemcpyHostToDevice, c->stream));
        k_sortin_i8<<<(unsigned)((c->n + 255) / 256), 256, 0, c->stream>>>(c->n, b.id, stage8, b.mgo);
        CK(cudaMemcpyAsync(stage, mg_time, sizeof(double) * (size_t)c->n, cudaMemcpyHostToDevice, c->stream));
        k_sortin_f64<<<(unsigned)std::min<int64_t>((c->n + 255) / 256, 148 * 16), 256, 0, c->stream>>>(
            c->n, b.id, stage, b.mgt);
        CKL();
    }
    CK(cudaStreamSynchronize(c->stream));
    c->has_mag = true;
    return I2G_OK;
}

int i2g_get_marker_mag(i2g_ctx *c, int64_t n, int8_t *mg_old, double *mg_time)
{
    int r = check_ctx(c, true);
    if (r) return r;
    if (n != c->n) return fail(c, I2G_EINVAL, "marker count differs from the count set");
    if (!c->has_mag) return fail(c, I2G_ESTATE, "magnetisation not produced (i2g_set_marker_mag)");
    const MarkerBuf &b = c->mb[c->cur];
    MarkerBuf &s = c->mb[1 - c->cur];
    if (n > 0 && mg_old) {
        c->launches += launch_unsort_i8(c->stream, n, b.id, b.mgo, s.type);
        CKL();
        CK(cudaMemcpyAsync(mg_old, s.type, (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    }
    if (n > 0 && mg_time) {
        c->launches += launch_unsort_f64(c->stream, n, b.id, b.mgt, s.x);
        CKL();
        CK(cudaMemcpyAsync(mg_time, s.x, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

static int prn_scratch(i2g_ctx *c)
{
    if (c->prn.buf) return I2G_OK;
    const int64_t cap = c->cap > 0 ? c->cap : 1;
    TRY(dalloc(c, &c->prn.buf, (int64_t)kPrnRecord * cap + 16));
    TRY(dalloc(c, &c->prn.pos, cap));
    TRY(dalloc(c, &c->prn.f, 9 * cap));
    TRY(dalloc(c, &c->prn.b, 2 * cap));
    TRY(dalloc(c, &c->prn.mgt, cap));
    return I2G_OK;
}

static inline unsigned prn_blocks(int64_t n) { return (unsigned)((n + kPrnBlock - 1) / kPrnBlock); }

int i2g_write_prn_markers(i2g_ctx *c, int64_t n, const float *gr, const float *acc, const char *mg_old,
                          const double *mg_time, void *out)
{
    int r = check_ctx(c, true);
    if (r) return r;
    if (n != c->n) return fail(c, I2G_EINVAL, "marker count differs from the count set");
    if (!out) return fail(c, I2G_EINVAL, "output buffer required");
    if (n == 0) return I2G_OK;
    TRY(prn_scratch(c));
    const int64_t cap = c->cap;
    float *dgr = gr ? c->prn.f + 6 * cap : nullptr, *dacc = acc ? c->prn.f + 8 * cap : nullptr;
    int8_t *dmgo = mg_old ? c->prn.b + cap : nullptr;
    double *dmgt = mg_time ? c->prn.mgt : nullptr;
    if (gr) CK(cudaMemcpyAsync(dgr, gr, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    if (acc) CK(cudaMemcpyAsync(dacc, acc, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    if (mg_old) CK(cudaMemcpyAsync(dmgo, mg_old, (size_t)n, cudaMemcpyHostToDevice, c->stream));
    if (mg_time) CK(cudaMemcpyAsync(dmgt, mg_time, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    const MarkerView M = marker_view(c, c->cur);
    k_prn_pos<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, M.id, c->prn.pos);
    k_prn_pack<<<prn_blocks(n), kPrnBlock, 0, c->stream>>>(n, c->prn.pos, M, dgr, dacc, dmgo, dmgt, c->prn.buf);
    c->launches += 2;
    CKL();
    CK(cudaMemcpyAsync(out, c->prn.buf, (size_t)kPrnRecord * n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

int i2g_read_prn_markers(i2g_ctx *c, int64_t n, const void *in, float *gr, float *acc, char *mg_old,
                         double *mg_time)
{
    int r = check_ctx(c, false);
    if (r) return r;
    if (n < 0 || (n > 0 && !in)) return fail(c, I2G_EINVAL, "input records required");
    if (n > c->cap) return fail(c, I2G_ECAPACITY, "more markers than max_markers");
    TRY(prn_scratch(c));
    const int64_t cap = c->cap;
    float *f = c->prn.f;
    if (n > 0) {
        CK(cudaMemcpyAsync(c->prn.buf, in, (size_t)kPrnRecord * n, cudaMemcpyHostToDevice, c->stream));
        k_prn_unpack<<<prn_blocks(n), kPrnBlock, 0, c->stream>>>(n, c->prn.buf, f, cap, c->prn.b, c->prn.b + cap,
                                                                 c->prn.mgt);
        c->launches++;
        CKL();
    }
    // the markers, then tmax, hi, por into their slots (loader's order of fields:
    // x, y, T, eta, hi, por, gr, tmax, acc)
    TRY(set_markers_impl(c, n, f, f + cap, f + 2 * cap, f + 3 * cap, c->prn.b, false, true));
    const int src[3] = {7, 4, 5};  // tmax, hi, por
    bool *flag[3] = {&c->has_tmax, &c->has_hi, &c->has_por};
    for (int k = 0; k < 3; k++) {
        for (int b = 0; b < 2; b++) {
            double **d = k == 0 ? &c->mb[b].tmax : (k == 1 ? &c->mb[b].hi : &c->mb[b].por);
            if (!*d) TRY(dalloc(c, d, c->cap));
        }
        double *dst = k == 0 ? c->mb[c->cur].tmax : (k == 1 ? c->mb[c->cur].hi : c->mb[c->cur].por);
        if (n > 0) {
            k_prn_sortin<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, c->mb[c->cur].id, f + src[k] * cap,
                                                                              dst);
            c->launches++;
        }
        *flag[k] = true;
    }
    CKL();
    if (n > 0) {
        if (gr) CK(cudaMemcpyAsync(gr, f + 6 * cap, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
        if (acc) CK(cudaMemcpyAsync(acc, f + 8 * cap, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
        if (mg_old) CK(cudaMemcpyAsync(mg_old, c->prn.b + cap, (size_t)n, cudaMemcpyDeviceToHost, c->stream));
        if (mg_time) CK(cudaMemcpyAsync(mg_time, c->prn.mgt, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

int i2g_fused_info(i2g_ctx *c, i2g_fused_stats *out)
{
    if (!c || !out) return I2G_EINVAL;
    out->enabled = c->fz.enabled ? 1 : 0;
    out->bucket_places = c->fz.cap;
    out->type_slots = c->fz.nt;
    out->uniform_grid = c->uni ? 1 : 0;
    out->fused_moves = c->fz.calls;
    out->bucket_growths = c->fz.overflows;
    return I2G_OK;
}

int i2g_set_reorder_interval(i2g_ctx *c, int32_t every)
{
    if (!c || every < 1) return fail(c, I2G_EINVAL, "reorder interval must be >= 1");
    c->reorder_every = every;
    return I2G_OK;
}

// The marker part of titerate() (heatmart.c:514-697) after the host's thermal
// solve.  The sums run in the cell-sorted order of the last ranking, which stays
// valid while the markers have not moved since (the reference calls titerate
// between ronurecalc and the next movemark); else the markers are ranked first.
static int titerate_impl(i2g_ctx *c, const double *tk_new, const double *tk_old, const double *kt,
                         const double *cp, const double *ro, double heatdif, double timestep, bool dev)
{
    int r = check_ctx(c, true);
    if (r) return r;
    if (!tk_new || !tk_old) return fail(c, I2G_EINVAL, "tk_new and tk_old are required");
    if (!std::isfinite(heatdif) || !std::isfinite(timestep)) return fail(c, I2G_EINVAL, "heatdif, timestep not finite");
    const size_t nb = sizeof(double) * (size_t)c->nn;
    const double *f[5] = {tk_new, tk_old, kt ? kt : c->node[N_KT], cp ? cp : c->node[N_CP], ro ? ro : c->node[N_RO]};
    if (!dev) {
        // host arrays: the temperatures into scratch, kt/cp/ro over the node fields
        double *d[5] = {c->tnode[0], c->tnode[1], c->node[N_KT], c->node[N_CP], c->node[N_RO]};
        for (int k = 0; k < 5; k++)
            if (k < 2 || f[k] != d[k]) {
                CK(cudaMemcpyAsync(d[k], f[k], nb, cudaMemcpyHostToDevice, c->stream));
                f[k] = d[k];
            }
    }
    const bool sums = heatdif != 0;
    c->fz.ready = false;  // marker temperatures change
    if (sums && !c->order_sorted && !c->ranks_valid) {
        TRY(refresh_keys(c));
        c->launches += c->keys_dirty ? rank_moved(c->stream, c->sb, c->n, c->ncells, c->mb[c->cur].id, c->sb.rank)
                                     : rank_markers(c->stream, c->sb, c->n, c->ncells, c->mb[c->cur].id, false);
        c->ranks_valid = true;
        c->nsorts++;
    }
    ThermArgs A{f[0], f[1], f[2], f[3], f[4], c->tnodef, c->idx2, c->idy2, heatdif, timestep};
    if (c->P.precision == I2G_PREC_MIXED)
        for (int k = 0; k < (sums ? 5 : 2); k++)
            c->launches += launch_f64_to_f32(c->stream, c->nn, f[k], c->tnodef + k * c->nn);
    AvgLaunch V{};
    V.cstart = c->sb.cstart;
    V.payload = c->payload;
    V.part = c->part;
    V.TX = c->TX;
    V.navg = nullptr;
    StepLaunch L{c->stream, grid_view(c), marker_view(c, c->cur), c->dtypes};
    const int32_t *rank = c->order_sorted ? nullptr : c->sb.rank;
    c->launches += c->P.precision == I2G_PREC_MIXED ? launch_titerate_mixed(L, A, rank, V, c->tnode[2])
                                                    : launch_titerate_fp64(L, A, rank, V, c->tnode[2]);
    CKL();
    return I2G_OK;
}

int i2g_interp_tnode(i2g_ctx *c, const double *tk, const double *tk2, double *out, double *out2)
{
    int r = check_ctx(c, true);
    if (r) return r;
    if (!tk || !out) return fail(c, I2G_EINVAL, "tk and out are required");
    if (!tk2 != !out2) return fail(c, I2G_EINVAL, "tk2 and out2 go together");
    if (!c->grid_set) return fail(c, I2G_ESTATE, "i2g_set_grid first");
    const size_t nb = sizeof(double) * (size_t)c->nn;
    CK(cudaMemcpyAsync(c->tnode[0], tk, nb, cudaMemcpyHostToDevice, c->stream));
    if (tk2) CK(cudaMemcpyAsync(c->tnode[1], tk2, nb, cudaMemcpyHostToDevice, c->stream));
    // caller-order results in the idle marker buffer (free between sorts)
    MarkerBuf &s = c->mb[1 - c->cur];
    StepLaunch L{c->stream, grid_view(c), marker_view(c, c->cur), c->dtypes};
    c->launches += launch_interp_tnode(L, c->tnode[0], tk2 ? c->tnode[1] : nullptr, s.x, tk2 ? s.y : nullptr);
    CKL();
    if (c->n > 0) {
        CK(cudaMemcpyAsync(out, s.x, sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
        if (out2) CK(cudaMemcpyAsync(out2, s.y, sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

int i2g_titerate_markers(i2g_ctx *c, const double *tk_new, const double *tk_old, const double *kt,
                         const double *cp, const double *ro, double heatdif, double timestep)
{
    return titerate_impl(c, tk_new, tk_old, kt, cp, ro, heatdif, timestep, false);
}

int i2g_titerate_markers_dev(i2g_ctx *c, const double *tk_new, const double *tk_old, const double *kt,
                             const double *cp, const double *ro, double heatdif, double timestep)
{
    return titerate_impl(c, tk_new, tk_old, kt, cp, ro, heatdif, timestep, true);
}

int i2g_step(i2g_ctx *c, double timestep, double timesum, int32_t nsteps, uint32_t mflags, uint32_t aflags)
{
    if (!c || nsteps < 0) return I2G_EINVAL;
    for (int32_t s = 0; s < nsteps; s++) {
        TRY(i2g_movemark(c, timestep, timesum, mflags));
        TRY(i2g_ronurecalc(c, timesum, aflags));
        timesum += timestep;
    }
    return I2G_OK;
}

void *i2g_stream(i2g_ctx *c) { return c ? (void *)c->stream : nullptr; }

int i2g_set_stream(i2g_ctx *c, void *stream)
{
    if (!c) return I2G_EINVAL;
    CK(cudaSetDevice(c->dev));
    CK(cudaStreamSynchronize(c->stream));
    if (c->own_stream) cudaStreamDestroy(c->stream);
    c->own_stream = false;
    c->stream = (cudaStream_t)stream;
    return I2G_OK;
}

int i2g_sync(i2g_ctx *c)
{
    if (!c) return I2G_EINVAL;
    CK(cudaSetDevice(c->dev));
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

int i2g_get_stats(i2g_ctx *c, i2g_stats *out)
{
    if (!c || !out) return I2G_EINVAL;
    CK(cudaSetDevice(c->dev));
    double st[2];
    unsigned long long na = 0;
    CK(cudaMemcpyAsync(st, c->stats, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&na, c->navg, sizeof(na), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out->numin = st[0];
    out->numax = st[1];
    out->marknum = c->n;
    out->nodenum = c->nn;
    out->markers_averaged = (int64_t)na;
    out->sorts = c->nsorts;
    return I2G_OK;
}

int i2g_profile_enable(i2g_ctx *c, int on)
{
    if (!c) return I2G_EINVAL;
    c->prof = on != 0;
    return I2G_OK;
}

int i2g_profile_read(i2g_ctx *c, i2g_profile *out, int reset)
{
    if (!c || !out) return I2G_EINVAL;
    CK(cudaSetDevice(c->dev));
    CK(cudaStreamSynchronize(c->stream));
    for (auto &p : c->pending) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, p.a, p.b));
        c->prof_ms[p.phase] += ms;
        c->prof_calls[p.phase] += 1;
        c->evpool.push_back(p.a);
        c->evpool.push_back(p.b);
    }
    c->pending.clear();
    for (int k = 0; k < I2G_PHASES; k++) {
        out->ms[k] = c->prof_ms[k];
        out->calls[k] = c->prof_calls[k];
    }
    out->launches = c->launches;
    if (reset) {
        for (int k = 0; k < I2G_PHASES; k++) {
            c->prof_ms[k] = 0;
            c->prof_calls[k] = 0;
        }
        c->launches = 0;
    }
    return I2G_OK;
}

}  // extern "C"

// ====================================================================== adjoint
extern "C" {

int i2g_adjoint_setup(i2g_ctx *c, int32_t nmodes, const double *mode_vx, const double *mode_vy)
{
    if (c) c->fz.ready = false;
    int r = check_ctx(c, true);
    if (r) return r;
    if (nmodes < 1 || nmodes > kMaxModes || !mode_vx || !mode_vy) return fail(c, I2G_EINVAL, "1..16 modes required");
    auto &A = c->adj;
    const int64_t nn = c->nn, n = c->n;
    if (!A.mvx) {
        TRY(dalloc(c, &A.mvx, nn * kMaxModes));
        TRY(dalloc(c, &A.mvy, nn * kMaxModes));
        TRY(dalloc(c, &A.amps, kMaxModes));
        TRY(dalloc(c, &A.w1, nn));
        TRY(dalloc(c, &A.g, nn));
        TRY(dalloc(c, &A.da, kMaxModes));
        TRY(dalloc(c, &A.T0, c->cap));
        TRY(dalloc(c, &A.dT, c->cap));
        TRY(dalloc(c, &A.type_by_id, c->cap));
        TRY(dalloc(c, &A.lam, c->cap));
        A.nblk = (int32_t)std::min<int64_t>((c->cap + 127) / 128, 148 * 8);
        if (A.nblk < 1) A.nblk = 1;
        TRY(dalloc(c, &A.dapart, (int64_t)A.nblk * kMaxModes));
    }
    // interleave to [node][mode] so one stencil corner reads every mode at once
    std::vector<double> hx((size_t)(nn * nmodes)), hy((size_t)(nn * nmodes));
    for (int32_t m = 0; m < nmodes; m++)
        for (int64_t i = 0; i < nn; i++) {
            hx[(size_t)(i * nmodes + m)] = mode_vx[(size_t)(m * nn + i)];
            hy[(size_t)(i * nmodes + m)] = mode_vy[(size_t)(m * nn + i)];
        }
    CK(cudaMemcpyAsync(A.mvx, hx.data(), sizeof(double) * hx.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A.mvy, hy.data(), sizeof(double) * hy.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    A.nm = nmodes;
    A.ready = false;
    (void)n;
    return I2G_OK;
}

int i2g_adjoint_forward(i2g_ctx *c, const double *amps, int32_t nsteps, double timestep, double timesum,
                        int32_t every, double *tk_out)
{
    if (c) c->fz.ready = false;
    int r = check_ctx(c, true);
    if (r) return r;
    auto &A = c->adj;
    if (!A.mvx || A.nm < 1) return fail(c, I2G_ESTATE, "i2g_adjoint_setup first");
    if (!amps || nsteps < 1 || every < 1 || every > kMaxCkptSeg) return fail(c, I2G_EINVAL, "bad adjoint arguments");
    const int64_t n = c->n;
    const int64_t nseg = (nsteps + every - 1) / every;
    if (nseg > A.ck_segs) {
        TRY(dalloc(c, &A.ck, nseg * (c->cap > 0 ? c->cap : 1)));
        A.ck_segs = nseg;
    }
    CK(cudaMemcpyAsync(A.amps, amps, sizeof(double) * A.nm, cudaMemcpyHostToDevice, c->stream));
    c->launches += launch_combine_modes(c->stream, c->nn, A.nm, A.mvx, A.mvy, A.amps, c->g[G_VX], c->g[G_VY],
                                        c->vxf, c->vyf);
    if (c->vxf) {
        c->launches += launch_quads(c->stream, c->nx, c->ny, c->vxf, c->vxq);
        c->launches += launch_quads(c->stream, c->nx, c->ny, c->vyf, c->vyq);
        if (c->vq4) c->launches += launch_quarters(c->stream, c->nx, c->ny, c->vxf, c->vyf, c->vq4);
    }
    c->gpresent[G_VX] = c->gpresent[G_VY] = true;
    if (!c->order_sorted) TRY(resort(c));
    const MarkerBuf &b = c->mb[c->cur];
    c->launches += launch_unsort_f64(c->stream, n, b.id, b.T, A.T0);
    c->launches += launch_unsort_i8(c->stream, n, b.id, b.type, A.type_by_id);
    c->launches += launch_ckpt(c->stream, marker_view(c, c->cur), A.ck);
    CKL();
    double ts = timesum;
    for (int32_t s = 0; s < nsteps; s++) {
        TRY(i2g_movemark(c, timestep, ts, 0));
        TRY(i2g_ronurecalc(c, ts, 0));
        ts += timestep;
        if ((s + 1) % every == 0 && s + 1 < nsteps)
            c->launches += launch_ckpt(c->stream, marker_view(c, c->cur), A.ck + (int64_t)((s + 1) / every) * n);
    }
    CKL();
    A.nsteps = nsteps;
    A.every = every;
    A.dt = timestep;
    A.ready = true;
    if (tk_out) {
        CK(cudaMemcpyAsync(tk_out, c->node[N_TK], sizeof(double) * c->nn, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return I2G_OK;
}

int i2g_adjoint_backward(i2g_ctx *c, const double *dL_dtk, double *dL_dT0, double *dL_damp)
{
    int r = check_ctx(c, true);
    if (r) return r;
    auto &A = c->adj;
    if (!A.ready) return fail(c, I2G_ESTATE, "i2g_adjoint_forward first");
    if (!dL_dtk) return fail(c, I2G_EINVAL, "dL_dtk required");
    CK(cudaMemcpyAsync(A.g, dL_dtk, sizeof(double) * c->nn, cudaMemcpyHostToDevice, c->stream));
    MoveArgs M{};
    M.timestep = A.dt;
    M.markmod = c->P.markmod;
    M.outgrid = c->P.outgrid;
    AdjLaunch J{};
    J.mvx = A.mvx;
    J.mvy = A.mvy;
    J.nmodes = A.nm;
    J.tk = c->node[N_TK];
    J.w1 = A.w1;
    J.g = A.g;
    J.T0 = A.T0;
    J.lam = A.lam;
    J.dT = A.dT;
    J.type_by_id = A.type_by_id;
    J.ck = A.ck;
    J.nsteps = A.nsteps;
    J.every = A.every;
    J.dapart = A.dapart;
    J.nblk = A.nblk;
    J.gridmod = c->P.gridmod;
    J.tmp_ambient = c->P.tmp_ambient;
    StepLaunch L{c->stream, grid_view(c), marker_view(c, c->cur), c->dtypes};
    c->launches += (c->P.precision == I2G_PREC_MIXED) ? launch_adjoint_mixed(L, M, J) : launch_adjoint_fp64(L, M, J);
    c->launches += launch_sum_partials(c->stream, A.dapart, A.nblk, A.nm, A.da);
    CKL();
    if (dL_dT0 && c->n > 0)
        CK(cudaMemcpyAsync(dL_dT0, A.dT, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
    if (dL_damp) CK(cudaMemcpyAsync(dL_damp, A.da, sizeof(double) * A.nm, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return I2G_OK;
}

}  // extern "C"

// ====================================================================== batches
struct i2g_batch {
    std::vector<i2g_ctx *> ctx;
    int dev = 0;
    bool mixed = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    InstDesc *dD = nullptr;
    int64_t *doff = nullptr;  // 4 x (n + 1) work offsets
    int32_t *dstep = nullptr;
    double *dstepc = nullptr;  // [n][kMaxSteps][4]
    std::vector<InstDesc> hD;
    std::vector<int64_t> hoff;
    int32_t TX = 16, move_per_sm = 8, avg_per_sm = 2, nsm = 148;
    int32_t strategy = I2G_BATCH_FUSED;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    // the streams strategy's captured step (every instance's fused step on its own
    // stream) and what it was captured for: a change of any makes it stale
    cudaGraphExec_t sexec = nullptr;
    cudaGraph_t sgraph = nullptr;
    std::vector<double> skey;
    bool graphs = true;  // i2g_batch_set_graphs
    BatchRun R{};
    std::string err;
    static constexpr int kMaxSteps = 256;
};

namespace {

int bfail(i2g_batch *b, int code, const std::string &m)
{
    if (b) b->err = m;
    return code;
}

#define BCK(call)                                                                                \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) return bfail(b, I2G_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// (re)build the descriptor table and work offsets for the current tile width
int batch_layout(i2g_batch *b)
{
    const int n = (int)b->ctx.size();
    b->hD.assign(n, InstDesc{});
    b->hoff.assign(4 * (n + 1), 0);
    int64_t *om = b->hoff.data(), *oc = om + (n + 1), *ot = oc + (n + 1), *ob = ot + (n + 1);
    for (int k = 0; k < n; k++) {
        i2g_ctx *c = b->ctx[k];
        InstDesc &d = b->hD[k];
        d.G = grid_view(c);
        d.buf[0] = marker_view(c, 0);
        d.buf[1] = marker_view(c, 1);
        d.cur = c->cur;
        d.track_tmax = 0;
        d.sb = c->sb;
        d.types = c->dtypes;
        d.part = c->part;
        d.mmpart = c->mmpart;
        d.stats = c->stats;
        d.T0 = c->T0;
        d.navg = c->navg;
        d.O = NodeOut{c->node[N_RO], c->node[N_NU], c->node[N_ND], c->node[N_ET], c->node[N_CP],
                      c->node[N_KT], c->node[N_HT], c->node[N_TK], c->node[N_PO]};
        d.payload = c->payload;
        d.move = MoveArgs{0.0, 0.0, c->P.relax_time, c->P.nubeg, c->P.nuend, c->P.markmod, c->P.outgrid, 0u};
        AvgArgsK A{};
        A.tmp_ambient = c->P.tmp_ambient;
        A.core_form_time = c->P.core_form_time;
        A.k_cutoff = c->P.k_cutoff;
        A.relax_time = c->P.relax_time;
        A.nubeg = c->P.nubeg;
        A.nuend = c->P.nuend;
        A.xmelt_si = c->P.xmelt_si;
        A.xmelt_fe = c->P.xmelt_fe;
        A.gridmod = c->P.gridmod;
        A.densimod = c->P.densimod;
        A.viscmod = c->P.viscmod;
        A.rad2 = radmax_sq_threshold(c->P.xsize);
        d.avg = A;
        d.nucontr = c->P.nucontr;
        d.n = c->n;
        d.ncells = c->ncells;
        d.nn = c->nn;
        d.ntx = (int32_t)((c->nx - 1 + b->TX - 1) / b->TX);
        const int64_t nty = (c->ny - 1 + 31) / 32;
        d.nblk = nodesum_blocks(c->nn);
        d.stepc = b->dstepc + (int64_t)k * i2g_batch::kMaxSteps * 4;
        om[k + 1] = om[k] + c->n;
        oc[k + 1] = oc[k] + c->ncells;
        ot[k + 1] = ot[k] + d.ntx * nty;
        ob[k + 1] = ob[k] + d.nblk;
    }
    BCK(cudaMemcpyAsync(b->dD, b->hD.data(), sizeof(InstDesc) * n, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->doff, b->hoff.data(), sizeof(int64_t) * 4 * (n + 1), cudaMemcpyHostToDevice, b->stream));
    b->R.D = b->dD;
    b->R.ninst = n;
    b->R.off_mark = b->doff;
    b->R.off_cell = b->doff + (n + 1);
    b->R.off_tile = b->doff + 2 * (n + 1);
    b->R.off_nblk = b->doff + 3 * (n + 1);
    b->R.tot_mark = om[n];
    b->R.tot_cell = oc[n];
    b->R.tot_tile = ot[n];
    b->R.tot_nblk = ob[n];
    b->R.step = b->dstep;
    b->R.TX = b->TX;
    return I2G_OK;
}

int batch_capture(i2g_batch *b)
{
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int mc = b->move_per_sm * b->nsm, ac = b->avg_per_sm * b->nsm;
    if (b->mixed) launch_batch_step_mixed(b->stream, b->R, mc, ac);
    else launch_batch_step_fp64(b->stream, b->R, mc, ac);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess) return bfail(b, I2G_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    b->graph = g;
    BCK(cudaGraphInstantiate(&b->exec, g, 0));
    return I2G_OK;
}

// per-instance timesum and radiogenic rates of steps s0 .. s0+ns-1 (host libm, as
// the single-instance path computes them)
int batch_stepconsts(i2g_batch *b, const double *timesum, int ns, std::vector<double> &ts_out)
{
    const int n = (int)b->ctx.size();
    std::vector<double> h((size_t)n * i2g_batch::kMaxSteps * 4, 0.0);
    ts_out.assign(timesum, timesum + n);
    for (int k = 0; k < n; k++) {
        double t = timesum[k];
        const double dt = b->hD[k].move.timestep;
        for (int s = 0; s < ns; s++) {
            double *q = &h[((size_t)k * i2g_batch::kMaxSteps + s) * 4];
            q[0] = t;
            radiogenic(t, b->ctx[k]->P.al2627_init, b->ctx[k]->P.fe6056_init, q[1], q[2], q[3]);
            t += dt;
        }
        ts_out[k] = t;
    }
    BCK(cudaMemcpyAsync(b->dstepc, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemsetAsync(b->dstep, 0, sizeof(int32_t), b->stream));
    return I2G_OK;
}

__global__ void k_batch_step_inc(int32_t *step) { *step += 1; }

// Whether one captured step can replay every step of this call: every instance
// takes the mixed form's fused step at the call's first and last timesum (the
// eligibility only changes once, at core formation), no phase profiling.
bool streams_graphable(i2g_batch *b, const double *timestep, const double *timesum, int32_t nsteps)
{
    if (!b->mixed || nsteps < 1) return false;
    for (size_t k = 0; k < b->ctx.size(); k++) {
        i2g_ctx *c = b->ctx[k];
        if (c->prof || c->n <= 0) return false;
        const double t1 = timesum[k] + (double)(nsteps - 1) * timestep[k];
        if (!fused_call(c, timesum[k]) || !fused_call(c, t1)) return false;
    }
    return true;
}

void streams_graph_drop(i2g_batch *b)
{
    if (b->sexec) cudaGraphExecDestroy(b->sexec);
    if (b->sgraph) cudaGraphDestroy(b->sgraph);
    b->sexec = nullptr;
    b->sgraph = nullptr;
    b->skey.clear();
}

// The streams strategy as a CUDA graph: one step of every instance (its own
// fused movemark and averaging, on its own stream, largest first) is captured
// with the per-step constants read from the batch's device table, then
// replayed once per step.  The host work the replays cannot repeat happens
// between calls: the bucket-overflow check before, the record moves (every
// reorder_every steps) after; a change of buffers, bucket sizes, timesteps or
// flags captures the step again.
int batch_run_streams_graph(i2g_batch *b, const double *timestep, double *timesum, int32_t nsteps, uint32_t flags,
                            float *ms)
{
    const int n = (int)b->ctx.size();
    for (auto *c : b->ctx) {
        if (fused_check_overflow(c) != I2G_OK) return bfail(b, I2G_ENOMEM, c->err);
    }
    std::vector<double> key;
    for (int k = 0; k < n; k++) {
        i2g_ctx *c = b->ctx[k];
        const uint32_t fk = ((flags & I2G_AVG_TRACK_TMAX) && c->has_tmax) ? I2G_AVG_TRACK_TMAX : 0u;
        key.insert(key.end(), {(double)c->cur, (double)(uintptr_t)c->fz.ra, (double)c->fz.cap, timestep[k],
                               (double)fk, (double)c->fz.nt, (double)c->n});
    }
    if (!b->sexec || key != b->skey) {
        streams_graph_drop(b);
        std::vector<size_t> order((size_t)n);
        for (int k = 0; k < n; k++) order[k] = (size_t)k;
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t c) { return b->ctx[a]->n > b->ctx[c]->n; });
        for (int k = 0; k < n; k++) {
            i2g_ctx *c = b->ctx[k];
            c->g_stepc = b->dstepc + (size_t)k * i2g_batch::kMaxSteps * 4;
            c->g_stepi = b->dstep;
            c->in_graph = true;
            c->fz.host_pending = false;  // every replay copies the counters out
        }
        int r = I2G_OK;
        cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            cudaEventRecord(b->ev, b->stream);
            for (auto *c : b->ctx) cudaStreamWaitEvent(c->stream, b->ev, 0);
            for (size_t q = 0; q < order.size() && r == I2G_OK; q++) {
                const size_t k = order[q];
                i2g_ctx *c = b->ctx[k];
                const uint32_t fk = ((flags & I2G_AVG_TRACK_TMAX) && c->has_tmax) ? I2G_AVG_TRACK_TMAX : 0u;
                r = i2g_movemark(c, timestep[k], timesum[k], 0u);
                if (r == I2G_OK) r = i2g_ronurecalc(c, timesum[k], fk);
                if (r != I2G_OK) b->err = std::string("instance ") + std::to_string(k) + ": " + c->err;
            }
            for (auto *c : b->ctx) {
                cudaEventRecord(c->xev[3], c->stream);
                cudaStreamWaitEvent(b->stream, c->xev[3], 0);
            }
            k_batch_step_inc<<<1, 1, 0, b->stream>>>(b->dstep);
            cudaGraph_t g = nullptr;
            e = cudaStreamEndCapture(b->stream, &g);
            if (e == cudaSuccess && r == I2G_OK) {
                b->sgraph = g;
                e = cudaGraphInstantiate(&b->sexec, g, 0);
            } else if (g) {
                cudaGraphDestroy(g);
            }
        }
        for (auto *c : b->ctx) {
            c->in_graph = false;
            c->g_stepc = nullptr;
            c->g_stepi = nullptr;
            c->fz.calls--;  // the captured movemark is counted with the replays
        }
        if (r != I2G_OK) return r;
        if (e != cudaSuccess) {
            cudaGetLastError();
            streams_graph_drop(b);
            return bfail(b, I2G_ECUDA, std::string("streams graph capture: ") + cudaGetErrorString(e));
        }
        b->skey = key;
    }
    for (int k = 0; k < n; k++) b->hD[k].move.timestep = timestep[k];
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms) {
        BCK(cudaEventCreate(&e0));
        BCK(cudaEventCreate(&e1));
    }
    bool first = true;
    for (int32_t done = 0; done < nsteps;) {
        const int ns = std::min<int32_t>(nsteps - done, i2g_batch::kMaxSteps);
        std::vector<double> tnext;
        TRY(batch_stepconsts(b, timesum, ns, tnext));
        if (ms && first) BCK(cudaEventRecord(e0, b->stream));
        first = false;
        for (int s = 0; s < ns; s++) BCK(cudaGraphLaunch(b->sexec, b->stream));
        for (int k = 0; k < n; k++) timesum[k] = tnext[k];
        done += ns;
    }
    if (ms) {
        BCK(cudaEventRecord(e1, b->stream));
        BCK(cudaEventSynchronize(e1));
        BCK(cudaEventElapsedTime(ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    // the contexts' streams order after the replays; record moves of the
    // instances that are due, copied back into the buffer the graph reads
    BCK(cudaEventRecord(b->ev, b->stream));
    for (auto *c : b->ctx) {
        BCK(cudaStreamWaitEvent(c->stream, b->ev, 0));
        c->fz.calls += nsteps;
        c->since_reorder += nsteps;
        if (c->since_reorder >= fused_reorder_every(c)) {
            if (resort_in_place(c) != I2G_OK) return bfail(b, I2G_ECUDA, c->err);
            c->since_reorder = 0;
        }
    }
    return I2G_OK;
}

// I2G_BATCH_STREAMS: every instance through its own context's step on its own
// stream; the contexts' streams start after the batch stream's earlier work and
// the batch stream waits for them at the end (the timing events sit on it)
int batch_run_streams(i2g_batch *b, const double *timestep, double *timesum, int32_t nsteps, uint32_t flags,
                      float *ms)
{
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms) {
        BCK(cudaEventCreate(&e0));
        BCK(cudaEventCreate(&e1));
        BCK(cudaEventRecord(e0, b->stream));
    }
    BCK(cudaEventRecord(b->ev, b->stream));
    for (auto *c : b->ctx) BCK(cudaStreamWaitEvent(c->stream, b->ev, 0));
    // largest instances first in every step, so their long kernels start before
    // the small ones fill the GPU
    std::vector<size_t> order(b->ctx.size());
    for (size_t k = 0; k < order.size(); k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t c) { return b->ctx[a]->n > b->ctx[c]->n; });
    int r = I2G_OK;
    for (int32_t s = 0; s < nsteps && r == I2G_OK; s++)
        for (size_t q = 0; q < order.size() && r == I2G_OK; q++) {
            const size_t k = order[q];
            i2g_ctx *c = b->ctx[k];
            const uint32_t fk = ((flags & I2G_AVG_TRACK_TMAX) && c->has_tmax) ? I2G_AVG_TRACK_TMAX : 0u;
            r = i2g_movemark(c, timestep[k], timesum[k], 0u);
            if (r == I2G_OK) r = i2g_ronurecalc(c, timesum[k], fk);
            if (r == I2G_OK) timesum[k] += timestep[k];
            if (r != I2G_OK) b->err = std::string("instance ") + std::to_string(k) + ": " + c->err;
        }
    for (auto *c : b->ctx) {
        BCK(cudaEventRecord(b->ev, c->stream));
        BCK(cudaStreamWaitEvent(b->stream, b->ev, 0));
    }
    if (ms) {
        BCK(cudaEventRecord(e1, b->stream));
        BCK(cudaEventSynchronize(e1));
        BCK(cudaEventElapsedTime(ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return r;
}

int batch_run(i2g_batch *b, const double *timestep, double *timesum, int32_t nsteps, uint32_t flags, float *ms)
{
    if (b->strategy == I2G_BATCH_STREAMS) {
        if (b->graphs && streams_graphable(b, timestep, timesum, nsteps))
            return batch_run_streams_graph(b, timestep, timesum, nsteps, flags, ms);
        return batch_run_streams(b, timestep, timesum, nsteps, flags, ms);
    }
    const int n = (int)b->ctx.size();
    bool changed = false;
    for (int k = 0; k < n; k++) {
        i2g_ctx *c = b->ctx[k];
        const int tm = ((flags & I2G_AVG_TRACK_TMAX) && c->has_tmax) ? 1 : 0;
        if (b->hD[k].move.timestep != timestep[k] || b->hD[k].track_tmax != tm || b->hD[k].cur != c->cur) changed = true;
        b->hD[k].move.timestep = timestep[k];
        b->hD[k].track_tmax = tm;
        b->hD[k].cur = c->cur;
    }
    // the batch stream waits for work queued on the contexts' streams
    for (auto *c : b->ctx) {
        BCK(cudaEventRecord(b->ev, c->stream));
        BCK(cudaStreamWaitEvent(b->stream, b->ev, 0));
    }
    if (changed) BCK(cudaMemcpyAsync(b->dD, b->hD.data(), sizeof(InstDesc) * n, cudaMemcpyHostToDevice, b->stream));
    if (!b->exec) TRY(batch_capture(b));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms) {
        BCK(cudaEventCreate(&e0));
        BCK(cudaEventCreate(&e1));
    }
    bool first = true;
    for (int32_t done = 0; done < nsteps;) {
        const int ns = std::min<int32_t>(nsteps - done, i2g_batch::kMaxSteps);
        std::vector<double> tnext;
        TRY(batch_stepconsts(b, timesum, ns, tnext));
        if (ms && first) BCK(cudaEventRecord(e0, b->stream));
        first = false;
        for (int s = 0; s < ns; s++) BCK(cudaGraphLaunch(b->exec, b->stream));
        for (int k = 0; k < n; k++) timesum[k] = tnext[k];
        done += ns;
    }
    if (ms) {
        BCK(cudaEventRecord(e1, b->stream));
        BCK(cudaEventSynchronize(e1));
        BCK(cudaEventElapsedTime(ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    // contexts: buffers flipped once per step, markers sorted, work ordered after the batch
    BCK(cudaEventRecord(b->ev, b->stream));
    for (int k = 0; k < n; k++) {
        i2g_ctx *c = b->ctx[k];
        if (nsteps & 1) c->cur = 1 - c->cur;
        b->hD[k].cur = c->cur;
        c->keys_dirty = false;
        c->keys_stale = true;
        c->fz.ready = false;
        c->order_sorted = true;
        c->ranks_valid = false;
        c->since_reorder = k % fused_reorder_every(c);  // staggered, as at batch creation
        c->nsorts += nsteps;
        BCK(cudaStreamWaitEvent(c->stream, b->ev, 0));
    }
    return I2G_OK;
}

}  // namespace

extern "C" {

int i2g_batch_destroy(i2g_batch *b)
{
    if (!b) return I2G_OK;
    cudaSetDevice(b->dev);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    streams_graph_drop(b);
    cudaFree(b->dD);
    cudaFree(b->doff);
    cudaFree(b->dstep);
    cudaFree(b->dstepc);
    if (b->ev) cudaEventDestroy(b->ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return I2G_OK;
}

int i2g_batch_create(i2g_batch **out, i2g_ctx *const *ctxs, int32_t n)
{
    if (!out || !ctxs || n <= 0) return I2G_EINVAL;
    *out = nullptr;
    for (int k = 0; k < n; k++) {
        if (!ctxs[k] || !ctxs[k]->grid_set || !ctxs[k]->markers_set) return I2G_ESTATE;
        if (ctxs[k]->P.densimod == 2 || ctxs[k]->has_por || ctxs[k]->has_mag)
            return I2G_EUNSUPPORTED;  // the table path, porosity and magnetisation run on single contexts
        if (ctxs[k]->dev != ctxs[0]->dev || ctxs[k]->P.precision != ctxs[0]->P.precision) return I2G_EINVAL;
        for (int j = 0; j < k; j++)
            if (ctxs[j] == ctxs[k]) return I2G_EINVAL;
    }
    i2g_batch *b = new i2g_batch();
    b->ctx.assign(ctxs, ctxs + n);
    // stagger the instances' record moves (every reorder_every-th averaging call),
    // so that a step of the streams strategy moves the records of a few instances,
    // not of all at once
    for (int k = 0; k < n; k++) ctxs[k]->since_reorder = k % fused_reorder_every(ctxs[k]);
    b->dev = ctxs[0]->dev;
    b->mixed = ctxs[0]->P.precision == I2G_PREC_MIXED;
    auto bail = [&](int r) {
        i2g_batch_destroy(b);
        return r;
    };
    if (cudaSetDevice(b->dev) != cudaSuccess) return bail(I2G_ECUDA);
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->dev);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(I2G_ECUDA);
    if (cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess) return bail(I2G_ECUDA);
    if (cudaMalloc(&b->dD, sizeof(InstDesc) * n) != cudaSuccess ||
        cudaMalloc(&b->doff, sizeof(int64_t) * 4 * (n + 1)) != cudaSuccess ||
        cudaMalloc(&b->dstep, sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&b->dstepc, sizeof(double) * (size_t)n * i2g_batch::kMaxSteps * 4) != cudaSuccess) {
        cudaGetLastError();
        return bail(I2G_ENOMEM);
    }
    // every instance starts from sorted markers
    for (int k = 0; k < n; k++) {
        i2g_ctx *c = ctxs[k];
        if (!c->order_sorted) {
            cudaSetDevice(c->dev);
            if (resort(c) != I2G_OK) return bail(I2G_ECUDA);
        }
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(I2G_ECUDA);
    }
    if (batch_layout(b) != I2G_OK) return bail(I2G_ECUDA);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bail(I2G_ECUDA);
    *out = b;
    return I2G_OK;
}

int i2g_batch_step(i2g_batch *b, const double *timestep, double *timesum, int32_t nsteps, uint32_t flags)
{
    if (!b || !timestep || !timesum || nsteps < 0) return I2G_EINVAL;
    if (flags & ~(uint32_t)I2G_AVG_TRACK_TMAX) return bfail(b, I2G_EINVAL, "unknown flag");
    BCK(cudaSetDevice(b->dev));
    return batch_run(b, timestep, timesum, nsteps, flags, nullptr);
}

int i2g_batch_set_graphs(i2g_batch *b, int enable)
{
    if (!b) return I2G_EINVAL;
    b->graphs = enable != 0;
    if (!b->graphs) streams_graph_drop(b);
    return I2G_OK;
}

int i2g_batch_set_tune(i2g_batch *b, const i2g_tune *t)
{
    if (!b || !t) return I2G_EINVAL;
    if (t->strategy != I2G_BATCH_FUSED && t->strategy != I2G_BATCH_STREAMS) return bfail(b, I2G_EINVAL, "strategy");
    BCK(cudaSetDevice(b->dev));
    BCK(cudaStreamSynchronize(b->stream));
    b->strategy = t->strategy;
    if (t->strategy == I2G_BATCH_STREAMS) return I2G_OK;
    if ((t->tile_cols != 8 && t->tile_cols != 16 && t->tile_cols != 32) || t->move_ctas_per_sm < 1 ||
        t->move_ctas_per_sm > 32 || t->avg_ctas_per_sm < 1 || t->avg_ctas_per_sm > 2)
        return bfail(b, I2G_EINVAL, "launch shape out of range");
    b->TX = t->tile_cols;
    b->move_per_sm = t->move_ctas_per_sm;
    b->avg_per_sm = t->avg_ctas_per_sm;
    TRY(batch_layout(b));
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    return I2G_OK;
}

int i2g_batch_autotune(i2g_batch *b, const double *timestep, double *timesum, int32_t steps_per_candidate,
                       i2g_tune *out)
{
    if (!b || !timestep || !timesum || steps_per_candidate < 1) return I2G_EINVAL;
    BCK(cudaSetDevice(b->dev));
    const int tiles[3] = {8, 16, 32}, moves[3] = {4, 8, 16}, avgs[2] = {1, 2};
    i2g_tune best{};
    best.ms_per_step = 1e300;
    int tried = 0;
    std::vector<i2g_tune> cands;
    for (int a : avgs)
        for (int t : tiles)
            for (int m : moves) cands.push_back(i2g_tune{t, m, a, 0.0, 0, I2G_BATCH_FUSED});
    cands.push_back(i2g_tune{b->TX, b->move_per_sm, b->avg_per_sm, 0.0, 0, I2G_BATCH_STREAMS});
    for (const i2g_tune &cand : cands) {
        TRY(i2g_batch_set_tune(b, &cand));
        TRY(batch_run(b, timestep, timesum, 1, 0, nullptr));  // capture + warm
        // the better of two timings (a record move of some instance can fall into one)
        double per = 1e300;
        for (int rep = 0; rep < 2; rep++) {
            float ms = 0.f;
            TRY(batch_run(b, timestep, timesum, steps_per_candidate, 0, &ms));
            per = std::min(per, (double)ms / steps_per_candidate);
        }
        tried++;
        if (per < best.ms_per_step) {
            best = cand;
            best.ms_per_step = per;
        }
    }
    best.candidates = tried;
    TRY(i2g_batch_set_tune(b, &best));
    if (out) *out = best;
    return I2G_OK;
}

void *i2g_batch_stream(i2g_batch *b) { return b ? (void *)b->stream : nullptr; }

int i2g_batch_sync(i2g_batch *b)
{
    if (!b) return I2G_EINVAL;
    BCK(cudaSetDevice(b->dev));
    BCK(cudaStreamSynchronize(b->stream));
    return I2G_OK;
}

}  // extern "C"
