/*
 * i2g.h -- C ABI of the B200 marker step for I2ELVIS_planet.
 *
 * The reference exposes the marker step as two argument-free functions over
 * process globals:
 *
 *   void movemark(void);     prototype headmart.c:365, body markmart.c:3-188,
 *                            called from i2mart.c:107
 *   void ronurecalc(void);   prototype headmart.c:366, body markmart.c:192-1019,
 *                            called from i2mart.c:146, in2mart.c:1458, impact.c:3015
 *
 * Their inputs and outputs are the global marker arrays (headmart.c:122-127),
 * node arrays (headmart.c:87-99), per-rock-type tables (headmart.c:128-132) and
 * scalar parameters (headmart.c:180-279).  This header replaces that implicit
 * interface with explicit, plain-C entry points: every array is passed as a
 * pointer plus a size, and every entry point returns a status code instead of
 * the reference's printf()+exit() (markmart.c:160, loadmart.c:910-930).
 *
 * Layout conventions are the reference's:
 *   - node index  m3 = m1*ynumy + m2  (m1 along x, m2 along y; headmart.c:87-99)
 *   - gx[xnumx], gy[ynumy] grid line coordinates in metres
 *   - staggered locations: vx at (gx[m1], (gy[m2]+gy[m2+1])/2), vy at
 *     ((gx[m1]+gx[m1+1])/2, gy[m2]), pr/exx/eyy/sxx/syy/ga at cell centres stored
 *     at index (m1>=1, m2>=1), exy/sxy and every averaged output at basic nodes,
 *     nd at cell centres (markmart.c:1378-1543, 859-872).
 *
 * Ownership: the caller keeps its arrays; the context owns device mirrors.
 * Markers stay resident on the device between calls, held internally in
 * cell-sorted order; get/set calls use the caller's marker order.
 * Threading: one context is not thread-safe; distinct contexts are independent.
 * There is no CPU fallback: without a CUDA device i2g_create() fails.
 */
#ifndef I2G_H
#define I2G_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define I2G_ABI_VERSION 1
#define I2G_MAXTYPES 200 /* MAXTMR, headmart.c:15 */

/* ---- status codes ------------------------------------------------------ */
#define I2G_OK 0
#define I2G_EINVAL 1       /* NULL pointer, bad size or flag */
#define I2G_ECAPACITY 2    /* more markers than the context holds (markmart.c:160 exits instead) */
#define I2G_ECUDA 3        /* a CUDA runtime call failed */
#define I2G_ETIMEOUT 4     /* a bounded device-side wait gave up */
#define I2G_EUNSUPPORTED 5 /* reference mode not implemented (see i2g_params) */
#define I2G_ENOMEM 6       /* device allocation failed */
#define I2G_ESTATE 7       /* call order (e.g. ronurecalc before markers are set) */

/* ---- precision forms ----------------------------------------------------- */
/* FP64: every operation in double precision, in the reference's order and
 *       without contraction, so marker positions, pressures and cell indices
 *       reproduce the reference arithmetic bit for bit.
 * MIXED: interpolation weights, interpolated velocities and property x weight
 *       products in FP32; marker coordinates, the RK4 displacement sum, the
 *       cell search, log-viscosity products and every per-node accumulation and
 *       normalisation in FP64.  Its fused step (constant-property calls) keeps
 *       each marker's averaging weights as 24-bit fixed point and its
 *       log-viscosity to 2.3e-10 of itself, and sums exactly. */
#define I2G_PREC_FP64 0
#define I2G_PREC_MIXED 1

/* ---- call flags ---------------------------------------------------------- */
/* i2g_movemark: also store the viscosity that movemark() computes with
 * viscalc() (markmart.c:57-68).  Off: per-marker viscosity is left as set. */
#define I2G_MOVE_UPDATE_VISC 0x1u
/* i2g_ronurecalc: keep the per-marker maximum temperature (marktmax,
 * markmart.c:354-360).  Needs marker extras set with a tmax array. */
#define I2G_AVG_TRACK_TMAX 0x1u

/* per-rock-type constants, headmart.c:128-132 (index = rock type) */
typedef struct i2g_types {
    double marknu[I2G_MAXTYPES], markdh[I2G_MAXTYPES], markdv[I2G_MAXTYPES];
    double markss[I2G_MAXTYPES], markmm[I2G_MAXTYPES], markll[I2G_MAXTYPES];
    double marka0[I2G_MAXTYPES], marka1[I2G_MAXTYPES], markb0[I2G_MAXTYPES];
    double markb1[I2G_MAXTYPES], marke0[I2G_MAXTYPES], marke1[I2G_MAXTYPES];
    double markro[I2G_MAXTYPES], markaa[I2G_MAXTYPES], markbb[I2G_MAXTYPES];
    double markcp[I2G_MAXTYPES], markkt[I2G_MAXTYPES], markht[I2G_MAXTYPES];
    double markkf[I2G_MAXTYPES], markkp[I2G_MAXTYPES], markn0[I2G_MAXTYPES];
    double markn1[I2G_MAXTYPES], marks0[I2G_MAXTYPES], marks1[I2G_MAXTYPES];
    int32_t markim[I2G_MAXTYPES];
} i2g_types;

/* scalar parameters and switches (headmart.c:180-279, mode.t3c:6010-6031,
 * init.t3c).  Supported: markmod 1|2, intermod = intermod1 = 0, gridmod >= 1,
 * densimod 0|1|2 (2 with i2g_set_td_table), viscmod 0|1|2, outgrid 0|1|2.
 * Everything else returns I2G_EUNSUPPORTED from i2g_create(). */
typedef struct i2g_params {
    int32_t abi_version; /* must be I2G_ABI_VERSION */
    int32_t precision;   /* I2G_PREC_FP64 | I2G_PREC_MIXED */
    int64_t xnumx, ynumy;
    int64_t max_markers;
    double xsize, ysize;
    int32_t markmod, outgrid, intermod, intermod1;
    int32_t gridmod, densimod, viscmod, dynamo;
    double nubeg, nuend, nucontr;
    double tmp_ambient, M_init, M_acc, core_form_time, k_cutoff;
    double al2627_init, fe6056_init, relax_time, por_init;
    /* melt fractions the reference reads from eps[21], eps[50], eps[52]
     * (markmart.c:287-289); only meltpart1() (markmart.c:2599-2645, densimod 2)
     * ever writes them, so with densimod 0|1 they are whatever was there (0).
     * With densimod 2 they are the starting state; see i2g_set_melt_state. */
    double xmelt_si, xmelt_fe, xmelt_ice;
    int32_t device;
    int32_t reserved[7];
} i2g_params;

typedef struct i2g_ctx i2g_ctx;

const char *i2g_strerror(int status);
/* message describing the last failure on this context ("" if none) */
const char *i2g_last_error(const i2g_ctx *ctx);
int i2g_abi_version(void);

/* Create a context for one planetesimal instance on params->device. */
int i2g_create(i2g_ctx **out, const i2g_params *params, const i2g_types *types);
int i2g_destroy(i2g_ctx *ctx);
int i2g_set_types(i2g_ctx *ctx, const i2g_types *types);

/* Grid input (host pointers, node layout, nodenum = xnumx*ynumy doubles each).
 * gx, gy are required; a NULL field is taken as all zero.  Replaces the node
 * globals that viterate() writes before movemark() (movemart.c:603). */
int i2g_set_grid(i2g_ctx *ctx, const double *gx, const double *gy, const double *vx,
                 const double *vy, const double *pr, const double *exx, const double *eyy,
                 const double *exy, const double *sxx, const double *syy, const double *sxy,
                 const double *ga, const double *mu);

/* Node state written by ronurecalc (ro, nu, nd, et, cp, kt, ht, tk, po).  The
 * reference updates a node only where markers contribute (markmart.c:917-993),
 * so set_nodes seeds the values kept elsewhere; NULL leaves a field as is. */
int i2g_set_nodes(i2g_ctx *ctx, const double *ro, const double *nu, const double *nd,
                  const double *et, const double *cp, const double *kt, const double *ht,
                  const double *tk, const double *po);
int i2g_get_nodes(i2g_ctx *ctx, double *ro, double *nu, double *nd, double *et, double *cp,
                  double *kt, double *ht, double *tk, double *po);

/* Markers in the caller's order: x, y (m), T = markk (K), eta = markv (Pa s),
 * type = markt.  Types >= 100 (immobile markers, markmart.c:30-41,118-144) are
 * rejected with I2G_EUNSUPPORTED, negative types with I2G_EINVAL; a rejected
 * call leaves the context without markers.  Returns once the host arrays may be
 * reused. */
int i2g_set_markers(i2g_ctx *ctx, int64_t n, const double *x, const double *y, const double *T,
                    const double *eta, const int8_t *type);
/* Optional per-marker fields: marktmax, markhi (impact time, used by viscalc),
 * markpor (porosity; cold pressing and sintering of markmart.c:362-466 update it
 * in i2g_ronurecalc).  NULL = not tracked (tmax) / zero (hi, por). */
int i2g_set_marker_extras(i2g_ctx *ctx, const double *tmax, const double *hi, const double *por);
/* the tracked extras in the caller's order (NULL skips; an untracked field asked
 * for is I2G_ESTATE) */
int i2g_get_marker_extras(i2g_ctx *ctx, int64_t n, double *tmax, double *hi, double *por);
/* Magnetisation (markmart.c:651-744, params->dynamo): markmg_old and
 * markmg_time in the caller's order; from then on every i2g_ronurecalc updates
 * them on the device (i2g_get_marker_mag reads them back).  ronurecalc() keeps
 * the magnetisation time in a local variable that only some branches assign, so
 * a marker stores the last value assigned before it in the caller's order; the
 * context carries it from call to call (starting at -1, where the reference's
 * local is uninitialised). */
int i2g_set_marker_mag(i2g_ctx *ctx, const int8_t *mg_old, const double *mg_time);
int i2g_get_marker_mag(i2g_ctx *ctx, int64_t n, int8_t *mg_old, double *mg_time);
/* Any NULL output is skipped.  p = markp (Pa), written by i2g_movemark. */
int i2g_get_markers(i2g_ctx *ctx, int64_t n, double *x, double *y, double *T, double *eta,
                    double *p, double *tmax, int8_t *type);

/* Same as the calls above for arrays that already live in device memory of
 * the context's device (plain device pointers). */
int i2g_set_markers_dev(i2g_ctx *ctx, int64_t n, const double *x, const double *y,
                        const double *T, const double *eta, const int8_t *type);
int i2g_get_markers_dev(i2g_ctx *ctx, int64_t n, double *x, double *y, double *T, double *eta,
                        double *p);
int i2g_get_nodes_dev(i2g_ctx *ctx, double *ro, double *nu, double *nd, double *et, double *cp,
                      double *kt, double *ht, double *tk, double *po);

/* Reference storage: the reference keeps markers in single precision
 * (headmart.c:122-125).  These accept/return those arrays directly. */
int i2g_set_markers_f32(i2g_ctx *ctx, int64_t n, const float *x, const float *y, const float *T,
                        const float *eta, const char *type);
int i2g_get_markers_f32(i2g_ctx *ctx, int64_t n, float *x, float *y, float *T, float *eta,
                        float *p);

/* movemark(): markmart.c:3-188.  timestep in seconds; timesum (s) is read only
 * by viscalc()'s impact-weakening test (markmart.c:1886-1889). */
int i2g_movemark(i2g_ctx *ctx, double timestep, double timesum, uint32_t flags);
/* ronurecalc() up to, not including, tkrecalc() (markmart.c:192-1009); the
 * boundary-temperature solve stays with the host (heatmart.c:758-829).  The
 * porosity sintering reads the global timestep: that of the last i2g_movemark,
 * or of i2g_set_timestep.  I2G_ETIMEOUT: the sintering's grain-size search did
 * not settle for some marker after 64 restarts (the reference repeats it
 * without bound, markmart.c:426-432); those markers keep their porosity. */
int i2g_ronurecalc(i2g_ctx *ctx, double timesum, uint32_t flags);
/* the timestep the next i2g_ronurecalc reads (the reference's global timestep) */
int i2g_set_timestep(i2g_ctx *ctx, double timestep);
/* nsteps x { movemark; ronurecalc; timesum += timestep } (i2mart.c:107-153
 * without the solvers in between). */
int i2g_step(i2g_ctx *ctx, double timestep, double timesum, int32_t nsteps, uint32_t move_flags,
             uint32_t avg_flags);

/* How often the averaging moves the marker records into the canonical order
 * (cell, then caller index).  On the other calls the records stay where the last
 * movemark left them and only their contributions are written in that order,
 * which saves moving every record; the results are identical for every
 * interval.  1 = every call; default 32.  The mixed form's fused step moves
 * them every 4 x that many calls.  No counterpart in the reference. */
int i2g_set_reorder_interval(i2g_ctx *ctx, int32_t every);

/* The mixed form's fused step (default on).  A movemark of a call whose
 * averaging has constant per-type properties (densimod 0, no temperature or
 * pressure terms in the conductivity, no molten material at that time, no
 * porosity; at most 4 rock types below 50 among the markers) also writes every
 * marker's averaging record into a bucket of its new cell, and the ronurecalc
 * that follows at the same timesum sums the buckets and finishes the nodes in
 * one kernel.  Those sums are exact (weights on a 2^-k grid, temperature and
 * log-viscosity terms on a common quantum), so node fields do not depend on the
 * order of the markers; they stay within 1e-6 of the FP64 form.  The sticky-air
 * temperature reset and marktmax of the averaging still happen in
 * i2g_ronurecalc.  Any other call, or a call between the two that changes the
 * markers, takes the general path.  enable = 0 turns it off (the general mixed
 * path, summed in the canonical order).  No counterpart in the reference. */
int i2g_set_fused(i2g_ctx *ctx, int enable);

/* densimod 2: the thermodynamic table of tdbasecalc() (markmart.c:2068-2276).
 * Replaces the table loadmart.c:116-209 reads from "mars_mantle" (database 0) and
 * "mars_crust" (database 1) into td[][][][] (headmart.c:137).  td points at that
 * array in the reference's layout, td[tk][pb][db][k] with declared dimensions
 * tkdim x pbdim x 2 x 5; only k = 0 (density, g/cm^3) and k = 1 (enthalpy,
 * kcal/kg) are read, for tk < tknum and pb < pbnum.  The grid of the table is
 * tkmin + i tkstp (K) by pbmin + j pbstp (bar) (loadmart.c:117-122).
 * si_melting, fe_melting, ice_melting: the mode.t3c switches meltpart1() reads
 * (loadmart.c:88-90).  Rock types 5, 6, 11, 12, 25, 26, 31, 32 take their
 * density, heat capacity, expansion term, conductivity and molten viscosity
 * from the table and flip between solid (< 20) and molten (> 20) type on their
 * melt fraction, which the context keeps on the device (i2g_get_markers type).
 * A context with densimod 2 needs the table before its first i2g_ronurecalc. */
typedef struct i2g_td_table {
    const double *td;
    int32_t tkdim, pbdim;
    int32_t tknum, pbnum;
    double tkmin, pbmin, tkstp, pbstp;
    int32_t si_melting, fe_melting, ice_melting, reserved;
} i2g_td_table;
int i2g_set_td_table(i2g_ctx *ctx, const i2g_td_table *table);

/* The globals meltpart1() leaves behind and ronurecalc() reads at the top of the
 * next marker (markmart.c:287-289): eps[21], eps[22], eps[50], eps[51], eps[52],
 * eps[53], in that order.  With densimod 2 the last table marker of each
 * i2g_ronurecalc sets them; get returns them after the context's pending work
 * (the shim copies them back into eps[]).  set also replaces params->xmelt_si,
 * xmelt_fe, xmelt_ice. */
int i2g_set_melt_state(i2g_ctx *ctx, const double *eps6);
int i2g_get_melt_state(i2g_ctx *ctx, double *eps6);

/* The marker section of the reference's binary output file (saver(),
 * loadmart.c:795-808, fl1otp = 1): per marker nine 4-byte floats (x, y, T, eta,
 * hi, por, grain size, tmax, accretion time) and three bytes (magnetisation
 * state, magnetisation time converted to char, type), I2G_PRN_RECORD_BYTES
 * each, packed, in the caller's order.  saver() writes markers 0..marknum (one
 * record past the last marker); these calls cover 0..n-1 and leave that last
 * record to the host.
 * i2g_write_prn_markers: out (host, n records) from the device-resident markers.
 * The library does not keep grain size and accretion time: pass the host's
 * arrays (caller order; NULL writes 0).  The magnetisation fields come from the
 * host's arrays when given, else from the context when it produces them
 * (i2g_set_marker_mag), else 0; tmax, hi and por are written as 0 when the
 * context does not track them.
 * i2g_read_prn_markers: loader() (loadmart.c:521-535) into the context: the
 * markers in the reference's single-precision storage (as i2g_set_markers_f32)
 * with tmax, hi and por (as i2g_set_marker_extras); gr, acc, mg_old, mg_time
 * (host, NULL = skip) receive what loader() leaves in markgr, markacc,
 * markmg_old and markmg_time: loader() stores the accretion time in both
 * magnetisation fields.  Like any new marker set it leaves the context without
 * magnetisation: hand mg_old and mg_time to i2g_set_marker_mag to carry them
 * into ronurecalc.  Errors as i2g_set_markers and i2g_set_marker_extras. */
#define I2G_PRN_RECORD_BYTES 39
int i2g_write_prn_markers(i2g_ctx *ctx, int64_t n, const float *gr, const float *acc, const char *mg_old,
                          const double *mg_time, void *out);
int i2g_read_prn_markers(i2g_ctx *ctx, int64_t n, const void *in, float *gr, float *acc, char *mg_old,
                         double *mg_time);

typedef struct i2g_fused_stats {
    int32_t enabled, bucket_places, type_slots, uniform_grid;
    int64_t fused_moves;   /* movemark calls that took the fused path */
    int64_t bucket_growths; /* times a full bucket made the context enlarge them */
} i2g_fused_stats;
int i2g_fused_info(i2g_ctx *ctx, i2g_fused_stats *out);

/* allintert() (markmart.c:1687-1745, intermod = 0) at every marker's current
 * position: the node temperature interpolated there, the point clamped to the box
 * first.  tk (and tk2, optional) are host node arrays (eps[2] and eps[3] of the
 * reference); out (and out2) receive one value per marker in the caller's order.
 * FP64 in both precision forms, in the reference's order of operations.
 * I2G_ESTATE before i2g_set_markers or i2g_set_grid; I2G_EINVAL for a NULL tk or
 * out, or tk2 without out2 (or the reverse). */
int i2g_interp_tnode(i2g_ctx *ctx, const double *tk, const double *tk2, double *out, double *out2);

/* The marker temperature update of titerate() (heatmart.c:514-697, replaces the
 * marker loops after the thermal solve there; intermod = 0), on the device-resident
 * markers.  tk_new / tk_old: node temperature after / before the host's thermal
 * solve (tk and tk2 there), host arrays in node layout.  kt, cp, ro: node fields
 * the diffusion term reads (host arrays copied over the context's node fields, as
 * i2g_set_nodes would); NULL keeps the context's (the last ronurecalc's output).
 * heatdif, timestep: the reference's globals (timestep as titerate() restores it).
 * Inside the box, fluid markers (types 50..99) take the new node temperature; rock
 * markers (< 50) without a temperature take the old one, then follow the node
 * change; with heatdif != 0 the subgrid diffusion and antidiffusion apply, their
 * node sums in the cell-sorted order of ronurecalc's.  I2G_ESTATE before
 * i2g_set_markers; I2G_EINVAL for NULL temperatures or non-finite scalars. */
int i2g_titerate_markers(i2g_ctx *ctx, const double *tk_new, const double *tk_old, const double *kt,
                         const double *cp, const double *ro, double heatdif, double timestep);
/* The same with device arrays (read in place on the context's stream, not copied;
 * kt, cp, ro NULL: the context's node fields). */
int i2g_titerate_markers_dev(i2g_ctx *ctx, const double *tk_new, const double *tk_old, const double *kt,
                             const double *cp, const double *ro, double heatdif, double timestep);

/* Stream that every kernel of the context runs on (cudaStream_t as void*). */
void *i2g_stream(i2g_ctx *ctx);
int i2g_set_stream(i2g_ctx *ctx, void *stream);
int i2g_sync(i2g_ctx *ctx);

/* Diagnostics of the last ronurecalc: viscosity limits used for the contrast
 * clamp (markmart.c:995-1009), marker and node counts. */
typedef struct i2g_stats {
    double numin, numax;
    int64_t marknum, nodenum;
    int64_t markers_averaged; /* markers that passed the ronurecalc filter (markmart.c:277) */
    int64_t sorts;            /* cell sorts performed so far */
} i2g_stats;
int i2g_get_stats(i2g_ctx *ctx, i2g_stats *out);

/* Device time per phase, measured with CUDA events recorded on the context's
 * stream around each phase (nothing else is synchronised).  Phases:
 * 0 movemark, 1 cell sort, 2 marker contributions (property model, weights,
 * sorted copy), 3 cell-corner sums, 4 node loop + contrast clamp.  Kernel
 * launches are counted whether or not timing is enabled. */
#define I2G_PHASES 5
typedef struct i2g_profile {
    double ms[I2G_PHASES];
    int64_t calls[I2G_PHASES];
    int64_t launches; /* kernels this context launched since the last reset */
} i2g_profile;
int i2g_profile_enable(i2g_ctx *ctx, int on);
/* Waits for the recorded phases, returns the sums; reset != 0 clears them. */
int i2g_profile_read(i2g_ctx *ctx, i2g_profile *out, int reset);

/* ---- adjoint ------------------------------------------------------------
 * Gradients of a loss of the final node temperatures with respect to the
 * initial marker temperatures and the amplitudes of velocity modes
 * v = sum_m a_m (vx_m, vy_m).  No counterpart in the reference.
 *
 * setup: nmodes (<= 16) unit-amplitude staggered velocity fields, node layout,
 *   nmodes*nodenum doubles each (mode-major).
 * forward: sets the grid velocity to sum_m amps[m] * mode_m, then runs nsteps x
 *   {movemark; ronurecalc; timesum += timestep} from the markers as currently
 *   set, keeping marker positions every ckpt_every (<= 16) steps; tk_out (may be
 *   NULL) receives the final node temperatures.
 * backward: dL_dtk[nodenum] in, dL_dT0[marker count] (caller order) and
 *   dL_damp[nmodes] out.  Temperatures the step replaces (sticky air
 *   markmart.c:296-309, markers leaving the box markmart.c:149-152) have zero
 *   gradient.  Positions are recomputed segment by segment from the checkpoints. */
int i2g_adjoint_setup(i2g_ctx *ctx, int32_t nmodes, const double *mode_vx, const double *mode_vy);
int i2g_adjoint_forward(i2g_ctx *ctx, const double *amps, int32_t nsteps, double timestep, double timesum,
                        int32_t ckpt_every, double *tk_out);
int i2g_adjoint_backward(i2g_ctx *ctx, const double *dL_dtk, double *dL_dT0, double *dL_damp);

/* ---- batches ------------------------------------------------------------
 * Many instances (planetesimals with their own grids and marker sets, all on
 * one device and in one precision form) stepped together: each phase of the
 * step is one launch over the work of every instance (movemark and the
 * averaging run as persistent grids), the eleven launches of a step are captured
 * once into a CUDA graph and replayed per step.  Results are identical, bit for
 * bit, to stepping each context alone; the batch borrows the contexts' device
 * state and leaves it current on return.  No counterpart in the reference,
 * which runs one planetesimal per process. */
typedef struct i2g_batch i2g_batch;

/* launch shape of a batch: averaging tile width in cell columns (8|16|32) and
 * persistent CTAs per SM for movemark and for the averaging */
typedef struct i2g_tune {
    int32_t tile_cols, move_ctas_per_sm, avg_ctas_per_sm;
    double ms_per_step;  /* measured by i2g_batch_autotune for the chosen shape */
    int32_t candidates;  /* shapes tried */
    /* I2G_BATCH_FUSED: one launch per phase over every instance, from a CUDA
     * graph (the shape fields apply); I2G_BATCH_STREAMS: every instance steps
     * through the single-context path on its own stream, the streams running
     * side by side (the shape fields are ignored).  When every instance takes the
     * mixed form's fused step for the whole call, the streams strategy captures
     * one step of all instances into a CUDA graph and replays it per step, the
     * per-step constants coming from a device table (i2g_batch_set_graphs). */
    int32_t strategy;
} i2g_tune;
#define I2G_BATCH_FUSED 0
#define I2G_BATCH_STREAMS 1

int i2g_batch_create(i2g_batch **out, i2g_ctx *const *ctxs, int32_t n);
int i2g_batch_destroy(i2g_batch *b);
/* nsteps x {movemark; ronurecalc} for every instance.  timestep[k] per instance;
 * timesum[k] is read as the first step's time and advanced by nsteps timesteps. */
int i2g_batch_step(i2g_batch *b, const double *timestep, double *timesum, int32_t nsteps, uint32_t avg_flags);
/* Times every launch shape of the fused strategy and the streams strategy for
 * steps_per_candidate steps each (these are real steps: the instances and
 * timesum advance) and keeps the fastest. */
int i2g_batch_autotune(i2g_batch *b, const double *timestep, double *timesum, int32_t steps_per_candidate,
                       i2g_tune *out);
int i2g_batch_set_tune(i2g_batch *b, const i2g_tune *t);
/* enable = 0: the streams strategy launches every step from the host (default
 * 1: replayed from a graph where it can be) */
int i2g_batch_set_graphs(i2g_batch *b, int enable);
void *i2g_batch_stream(i2g_batch *b);
int i2g_batch_sync(i2g_batch *b);

/* ---- averaging without allocation ---------------------------------------
 * No counterpart in the reference.  One ronurecalc (marker -> node averaging,
 * the same kernels and results as i2g_ronurecalc on a context that holds the
 * same markers) for callers that cannot allocate device memory at the point
 * where they average: their device memory belongs to a pool allocator that
 * must not be bypassed, or the host has reserved the device for itself, or the
 * time loop must not stall on the device synchronisation cudaMalloc/cudaFree
 * can bring.  No context and no allocation: the scratch is one static device
 * array of about 16.7 MB, held by every GPU that loads the library until the
 * process exits, which limits a call to i2g_static_max_markers() markers and
 * i2g_static_max_lines() grid lines per direction (65536 and 129); larger
 * problems return I2G_ECAPACITY.
 *
 * All array arguments are DEVICE pointers of the current device; params and
 * types are host structs (params->xnumx, ynumy, xsize, ysize, precision and the
 * averaging switches are read from it; max_markers and device are ignored).
 * pr is required; exx..sxy, ga, mu may be NULL (absent = zero / no override).
 * Markers are in the caller's order; T is in/out (the sticky-air reset).  The
 * nine node arrays are in/out: nodes that no marker reaches keep their values,
 * as in the reference.  Work is queued on `stream` (NULL = legacy default);
 * the call returns without synchronising.  The first call on each device looks
 * up the scratch array's device address: make it before any stream capture.
 * That address is kept for the life of the process; after a cudaDeviceReset
 * it no longer holds.  Every call reuses the one array, so calls that overlap
 * on the GPU (two streams or host threads on one device) race: serialise them.
 * Rock types are not validated here: a marker of a type outside [0, 50) is
 * skipped, as the reference's filter skips it (markmart.c:277), where the
 * context's i2g_set_markers rejects negative types and types >= 100. */
int64_t i2g_static_max_markers(void);
int64_t i2g_static_max_lines(void);
int i2g_ronurecalc_static(const i2g_params *params, const i2g_types *types, const double *gx, const double *gy,
                          const double *pr, const double *exx, const double *eyy, const double *exy,
                          const double *sxx, const double *syy, const double *sxy, const double *ga,
                          const double *mu, int64_t n, const double *x, const double *y, double *T,
                          const double *eta, const int8_t *type, double timesum, double *ro, double *nu, double *nd,
                          double *et, double *cp, double *kt, double *ht, double *tk, double *po, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* I2G_H */
