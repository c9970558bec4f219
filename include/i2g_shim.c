/*
 * i2g_shim.c -- movemark() and ronurecalc() of I2ELVIS_planet over the
 * reference's own globals (headmart.c), computed by libi2g on the GPU.
 *
 * The reference compiles as one translation unit: i2mart.c #includes headmart.c,
 * markmart.c and the rest.  A maintainer adds
 *
 *     #include "i2g_shim.c"
 *
 * after those includes, builds with -DUSE_I2G -I<this directory>, links with
 * -li2g -lcudart, and guards the two original bodies in markmart.c (lines 3-188
 * and 192-1019) with #ifndef USE_I2G / #endif.  The callers (i2mart.c:107,
 * i2mart.c:146, in2mart.c:1458, impact.c:3015) stay as they are.  In heatmart.c
 * the marker loops that end titerate() (lines 514-697) are guarded the same way
 * and replaced by a call to titerate_markers().
 *
 * Markers cross in the reference's single-precision storage (headmart.c:122-125).
 * I2G_SHIM_PRECISION selects the precision form (default: the mixed form;
 * I2G_PREC_FP64 gives the reference's arithmetic operation by operation).
 */
#ifdef USE_I2G
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "i2g.h"

#ifndef I2G_SHIM_PRECISION
#define I2G_SHIM_PRECISION I2G_PREC_MIXED
#endif

static i2g_ctx *g_ctx;
static double *g_tmax, *g_hi, *g_por; /* FP64 copies of marktmax, markhi, markpor */
static long g_nbuf;
static int g_have_grid; /* the context holds a grid (set by the first movemark) */

static void i2g_ok(int rc, const char *where)
{
    if (rc == I2G_OK) return;
    printf("%s: %s (%s)\n", where, i2g_strerror(rc), g_ctx ? i2g_last_error(g_ctx) : "");
    exit(0); /* the reference's own error convention, markmart.c:160 */
}

static void i2g_shim_init(void)
{
    if (g_ctx) return;
    i2g_params P;
    memset(&P, 0, sizeof P);
    P.abi_version = I2G_ABI_VERSION;
    P.precision = I2G_SHIM_PRECISION;
    P.xnumx = xnumx; P.ynumy = ynumy; P.max_markers = MAXMRK;
    P.xsize = xsize; P.ysize = ysize;
    P.markmod = markmod; P.outgrid = outgrid; P.intermod = intermod; P.intermod1 = intermod1;
    P.gridmod = gridmod; P.densimod = densimod; P.viscmod = viscmod; P.dynamo = dynamo;
    P.nubeg = nubeg; P.nuend = nuend; P.nucontr = nucontr;
    P.tmp_ambient = tmp_ambient; P.M_init = M_init; P.M_acc = M_acc;
    P.core_form_time = core_form_time; P.k_cutoff = k_cutoff;
    P.al2627_init = al2627_init; P.fe6056_init = fe6056_init;
    P.relax_time = relax_time; P.por_init = por_init;
    P.xmelt_si = eps[21]; P.xmelt_fe = eps[50]; P.xmelt_ice = eps[52];
    P.device = 0;
    static i2g_types T;
#define TAB(a) memcpy(T.a, a, sizeof T.a)
    TAB(marknu); TAB(markdh); TAB(markdv); TAB(markss); TAB(markmm); TAB(markll);
    TAB(marka0); TAB(marka1); TAB(markb0); TAB(markb1); TAB(marke0); TAB(marke1);
    TAB(markro); TAB(markaa); TAB(markbb); TAB(markcp); TAB(markkt); TAB(markht);
    TAB(markkf); TAB(markkp); TAB(markn0); TAB(markn1); TAB(marks0); TAB(marks1);
#undef TAB
    for (int k = 0; k < I2G_MAXTYPES; k++) T.markim[k] = markim[k];
    i2g_ok(i2g_create(&g_ctx, &P, &T), "i2g_create");
    if (densimod == 2) {
        /* the table loadmart.c:116-209 read, and the melting switches of mode.t3c */
        i2g_td_table D;
        memset(&D, 0, sizeof D);
        D.td = &td[0][0][0][0];
        D.tkdim = 350; D.pbdim = 350; D.tknum = tknum; D.pbnum = pbnum;
        D.tkmin = tkmin; D.pbmin = pbmin; D.tkstp = tkstp; D.pbstp = pbstp;
        D.si_melting = si_melting; D.fe_melting = fe_melting; D.ice_melting = ice_melting;
        i2g_ok(i2g_set_td_table(g_ctx, &D), "i2g_set_td_table");
    }
}

/* markers (and their maximum temperature, impact time and porosity, widened) to
 * the device; porosity in the sintering range (markmart.c:363-472) is refused */
static void i2g_shim_upload(void)
{
    if (marknum > g_nbuf) {
        free(g_tmax);
        free(g_hi);
        free(g_por);
        g_tmax = (double *)malloc(sizeof(double) * (size_t)marknum);
        g_hi = (double *)malloc(sizeof(double) * (size_t)marknum);
        g_por = (double *)malloc(sizeof(double) * (size_t)marknum);
        if (!g_tmax || !g_hi || !g_por) i2g_ok(I2G_ENOMEM, "i2g_shim_upload");
        g_nbuf = marknum;
    }
    for (long i = 0; i < marknum; i++) {
        g_tmax[i] = marktmax[i];
        g_hi[i] = markhi[i];
        g_por[i] = markpor[i];
    }
    i2g_ok(i2g_set_markers_f32(g_ctx, marknum, markx, marky, markk, markv, markt), "set_markers");
    i2g_ok(i2g_set_marker_extras(g_ctx, g_tmax, g_hi, g_por), "set_marker_extras");
    /* magnetisation state and time, updated by ronurecalc() (markmart.c:651-744) */
    i2g_ok(i2g_set_marker_mag(g_ctx, (const int8_t *)markmg_old, markmg_time), "set_marker_mag");
}

/* the node fields viterate() leaves (movemart.c:603) to the device */
static void i2g_shim_grid(void)
{
    i2g_ok(i2g_set_grid(g_ctx, gx, gy, vx, vy, pr, exx, eyy, exy, sxx, syy, sxy, ga, mu), "set_grid");
    g_have_grid = 1;
}

#ifdef I2G_SHIM_RESIDENT
/* Resident markers (-DI2G_SHIM_RESIDENT): the markers stay on the device
 * between the calls and go up only when the host changed them; the host's
 * marker arrays are current only after i2g_shim_sync_host().  Host code that
 * reads markers (output, impact(), pebbleaccr()) calls i2g_shim_sync_host()
 * first; host code that writes them sets i2g_shim_markers_changed = 1 after. */
int i2g_shim_markers_changed = 1;
static int g_host_stale, g_p_on_device; /* markp is on the device from a movemark until the next upload */

void i2g_shim_sync_host(void)
{
    if (!g_ctx || !g_host_stale) return;
    i2g_ok(i2g_get_markers_f32(g_ctx, marknum, markx, marky, markk, markv, g_p_on_device ? markp : NULL),
           "get_markers");
    i2g_ok(i2g_get_markers(g_ctx, marknum, NULL, NULL, NULL, NULL, NULL, g_tmax, (int8_t *)markt), "get_markers");
    i2g_ok(i2g_get_marker_extras(g_ctx, marknum, NULL, NULL, g_por), "get_marker_extras");
    i2g_ok(i2g_get_marker_mag(g_ctx, marknum, (int8_t *)markmg_old, markmg_time), "get_marker_mag");
    for (long i = 0; i < marknum; i++) {
        marktmax[i] = g_tmax[i];
        markpor[i] = (float)g_por[i];
    }
    g_host_stale = 0;
}

/* the host's markers to the device, when they changed since the last call */
static void i2g_shim_refresh(void)
{
    if (!i2g_shim_markers_changed) return;
    i2g_shim_upload();
    i2g_shim_markers_changed = 0;
    g_p_on_device = 0;
}
#endif

/* movemark() recomputes the viscosity of rock markers with viscalc
 * (markmart.c:46-68): I2G_MOVE_UPDATE_VISC */
void movemark(void)
{
    i2g_shim_init();
    i2g_shim_grid();
#ifdef I2G_SHIM_RESIDENT
    i2g_shim_refresh();
    i2g_ok(i2g_movemark(g_ctx, timestep, timesum, I2G_MOVE_UPDATE_VISC), "movemark");
    g_host_stale = 1;
    g_p_on_device = 1;
#else
    i2g_shim_upload();
    i2g_ok(i2g_movemark(g_ctx, timestep, timesum, I2G_MOVE_UPDATE_VISC), "movemark");
    i2g_ok(i2g_get_markers_f32(g_ctx, marknum, markx, marky, markk, markv, markp), "get_markers");
#endif
}

void ronurecalc(void)
{
    i2g_shim_init();
    /* the start-up call (in2mart.c:1458) comes before any movemark(); later calls
     * follow the cycle's movemark(), whose grid is still current (only viterate()
     * changes it, before movemark()) */
    if (!g_have_grid) i2g_shim_grid();
    /* impact() and pebbleaccr() run between the two calls and may change markers */
#ifdef I2G_SHIM_RESIDENT
    i2g_shim_refresh();
#else
    i2g_shim_upload();
#endif
    i2g_ok(i2g_set_nodes(g_ctx, ro, nu, nd, et, cp, kt, ht, tk, po), "set_nodes");
    /* the melt state meltpart1() left in eps[] (markmart.c:287-289) */
    double melt[6] = {eps[21], eps[22], eps[50], eps[51], eps[52], eps[53]};
    i2g_ok(i2g_set_melt_state(g_ctx, melt), "set_melt_state");
    i2g_ok(i2g_set_timestep(g_ctx, timestep), "set_timestep"); /* the sintering's step (markmart.c:445) */
    i2g_ok(i2g_ronurecalc(g_ctx, timesum, I2G_AVG_TRACK_TMAX), "ronurecalc");
    i2g_ok(i2g_get_nodes(g_ctx, ro, nu, nd, et, cp, kt, ht, tk, po), "get_nodes");
#ifdef I2G_SHIM_RESIDENT
    g_host_stale = 1;
#else
    i2g_ok(i2g_get_markers_f32(g_ctx, marknum, NULL, NULL, markk, NULL, NULL), "get_markers");
    /* densimod 2 flips marker types with their melt (markmart.c:2180-2181) */
    i2g_ok(i2g_get_markers(g_ctx, marknum, NULL, NULL, NULL, NULL, NULL, g_tmax,
                           densimod == 2 ? (int8_t *)markt : NULL), "get_markers");
    /* porosity after cold pressing and sintering (markmart.c:362-472) */
    i2g_ok(i2g_get_marker_extras(g_ctx, marknum, NULL, NULL, g_por), "get_marker_extras");
    i2g_ok(i2g_get_marker_mag(g_ctx, marknum, (int8_t *)markmg_old, markmg_time), "get_marker_mag");
    for (long i = 0; i < marknum; i++) {
        markpor[i] = (float)g_por[i];
        marktmax[i] = g_tmax[i];
    }
#endif
    i2g_ok(i2g_get_melt_state(g_ctx, melt), "get_melt_state");
    eps[21] = melt[0]; eps[22] = melt[1]; eps[50] = melt[2]; eps[51] = melt[3]; eps[52] = melt[4]; eps[53] = melt[5];
    i2g_stats st;
    i2g_ok(i2g_get_stats(g_ctx, &st), "get_stats");
    printf("Min, Max viscosity %e %e \n", st.numin, st.numax);
    for (long m3 = 0; m3 < nodenum; m3++) tk3[m3] = 0; /* markmart.c:998 */
    tkrecalc();                                          /* markmart.c:1013, on the host */
}

/* titerate(): the thermal solve stays on the host; its marker loops after
 * "Restore timestep" (heatmart.c:514-697) become this call.  tk2 holds the node
 * temperature from before the solve (heatmart.c:383), timestep the restored step. */
void titerate_markers(void)
{
    i2g_shim_init();
    i2g_ok(i2g_titerate_markers(g_ctx, tk, tk2, kt, cp, ro, heatdif, timestep), "titerate_markers");
#ifdef I2G_SHIM_RESIDENT
    g_host_stale = 1;
#else
    /* the host's markk for the next movemark() upload */
    i2g_ok(i2g_get_markers_f32(g_ctx, marknum, NULL, NULL, markk, NULL, NULL), "get_markers");
#endif
}
/* saver()'s marker section (loadmart.c:795-808) from the device-resident
 * markers: replaces the marker loop of the binary branch of saver(), guarded
 * with #ifndef USE_I2G / #endif, by i2g_shim_save_markers(fl).  Grain size,
 * accretion time and the magnetisation fields come from the host arrays, and
 * so does the record past the last marker (saver() writes markers 0..marknum). */
void i2g_shim_save_markers(FILE *fl)
{
    i2g_shim_init();
    if (!g_have_grid) i2g_shim_grid(); /* markers live on a grid: a save before the first movemark */
#ifdef I2G_SHIM_RESIDENT
    i2g_shim_refresh();
#else
    i2g_shim_upload();
#endif
    size_t rb = I2G_PRN_RECORD_BYTES, nb = rb * (size_t)(marknum + 1);
    unsigned char *buf = (unsigned char *)malloc(nb);
    if (!buf) i2g_ok(I2G_ENOMEM, "i2g_shim_save_markers");
    /* the host's magnetisation arrays: the same values the device holds after a
     * ronurecalc() (the shim copies them back) */
    i2g_ok(i2g_write_prn_markers(g_ctx, marknum, markgr, markacc, markmg_old, markmg_time, buf), "write_prn_markers");
    unsigned char *r = buf + rb * (size_t)marknum;
    float f[9] = {markx[marknum], marky[marknum], markk[marknum], markv[marknum], markhi[marknum],
                  markpor[marknum], markgr[marknum], marktmax[marknum], markacc[marknum]};
    memcpy(r, f, sizeof f);
    r[36] = (unsigned char)markmg_old[marknum];
    r[37] = (unsigned char)(char)markmg_time[marknum];
    r[38] = (unsigned char)markt[marknum];
    fwrite(buf, 1, nb, fl);
    free(buf);
}
#endif
