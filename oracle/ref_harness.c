/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * Driver for the UNMODIFIED reference marker step.  The reference sources are
 * #included from the reference tree at build time (oracle/Makefile passes
 * -I<reference>); nothing of them is copied here.  The reference compiles as one
 * translation unit (i2mart.c:10-19 does the same #include chain), so this file
 * plays the role of i2mart.c's main() for the two hot-path calls only:
 *
 *   movemark()    markmart.c:3-188     (called from i2mart.c:107)
 *   ronurecalc()  markmart.c:192-1019  (called from i2mart.c:146)
 *   timesum += timestep                (i2mart.c:153)
 *
 * Mode 1 (hdr[17]) instead calls titerate() (heatmart.c:320-698) once: with the
 * PARDISO stub the thermal solve leaves the solution vector x[] as this driver
 * presets it, so the node temperature after the "solve" is the given tk_new and
 * the marker temperature update that follows (heatmart.c:514-697) runs on it
 * unmodified.  Boundary nodes are marked as fixed-T boundary equations so that
 * heaterr() only ever sees interior nodes.
 *
 * Mode 2 writes the reference's binary output file with saver() (loadmart.c:553-845,
 * fl1otp = 1) into the working directory as out.prn, clears the marker arrays and
 * reads the file back with loader() (loadmart.c:218-550, fl1itp = 1): the marker
 * section of the file and the arrays loader() fills pin the library's codec.
 *
 * Mode 3 calls allintert() (markmart.c:1687-1745) at every marker with the node
 * temperature tk (the input's node field) and tk2 (given after the markers), and
 * appends eps[2] and eps[3] of each call to the output.
 *
 * Built twice: "ref32" (reference storage: float markers) and "ref64"
 * (-Dfloat=double: identical source, FP64 marker storage).  This file therefore
 * never spells the C keyword for single precision.  With -DI2G_DROPIN it is
 * also built with the C host shim in place of the two calls ("dropin32",
 * "dropin32m": the FP64 and mixed forms of libi2g, reference storage;
 * "dropin32r": the FP64 form with the markers resident on the device).
 *
 * Input/output are the little-endian binary files written/read by
 * oracle/refio.py (layout documented there).
 */
#include <stdio.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <stdint.h>
#include "mkl.h"
#include "headmart.c"
#include "loadmart.c"
#include "movemart.c"
#include "markmart.c"
#include "gausmart.c"
#include "heatmart.c"

#ifdef I2G_DROPIN
/* The drop-in build: the C host shim's movemark()/ronurecalc() (include/i2g_shim.c,
 * libi2g on the GPU) under other names beside the reference's own, and the step
 * loop below calls the shim's.  Everything else -- globals, reinjection, tkrecalc,
 * input and output -- is the same as in the reference build. */
#define movemark shim_movemark
#define ronurecalc shim_ronurecalc
#define titerate_markers shim_titerate_markers
#include "i2g_shim.c"
#undef movemark
#undef ronurecalc
#undef titerate_markers
#define STEP_MOVE shim_movemark
#define STEP_AVG shim_ronurecalc
#else
#define STEP_MOVE movemark
#define STEP_AVG ronurecalc
#endif

#define H_MAGIC 0x31473249LL /* "I2G1" */
#define NHDR 32
#define NSCAL 64
#define NTAB 24
#define NTYPES 200

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void rd(void *p, size_t sz, size_t n, FILE *f)
{
    if (fread(p, sz, n, f) != n) { fprintf(stderr, "ref_harness: short read\n"); exit(3); }
}

static void wr(const void *p, size_t sz, size_t n, FILE *f)
{
    if (fwrite(p, sz, n, f) != n) { fprintf(stderr, "ref_harness: short write\n"); exit(4); }
}

/* per-type table destinations, in the order refio.TYPE_TABLES lists them */
static double *type_table(int k)
{
    double *t[NTAB] = {marknu, markdh, markdv, markss, markmm, markll, marka0, marka1,
                       markb0, markb1, marke0, marke1, markro, markaa, markbb, markcp,
                       markkt, markht, markkf, markkp, markn0, markn1, marks0, marks1};
    return t[k];
}

/* node arrays read as input, in refio.NODE_IN order */
static double *node_in(int k)
{
    double *t[20] = {vx, vy, pr, exx, eyy, exy, sxx, syy, sxy, ga, mu,
                     ro, nu, nd, et, cp, kt, ht, tk, po};
    return t[k];
}

/* node arrays written as output, in refio.NODE_OUT order */
static double *node_out(int k)
{
    double *t[9] = {ro, nu, nd, et, cp, kt, ht, tk, po};
    return t[k];
}

int main(int argc, char **argv)
{
    if (argc < 3) { fprintf(stderr, "usage: %s in.i2gin out.i2gout\n", argv[0]); return 2; }
    FILE *fi = fopen(argv[1], "rb");
    if (!fi) { fprintf(stderr, "cannot open %s\n", argv[1]); return 2; }
    int64_t h[NHDR];
    double s[NSCAL];
    rd(h, sizeof(int64_t), NHDR, fi);
    rd(s, sizeof(double), NSCAL, fi);
    if (h[0] != H_MAGIC) { fprintf(stderr, "bad magic\n"); return 2; }

    xnumx = h[1]; ynumy = h[2]; marknum = h[3];
    long nsteps = (long)h[4];
    markmod = (int)h[5]; outgrid = (int)h[6]; intermod = (int)h[7]; intermod1 = (int)h[8];
    gridmod = (int)h[9]; densimod = (int)h[10]; viscmod = (int)h[11]; dynamo = (int)h[12];
    int reinject = (int)h[13];
    mnumx = h[14]; mnumy = h[15]; printmod = h[16];
    int mode = (int)h[17];
    xsize = s[0]; ysize = s[1]; timestep = s[2]; timesum = s[3];
    nubeg = s[4]; nuend = s[5]; nucontr = s[6]; tmp_ambient = s[7];
    M_init = s[8]; M_acc = s[9]; core_form_time = s[10]; k_cutoff = s[11];
    al2627_init = s[12]; fe6056_init = s[13]; relax_time = s[14]; por_init = s[15];
    eps[21] = s[16]; eps[50] = s[17]; eps[52] = s[18];
    if (marknum > MAXMRK || xnumx > MAXXLN || ynumy > MAXYLN) { fprintf(stderr, "size over reference limits\n"); return 2; }
    gridcheck();

    for (int k = 0; k < NTAB; k++) rd(type_table(k), sizeof(double), NTYPES, fi);
    int64_t im[NTYPES];
    rd(im, sizeof(int64_t), NTYPES, fi);
    for (int k = 0; k < NTYPES; k++) markim[k] = (int)im[k];
    rd(gx, sizeof(double), (size_t)xnumx, fi);
    rd(gy, sizeof(double), (size_t)ynumy, fi);
    for (int k = 0; k < 20; k++) rd(node_in(k), sizeof(double), (size_t)nodenum, fi);

    long n = marknum;
    double *buf = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *eta_in = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    int8_t *cbuf = (int8_t *)malloc((size_t)(n > 0 ? n : 1));
    long i;
    rd(buf, 8, (size_t)n, fi); for (i = 0; i < n; i++) markx[i] = buf[i];
    rd(buf, 8, (size_t)n, fi); for (i = 0; i < n; i++) marky[i] = buf[i];
    rd(buf, 8, (size_t)n, fi); for (i = 0; i < n; i++) markk[i] = buf[i];
    rd(eta_in, 8, (size_t)n, fi); for (i = 0; i < n; i++) markv[i] = eta_in[i];
    /* re-injected values are what the reference storage holds after the store */
    for (i = 0; i < n; i++) eta_in[i] = (double)markv[i];
    rd(buf, 8, (size_t)n, fi); for (i = 0; i < n; i++) markhi[i] = buf[i];
    rd(buf, 8, (size_t)n, fi); for (i = 0; i < n; i++) markpor[i] = buf[i];
    rd(buf, 8, (size_t)n, fi); for (i = 0; i < n; i++) marktmax[i] = buf[i];
    rd(markmg_time, 8, (size_t)n, fi);
    rd(cbuf, 1, (size_t)n, fi); for (i = 0; i < n; i++) markt[i] = (char)cbuf[i];
    rd(cbuf, 1, (size_t)n, fi); for (i = 0; i < n; i++) markmg_old[i] = (char)cbuf[i];
    if (mode == 1) {
        heatdif = s[19];
        rd(x, sizeof(double), (size_t)nodenum, fi); /* tk_new: the solution titerate() reads back */
    }
    if (mode == 3) rd(tk2, sizeof(double), (size_t)nodenum, fi); /* allintert()'s second field */
    if (h[24]) {
        /* grain size and accretion time (headmart.c:119-124), for the output file */
        rd(buf, 8, (size_t)n, fi); for (i = 0; i < n; i++) markgr[i] = buf[i];
        rd(buf, 8, (size_t)n, fi); for (i = 0; i < n; i++) markacc[i] = buf[i];
    }
    if (h[18]) {
        /* densimod 2: the P-T table loadmart.c:116-209 would read from mars_mantle /
         * mars_crust, given here as density and enthalpy per [tk][pb][db] node, and the
         * melting switches loadmart.c:88-90 reads from mode.t3c */
        si_melting = (int)h[19]; fe_melting = (int)h[20]; ice_melting = (int)h[21];
        tknum = (int)h[22]; pbnum = (int)h[23];
        tkmin = s[20]; pbmin = s[21]; tkstp = s[22]; pbstp = s[23];
        if (tknum < 2 || pbnum < 2 || tknum > 350 || pbnum > 350) { fprintf(stderr, "bad table size\n"); return 2; }
        double v[2];
        for (int n1 = 0; n1 < tknum; n1++)
            for (int n2 = 0; n2 < pbnum; n2++)
                for (int db = 0; db < 2; db++) {
                    rd(v, sizeof(double), 2, fi);
                    td[n1][n2][db][0] = v[0];
                    td[n1][n2][db][1] = v[1];
                }
    }
    fclose(fi);

    /* the reference prints progress inside the hot path (markmart.c:185,225,230,995) */
    if (!printmod) { if (!freopen("/dev/null", "w", stdout)) return 5; }

    double *tim = (double *)calloc((size_t)(2 * (nsteps > 0 ? nsteps : 1)), sizeof(double));
    if (mode == 1) {
        heatmod = 0;
        maxtkstep = 1e30;
        adiabyn = 0;
        frictyn = 0;
        bondv[1][0] = 0;
        bondn[1][0] = bondn[1][1] = bondn[1][2] = 0;
        for (long a = 0; a < xnumx; a++)
            for (long b = 0; b < ynumy; b++)
                bondm[nodenum3 + a * ynumy + b] = (a == 0 || b == 0 || a == xnumx - 1 || b == ynumy - 1) ? 1 : 0;
        double t0 = now_s();
        titerate(0);
        tim[0] = now_s() - t0;
        nsteps = 0;
    }
    if (mode == 2) {
        FILE *sy = fopen("stop.yn", "wt");
        if (!sy) return 5;
        fprintf(sy, "n \n");
        fclose(sy);
#ifdef I2G_DROPIN
        /* the shim's marker section of the same markers, for comparison */
        FILE *fs = fopen("shim.prn", "wb");
        if (!fs) return 5;
        i2g_shim_save_markers(fs);
        fclose(fs);
#endif
        fl1otp = 1;
        strcpy(fl1out, "out.prn");
        saver(0, 0);
        for (i = 0; i <= marknum; i++) {
            markx[i] = marky[i] = markk[i] = markv[i] = markhi[i] = markpor[i] = 0;
            markgr[i] = marktmax[i] = markacc[i] = 0;
            markt[i] = markmg_old[i] = 0;
            markmg_time[i] = 0;
        }
        fl1itp = 1;
        strcpy(fl1in, "out.prn");
        loader();
        nsteps = 0;
    }
    double *interp = NULL;
    if (mode == 3) {
        interp = (double *)malloc(sizeof(double) * (size_t)(2 * (n > 0 ? n : 1)));
        if (!interp) return 5;
        for (i = 0; i < n; i++) {
            allintert((double)(markx[i]), (double)(marky[i]));
            interp[i] = eps[2];
            interp[n + i] = eps[3];
        }
        nsteps = 0;
    }
    for (long st = 0; st < nsteps; st++) {
        double t0 = now_s();
        if (markmod && timestep) STEP_MOVE();
        double t1 = now_s();
#ifdef I2G_SHIM_RESIDENT
        /* the host writes markers: current host arrays first, the change flagged after */
        if (reinject) i2g_shim_sync_host();
#endif
        if (reinject) for (i = 0; i < marknum; i++) markv[i] = eta_in[i];
#ifdef I2G_SHIM_RESIDENT
        if (reinject) i2g_shim_markers_changed = 1;
#endif
        double t2 = now_s();
        if (gridmod) STEP_AVG();
        double t3 = now_s();
        timesum += timestep;
        tim[2 * st + 0] = t1 - t0;
        tim[2 * st + 1] = t3 - t2;
    }
#ifdef I2G_SHIM_RESIDENT
    i2g_shim_sync_host(); /* the markers the output below reads */
#endif
    /* tkrecalc() runs at the end of every ronurecalc (markmart.c:1013); time one more call alone */
    double tk0s = now_s();
    tkrecalc();
    double tkrs = now_s() - tk0s;

    FILE *fo = fopen(argv[2], "wb");
    if (!fo) return 6;
    int64_t oh[8] = {H_MAGIC, marknum, nodenum, nsteps, (int64_t)sizeof(markx[0]), mode, 0, 0};
    wr(oh, 8, 8, fo);
    n = marknum;
    for (i = 0; i < n; i++) buf[i] = (double)markx[i]; wr(buf, 8, (size_t)n, fo);
    for (i = 0; i < n; i++) buf[i] = (double)marky[i]; wr(buf, 8, (size_t)n, fo);
    for (i = 0; i < n; i++) buf[i] = (double)markk[i]; wr(buf, 8, (size_t)n, fo);
    for (i = 0; i < n; i++) buf[i] = (double)markv[i]; wr(buf, 8, (size_t)n, fo);
    for (i = 0; i < n; i++) buf[i] = (double)markp[i]; wr(buf, 8, (size_t)n, fo);
    for (i = 0; i < n; i++) buf[i] = (double)markpor[i]; wr(buf, 8, (size_t)n, fo);
    for (i = 0; i < n; i++) buf[i] = (double)marktmax[i]; wr(buf, 8, (size_t)n, fo);
    wr(markmg_time, 8, (size_t)n, fo);
    for (i = 0; i < n; i++) cbuf[i] = (int8_t)markt[i]; wr(cbuf, 1, (size_t)n, fo);
    for (i = 0; i < n; i++) cbuf[i] = (int8_t)markmg_old[i]; wr(cbuf, 1, (size_t)n, fo);
    for (int k = 0; k < 9; k++) wr(node_out(k), 8, (size_t)nodenum, fo);
    wr(tim, 8, (size_t)(2 * nsteps), fo);
    wr(&tkrs, 8, 1, fo);
    /* the melt state meltpart1() leaves for the next ronurecalc (markmart.c:287-289) */
    double melt[6] = {eps[21], eps[22], eps[50], eps[51], eps[52], eps[53]};
    wr(melt, 8, 6, fo);
    for (i = 0; i < n; i++) buf[i] = (double)markgr[i]; wr(buf, 8, (size_t)n, fo);
    for (i = 0; i < n; i++) buf[i] = (double)markacc[i]; wr(buf, 8, (size_t)n, fo);
    if (interp) wr(interp, 8, (size_t)(2 * n), fo);
    fclose(fo);
    return 0;
}
