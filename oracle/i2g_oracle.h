/*
 * TEST INFRASTRUCTURE ONLY.  Sequential CPU restatement of the I2ELVIS marker
 * step (movemark markmart.c:3-188, ronurecalc markmart.c:192-1009) used as the
 * checker for the CUDA path.  Never linked into, or called by, the product.
 */
#ifndef I2G_ORACLE_H
#define I2G_ORACLE_H
#include <stdint.h>
#include "../include/i2g.h"

typedef struct ora_grid {
    int64_t xnumx, ynumy;
    const double *gx, *gy;
    const double *vx, *vy, *pr, *exx, *eyy, *exy, *sxx, *syy, *sxy, *ga, *mu;
} ora_grid;

/* node state, updated in place (ro, nu, nd, et, cp, kt, ht, tk, po) */
typedef struct ora_nodes {
    double *ro, *nu, *nd, *et, *cp, *kt, *ht, *tk, *po;
} ora_nodes;

/* summation orders for the marker -> node sums */
#define ORA_ORDER_REFERENCE 0 /* marker storage order, as markmart.c:271-913 */
#define ORA_ORDER_CELL 1      /* per cell corner sums by marker index, then per node the cells
                                 (m1-1,m2-1),(m1-1,m2),(m1,m2-1),(m1,m2): the CUDA order */

int64_t ora_m1serch(const double *g, int64_t n, double x);
void ora_fdweight1(double x0, double x1, double xi, double *w0, double *w1);
void ora_allinterv(const i2g_params *P, const ora_grid *G, double x, double y, double *vx, double *vy);
/* e[0..7] = exy, sxy, exx, sxx, eyy, syy, pr, ga ; cell[0..1] = m10, m20 */
void ora_allintere(const i2g_params *P, const ora_grid *G, double x, double y, double *e, int64_t *cell);
double ora_viscalc(const i2g_params *P, const i2g_types *Ty, double mtk, double mpb, double hi,
                   double eii, double sii, double rii, double timesum, int mm2);
double ora_radiogenic(int mm2, double timesum, double al2627_init, double fe6056_init);

int ora_movemark(const i2g_params *P, const i2g_types *Ty, const ora_grid *G, int64_t n, double *x,
                 double *y, double *T, double *eta, double *p, const int8_t *type, const double *hi,
                 double timestep, double timesum, uint32_t flags);
/* the porosity sintering of markmart.c:362-466: the global timestep it reads,
 * markpor[] in single-precision storage (f32), and, out, whether a grain-size
 * search gave up (stuck); the magnetisation of markmart.c:651-744: markmg_old
 * and markmg_time (NULL: not produced) and mag_time, ronurecalc()'s local that
 * carries the last assigned magnetisation time from marker to marker (in/out) */
typedef struct ora_sinter_args {
    double timestep;
    int f32;
    int stuck;
    int8_t *mg_old;
    double *mg_time;
    double mag_time;
} ora_sinter_args;

/* td: the densimod 2 table (NULL otherwise); melt_state: eps[21], eps[22],
 * eps[50], eps[51], eps[52], eps[53] in and out (NULL: start from params' xmelt_*).
 * With densimod 2 the table types' marker types change in place.  sinter: NULL
 * for a timestep of 0 with FP64 porosity. */
int ora_ronurecalc(const i2g_params *P, const i2g_types *Ty, const ora_grid *G, int64_t n,
                   const double *x, const double *y, double *T, const double *eta, int8_t *type,
                   const double *hi, double *tmax, double *por, double timesum, uint32_t flags, int order,
                   const i2g_td_table *td, double *melt_state, ora_sinter_args *sinter, ora_nodes *out,
                   double *numin_numax);

/* The marker temperature update of titerate(), heatmart.c:514-697 (intermod = 0),
 * after the host's thermal solve: fluid markers (types 50..99) take the new node
 * temperature; rock markers (< 50) follow the node change, with the subgrid
 * diffusion and antidiffusion of heatdif != 0.  tk_new / tk_old: node T after /
 * before the solve; kt, cp, ro: node fields.  order: ORA_ORDER_REFERENCE sums the
 * antidiffusion node terms in marker order, ORA_ORDER_CELL in the CUDA order. */
/* allintert() (markmart.c:1687-1745, intermod = 0) at each marker: the point
 * clamped to the box, eps[2] from tk and eps[3] from tk2 (NULL: skipped) */
void ora_interp_tnode(const i2g_params *P, const ora_grid *G, int64_t n, const double *x, const double *y,
                      const double *tk, const double *tk2, double *out, double *out2);
int ora_titerate_markers(const i2g_params *P, const ora_grid *G, int64_t n, const double *x, const double *y,
                         double *T, const int8_t *type, const double *tk_new, const double *tk_old,
                         const double *kt, const double *cp, const double *ro, double heatdif, double timestep,
                         int order);

/* cell of a marker position as ronurecalc bins it (allintere clamps, markmart.c:1468-1475) */
int64_t ora_cell_key(const i2g_params *P, const ora_grid *G, double x, double y);
#endif
