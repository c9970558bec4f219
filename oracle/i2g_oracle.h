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
int ora_ronurecalc(const i2g_params *P, const i2g_types *Ty, const ora_grid *G, int64_t n,
                   const double *x, const double *y, double *T, const double *eta, const int8_t *type,
                   const double *hi, double *tmax, double *por, double timesum, uint32_t flags, int order,
                   ora_nodes *out, double *numin_numax);

/* cell of a marker position as ronurecalc bins it (allintere clamps, markmart.c:1468-1475) */
int64_t ora_cell_key(const i2g_params *P, const ora_grid *G, double x, double y);
#endif
