/* Internal declarations shared by the host C sources and the CUDA sources of libh2b200. */
#ifndef H2B200_INTERNAL_H
#define H2B200_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include "h2b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Thread-local last error (printf-style). */
void h2b_set_error(const char *fmt, ...);

/* ---------------- quadrature tables (host) ---------------- */

/* One Sauter-Schwab rule: n points; x0,x1 = reference coordinates (t, s) on the row triangle,
 * y0,y1 on the column triangle; w[10][n]: rows 0..8 basis-weighted (row basis i, column basis j at
 * row i + 3j), row 9 the raw weight. */
typedef struct {
  uint32_t n;
  double *x0, *x1, *y0, *y1;
  double *w;   /* 10 * n */
} h2b_rule;

enum { H2B_RULE_DIST = 0, H2B_RULE_VERT = 1, H2B_RULE_EDGE = 2, H2B_RULE_ID = 3 };

typedef struct {
  uint32_t q, q2;
  h2b_rule rule[4];      /* indexed by number of shared vertices: 0 dist, 1 vert, 2 edge, 3 id */
  /* single-triangle rule (q^2 points): xs, ys, ws[4][n] (rows 0..2 linear-basis weighted, 3 raw) */
  uint32_t ns;
  double *xs, *ys, *ws;
} h2b_quad;

int h2b_gauss_legendre01(uint32_t m, double *x, double *w);
int h2b_quad_build(uint32_t q, uint32_t q2, int row_basis, int col_basis, h2b_quad *out);
void h2b_quad_free(h2b_quad *qd);
/* Edge (which = 2) or identical (3) rule with the points that share a kernel argument merged:
 * (a, b, c) per point in abc[3 n'], summed basis-weighted weight rows in w9[9 n'] (malloc'ed). */
int h2b_quad_reduce(const h2b_rule *r, int which, uint32_t q2, uint32_t *n_out, double **abc,
                    double **w9);
/* Common-vertex rule in tensor form: 2 q2^2 groups of q2 row points x q2 column points. */
int h2b_quad_vert_tensor(uint32_t q2, int row_basis, int col_basis, uint32_t *ngroups,
                         double **out);
/* Common-vertex rule with the radial sum folded into moments (kernels homogeneous of degree -1
 * or -2): 2 q2^2 items of one row point and q2 column points each. */
int h2b_quad_vert_merged(uint32_t q2, int row_basis, int col_basis, uint32_t *n_out,
                         double **out);

/* ---------------- cluster / block trees (host) ---------------- */

typedef struct {
  uint32_t n;          /* number of clusters (pre-order) */
  uint32_t *off;       /* offset of the cluster's indices inside idx */
  uint32_t *size;
  uint32_t *sons;      /* number of sons (0 or 2 for adaptive bisection) */
  uint32_t *son0;      /* pre-order id of the first son (sons are consecutive subtrees) */
  uint32_t *son1;
  uint32_t *father;    /* UINT32_MAX for the root */
  uint32_t *level;
  double *bmin, *bmax; /* 3 per cluster */
  uint32_t nidx;
  uint32_t *idx;
  uint32_t depth;
} h2b_ctree;

typedef struct {
  uint32_t n;          /* number of leaf blocks, block-tree pre-order */
  uint32_t *rc, *cc;   /* cluster ids in the row / column tree */
  uint8_t *adm;        /* 1 admissible (coupling block), 0 inadmissible (nearfield block) */
} h2b_blist;

void h2b_ctree_free(h2b_ctree *t);
void h2b_blist_free(h2b_blist *b);

#ifdef __cplusplus
}
#endif

#endif
