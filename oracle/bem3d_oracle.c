/* CPU oracle for the B200 BEM path — TEST INFRASTRUCTURE ONLY (see bem3d_oracle.h).
 *
 * Restates, with plain loops in the reference's order of operations:
 *   Library/gaussquad.c:11            Gauss-Legendre rule (here: Newton on P_m)
 *   Library/singquad2d.c:25-320       Sauter-Schwab rules, :456-530 basis weights,
 *                                     :549 pair classification / vertex permutation
 *   Library/bem3d.c:1151              assemble_cc_near_bem3d
 *   Library/bem3d.c:1798/2394/3038    assemble_{cl,lc,ll}_near_bem3d
 *   Library/laplacebem3d.c:36/84/136      Laplace single / double / adjoint double layer kernels
 *   Library/helmholtzbem3d.c:27/140/209   Helmholtz single / double / adjoint double layer
 *   Library/bem3d.c:4978/5179/5236    Chebyshev points and interpolation boxes
 *   Library/bem3d.c:7555-8540         Lagrange polynomials, leaf bases (c/l, normal derivative),
 *                                     transfer matrices
 *   Library/bem3d.c:6079, :3439       coupling matrices
 *   Library/clusterbasis.c:524/749,   forward / backward transforms,
 *   Library/h2matrix.c:1211/1269      coupling + nearfield sweep, addeval
 *   Library/krylov.c:551-769,         Householder GMRES with Givens rotations,
 *   Library/krylovsolvers.c:183       restarted driver
 *   Library/factorizations.c:2179/2822 Householder QR and its application (pure-C path)
 *   Library/bem3d.c:9009/8878/8954/8704 L2 projection (linear basis), mass matvec, L2 errors
 * Nothing in the product library links this file.
 */
#include <complex.h>
#include <stdio.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "bem3d_oracle.h"

typedef double _Complex cplx;

#define INTERPOLATION_EPS 5.0e-3
#define KCONST 0.0795774715459476679

/* ------------------------------------------------------------------ quadrature */

int
orc_gauss01(uint32_t m, double *x, double *w)
{
  uint32_t i, k, it;
  if (m < 1 || m > 64)
    return -1;
  for (i = 0; i < (m + 1) / 2; i++) {
    double z = cos(M_PI * (i + 0.75) / (m + 0.5)), p0 = 1.0, p1 = 0.0, dp = 1.0;
    for (it = 0; it < 200; it++) {
      double zold = z;
      p0 = 1.0;
      p1 = z;
      for (k = 2; k <= m; k++) {
        double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (m == 1) {
        p1 = z;
        p0 = 1.0;
      }
      dp = m * (z * p1 - p0) / (z * z - 1.0);
      z = zold - p1 / dp;
      if (fabs(z - zold) < 1e-17)
        break;
    }
    {
      double ww = 2.0 / ((1.0 - z * z) * dp * dp);
      /* symmetric pair, ascending on [0,1] */
      x[i] = 0.5 - 0.5 * z;
      x[m - 1 - i] = 0.5 + 0.5 * z;
      w[i] = w[m - 1 - i] = 0.5 * ww;
    }
  }
  if (m % 2 == 1) {
    x[m / 2] = 0.5;
  }
  if (m == 1)
    w[0] = 1.0;
  return 0;
}

typedef struct {
  uint32_t n;
  double *x0, *x1, *y0, *y1, *w;
} rule_t;

static void
rule_free(rule_t *r)
{
  free(r->x0);
  free(r->x1);
  free(r->y0);
  free(r->y1);
  free(r->w);
  memset(r, 0, sizeof(*r));
}

static int
rule_make(uint32_t q, uint32_t q2, int which, rule_t *r)
{
  double g[64], gw[64];
  uint32_t qq = (which == 0) ? q : q2, n, i, j, k, l, p = 0;
  if (orc_gauss01(qq, g, gw))
    return -1;
  n = qq * qq * qq * qq * (which == 0 ? 1 : which == 1 ? 2 : 6);
  r->n = n;
  r->x0 = malloc(sizeof(double) * n);
  r->x1 = malloc(sizeof(double) * n);
  r->y0 = malloc(sizeof(double) * n);
  r->y1 = malloc(sizeof(double) * n);
  r->w = malloc(sizeof(double) * n);
  if (!r->x0 || !r->x1 || !r->y0 || !r->y1 || !r->w)
    return -1;
#define PUT(W, A, B, C, D) \
  do { r->w[p] = (W); r->x0[p] = (A); r->x1[p] = (B); r->y0[p] = (C); r->y1[p] = (D); p++; } while (0)
  for (i = 0; i < qq; i++)
    for (j = 0; j < qq; j++)
      for (k = 0; k < qq; k++)
        for (l = 0; l < qq; l++) {
          if (which == 0) {
            PUT(gw[i] * gw[j] * gw[k] * gw[l] * g[i] * g[k], g[i], g[i] * g[j], g[k], g[k] * g[l]);
          }
          else if (which == 1) {
            double e1 = g[i], e2 = g[j], e3 = g[k], xi = g[l];
            double wl = gw[l] * gw[k] * gw[j] * gw[i], ww = wl * xi * xi * xi * e1;
            PUT(ww, xi, e2 * xi, e1 * xi, e1 * e3 * xi);
            PUT(ww, e1 * xi, e1 * e3 * xi, xi, e2 * xi);
          }
          else if (which == 2) {
            double e1 = g[i], e2 = g[j], x1 = g[k], x2 = g[l] * (1.0 - x1);
            double wl = gw[l] * (gw[k] * (gw[j] * gw[i])) * (1.0 - x1), ww = wl * x1 * x1 * e1;
            PUT(ww, x1 + x2, x1 * e1 * e2, x1 * (1.0 - e1) + x2, x1 * (1.0 - e1));
            PUT(ww, x1 + x2, x1 * e1, x1 * (1.0 - e1 * e2) + x2, x1 * (1.0 - e1 * e2));
            PUT(ww, x1 + x2, x1, x1 * e1 + x2, x1 * e1 * e2);
            PUT(ww, x1 * (1.0 - e1 + e1 * e2) + x2, x1 * e1 * e2, x1 + x2, x1);
            PUT(ww, x1 * e1 * e2 + x2, x1 * e1 * e2, x1 + x2, x1 * e1);
            PUT(ww, x1 * e1 + x2, x1 * e1, x1 + x2, x1 * e1 * e2);
          }
          else {
            double eta = g[i], x1 = g[j], x2 = g[k] * (1.0 - x1), x3 = g[l] * (1.0 - x1 - x2);
            double wk = gw[k] * (gw[j] * gw[i]) * (1.0 - x1);
            double ww = gw[l] * wk * (1.0 - x1 - x2) * x1, a = x1 * (1.0 - eta);
            PUT(ww, x1 + x2 + x3, x1 + x2, a + x2 + x3, x2);
            PUT(ww, a + x2 + x3, a + x2, x1 + x2 + x3, x2);
            PUT(ww, x1 + x2 + x3, x1 * eta + x2, x2 + x3, x2);
            PUT(ww, a + x2 + x3, x2, x1 + x2 + x3, x1 + x2);
            PUT(ww, x1 + x2 + x3, x2, a + x2 + x3, a + x2);
            PUT(ww, x2 + x3, x2, x1 + x2 + x3, x1 * eta + x2);
          }
        }
#undef PUT
  return 0;
}

int
orc_rule(uint32_t q, uint32_t q2, int which, uint32_t *n, double *x0, double *x1, double *y0,
         double *y1, double *w)
{
  rule_t r;
  memset(&r, 0, sizeof(r));
  if (which < 0 || which > 3 || rule_make(q, q2, which, &r)) {
    rule_free(&r);
    return -1;
  }
  *n = r.n;
  if (x0) memcpy(x0, r.x0, sizeof(double) * r.n);
  if (x1) memcpy(x1, r.x1, sizeof(double) * r.n);
  if (y0) memcpy(y0, r.y0, sizeof(double) * r.n);
  if (y1) memcpy(y1, r.y1, sizeof(double) * r.n);
  if (w) memcpy(w, r.w, sizeof(double) * r.n);
  rule_free(&r);
  return 0;
}

/* single-triangle rule: xs = g_i, ys = g_i g_j, ws = w_i w_j g_i */
static int
single_rule(uint32_t q, double *xs, double *ys, double *ws)
{
  double g[64], gw[64];
  uint32_t i, j, p = 0;
  if (orc_gauss01(q, g, gw))
    return -1;
  for (i = 0; i < q; i++)
    for (j = 0; j < q; j++) {
      ws[p] = gw[i] * gw[j] * g[i];
      xs[p] = g[i];
      ys[p] = g[i] * g[j];
      p++;
    }
  return 0;
}

/* ------------------------------------------------------------------ operator */

typedef struct {
  uint32_t nv, nt;
  const double *x, *n, *g;
  const uint32_t *t;
  int pde, layer, rb, cb;
  double k_re, k_imn;   /* -Im k, as in the reference kernels */
  cplx alpha;
  rule_t rule[4];
  uint32_t ns;
  double xs[64 * 64], ys[64 * 64], ws[64 * 64];
  double mass[9];
  uint32_t *v2t_off, *v2t;
} op_t;

static void
op_free(op_t *o)
{
  int i;
  for (i = 0; i < 4; i++)
    rule_free(&o->rule[i]);
  free(o->v2t_off);
  free(o->v2t);
}

static int
op_init(op_t *o, uint32_t nv, const double *x, uint32_t nt, const uint32_t *t, const double *n,
        const double *g, int pde, int layer, int rb, int cb, uint32_t q, uint32_t q2,
        double k_re, double k_im, double a_re, double a_im)
{
  uint32_t i, k, *fill;
  int c;
  memset(o, 0, sizeof(*o));
  o->nv = nv; o->nt = nt; o->x = x; o->t = t; o->n = n; o->g = g;
  o->pde = pde; o->layer = layer; o->rb = rb; o->cb = cb;
  o->k_re = k_re; o->k_imn = -k_im;
  o->alpha = a_re + a_im * I;
  for (c = 0; c < 4; c++)
    if (rule_make(q, q2, c, &o->rule[c]))
      return -1;
  o->ns = q * q;
  if (single_rule(q, o->xs, o->ys, o->ws))
    return -1;
  for (i = 0; i < 9; i++)
    o->mass[i] = 0.0;
  if (rb == ORC_BASIS_LINEAR && cb == ORC_BASIS_LINEAR)
    for (i = 0; i < 9; i++)
      o->mass[i] = (i % 4 == 0) ? 1.0 / 12.0 : 1.0 / 24.0;
  else if (rb != cb)
    for (i = 0; i < 3; i++)
      o->mass[i] = 1.0 / 6.0;
  o->v2t_off = calloc(nv + 1, sizeof(uint32_t));
  o->v2t = malloc(sizeof(uint32_t) * 3 * nt);
  fill = malloc(sizeof(uint32_t) * (nv + 1));
  if (!o->v2t_off || !o->v2t || !fill) {
    free(fill);
    return -1;
  }
  for (i = 0; i < nt; i++)
    for (k = 0; k < 3; k++)
      o->v2t_off[t[3 * i + k] + 1]++;
  for (i = 0; i < nv; i++)
    o->v2t_off[i + 1] += o->v2t_off[i];
  memcpy(fill, o->v2t_off, sizeof(uint32_t) * (nv + 1));
  for (i = 0; i < nt; i++)
    for (k = 0; k < 3; k++)
      o->v2t[fill[t[3 * i + k]]++] = i;
  free(fill);
  return 0;
}

/* kernel at (x, y) with row normal nx and column normal ny; layer 0 single, 1 double, 2 adjoint
 * double layer (Library/laplacebem3d.c:36/84/136, Library/helmholtzbem3d.c:27/140/209) */
static cplx
kernel(const op_t *o, const double *xx, const double *yy, const double *nx, const double *ny)
{
  double d[3] = {xx[0] - yy[0], xx[1] - yy[1], xx[2] - yy[2]};
  double n2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  double rn = 1.0 / sqrt(n2), dot = 0.0;
  if (o->layer == 1)
    dot = d[0] * ny[0] + d[1] * ny[1] + d[2] * ny[2];
  else if (o->layer == 2)  /* <y - x, n_x> */
    dot = (yy[0] - xx[0]) * nx[0] + (yy[1] - xx[1]) * nx[1] + (yy[2] - xx[2]) * nx[2];
  if (o->pde == 0) {
    if (o->layer == 0)
      return rn;
    rn = rn * rn * rn;
    return dot * rn;
  }
  if (o->layer == 0) {
    double norm = n2 * rn;
    if (o->k_imn != 0.0)
      rn *= exp(o->k_imn * norm);
    norm = o->k_re * norm;
    return rn * cos(norm) + (sin(norm) * rn) * I;
  }
  {
    double re = (rn * rn * rn) * dot;
    double norm = n2 * rn, s, c;
    if (o->k_imn != 0.0)
      re *= exp(o->k_imn * norm);
    norm = o->k_re * norm;
    s = sin(norm);
    c = cos(norm);
    return (c + norm * s) * re + ((s - c * norm) * re) * I;
  }
}

/* Classification and permutation (shared vertices first, in the row triangle's order). */
static uint32_t
select_quad(const uint32_t *tv, const uint32_t *sv, uint32_t *tp, uint32_t *sp)
{
  uint32_t p = 0, i, j, q, c;
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++)
      p += tv[i] == sv[j];
  for (i = 0; i < 3; i++)
    tp[i] = sp[i] = i;
  if (p == 0 || p >= 3)
    return p > 3 ? 3 : p;
  c = 0;
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++)
      if (tv[i] == sv[j]) {
        tp[c] = i;
        sp[c] = j;
        c++;
        break;
      }
  q = c;
  for (i = 0; i < 3; i++) {
    for (j = 0; j < q && tv[i] != tv[tp[j]]; j++);
    if (j == q) tp[q++] = i;
  }
  q = c;
  for (i = 0; i < 3; i++) {
    for (j = 0; j < q && sv[i] != sv[sp[j]]; j++);
    if (j == q) sp[q++] = i;
  }
  return p;
}

static double
nodal(int lin, int i, double a, double b)
{
  if (!lin)
    return 1.0;
  return i == 0 ? 1.0 - a : (i == 1 ? a - b : b);
}

/* 3x3 (or fewer) weighted integrals of one triangle pair; res[l + 3k] for permuted local row
 * basis l, column basis k; tp/sp returned. */
static void
pair_integrals(const op_t *o, uint32_t tt, uint32_t ss, cplx *res, uint32_t *tp, uint32_t *sp)
{
  const uint32_t *tv = o->t + 3 * (size_t) tt, *sv = o->t + 3 * (size_t) ss;
  uint32_t c = select_quad(tv, sv, tp, sp), q, l, k;
  const rule_t *r = &o->rule[c];
  const double *At = o->x + 3 * (size_t) tv[tp[0]], *Bt = o->x + 3 * (size_t) tv[tp[1]],
               *Ct = o->x + 3 * (size_t) tv[tp[2]];
  const double *As = o->x + 3 * (size_t) sv[sp[0]], *Bs = o->x + 3 * (size_t) sv[sp[1]],
               *Cs = o->x + 3 * (size_t) sv[sp[2]];
  const double *nx = o->n + 3 * (size_t) tt, *ny = o->n + 3 * (size_t) ss;
  int rl = o->rb == ORC_BASIS_LINEAR, cl = o->cb == ORC_BASIS_LINEAR;
  for (l = 0; l < 9; l++)
    res[l] = 0.0;
  for (q = 0; q < r->n; q++) {
    double tx = r->x0[q], sx = r->x1[q], ty = r->y0[q], sy = r->y1[q];
    double Ax = 1.0 - tx, Bx = tx - sx, Cx = sx, Ay = 1.0 - ty, By = ty - sy, Cy = sy;
    double xx[3], yy[3];
    cplx kv;
    int d;
    for (d = 0; d < 3; d++) {
      xx[d] = At[d] * Ax + Bt[d] * Bx + Ct[d] * Cx;
      yy[d] = As[d] * Ay + Bs[d] * By + Cs[d] * Cy;
    }
    kv = kernel(o, xx, yy, nx, ny);
    for (k = 0; k < (cl ? 3u : 1u); k++)
      for (l = 0; l < (rl ? 3u : 1u); l++)
        res[l + 3 * k] += (r->w[q] * nodal(rl, l, tx, sx) * nodal(cl, k, ty, sy)) * kv;
  }
}

static void
put(double *N, int cplxout, uint64_t idx, cplx v, int add)
{
  if (cplxout) {
    if (add) {
      N[2 * idx] += creal(v);
      N[2 * idx + 1] += cimag(v);
    }
    else {
      N[2 * idx] = creal(v);
      N[2 * idx + 1] = cimag(v);
    }
  }
  else {
    if (add)
      N[idx] += creal(v);
    else
      N[idx] = creal(v);
  }
}

/* Entry-by-entry fill of a block into N (column-major, ld). */
static int
op_nearfield(const op_t *o, const uint32_t *ridx, uint32_t rows, const uint32_t *cidx,
             uint32_t cols, int ntrans, double *N, uint64_t ld)
{
  int rl = o->rb == ORC_BASIS_LINEAR, cl = o->cb == ORC_BASIS_LINEAR, cx = o->pde == 1;
  uint32_t i, j;
  int32_t *rloc = NULL, *cloc = NULL;
  uint32_t *rt = NULL, *ct = NULL, nrt = 0, nct = 0;
  uint8_t *seen;
  uint32_t nr_all = rl ? o->nv : o->nt, nc_all = cl ? o->nv : o->nt;

  /* clear the block */
  for (j = 0; j < (ntrans ? rows : cols); j++)
    for (i = 0; i < (ntrans ? cols : rows); i++)
      put(N, cx, i + (uint64_t) j * ld, 0.0, 0);

  /* local indices and the triangles touching each side */
  rloc = malloc(sizeof(int32_t) * nr_all);
  cloc = malloc(sizeof(int32_t) * nc_all);
  rt = malloc(sizeof(uint32_t) * o->nt);
  ct = malloc(sizeof(uint32_t) * o->nt);
  seen = calloc(o->nt, 1);
  if (!rloc || !cloc || !rt || !ct || !seen)
    return -1;
  for (i = 0; i < nr_all; i++) rloc[i] = -1;
  for (i = 0; i < nc_all; i++) cloc[i] = -1;
  for (i = 0; i < rows; i++) rloc[ridx ? ridx[i] : i] = (int32_t) i;
  for (i = 0; i < cols; i++) cloc[cidx ? cidx[i] : i] = (int32_t) i;
  for (i = 0; i < rows; i++) {
    uint32_t v = ridx ? ridx[i] : i, a;
    if (!rl) { rt[nrt++] = v; continue; }
    for (a = o->v2t_off[v]; a < o->v2t_off[v + 1]; a++)
      if (!(seen[o->v2t[a]] & 1)) { seen[o->v2t[a]] |= 1; rt[nrt++] = o->v2t[a]; }
  }
  for (i = 0; i < cols; i++) {
    uint32_t v = cidx ? cidx[i] : i, a;
    if (!cl) { ct[nct++] = v; continue; }
    for (a = o->v2t_off[v]; a < o->v2t_off[v + 1]; a++)
      if (!(seen[o->v2t[a]] & 2)) { seen[o->v2t[a]] |= 2; ct[nct++] = o->v2t[a]; }
  }

  for (j = 0; j < nct; j++) {
    uint32_t ss = ct[j];
    for (i = 0; i < nrt; i++) {
      uint32_t tt = rt[i], tp[3], sp[3], l, k;
      cplx res[9], f2 = (o->g[ss] * KCONST) * o->g[tt];
      pair_integrals(o, tt, ss, res, tp, sp);
      for (k = 0; k < (cl ? 3u : 1u); k++) {
        int32_t lc = cl ? cloc[o->t[3 * (size_t) ss + sp[k]]] : cloc[ss];
        if (lc < 0) continue;
        for (l = 0; l < (rl ? 3u : 1u); l++) {
          int32_t lr = rl ? rloc[o->t[3 * (size_t) tt + tp[l]]] : rloc[tt];
          cplx v = res[l + 3 * k] * f2;
          if (lr < 0) continue;
          if (ntrans)
            put(N, cx, (uint64_t) lc + (uint64_t) lr * ld, conj(v), 1);
          else
            put(N, cx, (uint64_t) lr + (uint64_t) lc * ld, v, 1);
        }
      }
      if (tt == ss && o->alpha != 0.0) {
        if (!rl && !cl) {
          int32_t lr = rloc[tt], lc = cloc[ss];
          cplx v = 0.5 * o->alpha * o->g[tt];
          if (ntrans)
            put(N, cx, (uint64_t) lc + (uint64_t) lr * ld, conj(v), 1);
          else
            put(N, cx, (uint64_t) lr + (uint64_t) lc * ld, v, 1);
        }
        else {
          /* mixed bases: mass[i] = 1/6 for the linear side's local function i
           * (Library/bem3d.c:1936-1963 and the lc counterpart) */
          for (k = 0; k < (cl ? 3u : 1u); k++)
            for (l = 0; l < (rl ? 3u : 1u); l++) {
              int32_t lr = rl ? rloc[o->t[3 * (size_t) tt + l]] : rloc[tt];
              int32_t lc = cl ? cloc[o->t[3 * (size_t) ss + k]] : cloc[ss];
              double m = (rl && cl) ? o->mass[l + 3 * k] : o->mass[rl ? l : k];
              cplx v = m * (o->alpha * o->g[tt]);
              if (lr < 0 || lc < 0) continue;
              if (ntrans)
                put(N, cx, (uint64_t) lc + (uint64_t) lr * ld, conj(v), 1);
              else
                put(N, cx, (uint64_t) lr + (uint64_t) lc * ld, v, 1);
            }
        }
      }
    }
  }
  free(rloc); free(cloc); free(rt); free(ct); free(seen);
  return 0;
}

int
orc_nearfield(uint32_t nv, const double *x, uint32_t nt, const uint32_t *t, const double *n,
              const double *g, int pde, int layer, int row_basis, int col_basis, uint32_t q,
              uint32_t q2, double k_re, double k_im, double alpha_re, double alpha_im,
              const uint32_t *ridx, uint32_t rows, const uint32_t *cidx, uint32_t cols,
              int ntrans, double *N, uint64_t ld)
{
  op_t o;
  int rc;
  if (op_init(&o, nv, x, nt, t, n, g, pde, layer, row_basis, col_basis, q, q2, k_re, k_im,
              alpha_re, alpha_im)) {
    op_free(&o);
    return -1;
  }
  rc = op_nearfield(&o, ridx, rows, cidx, cols, ntrans, N, ld);
  op_free(&o);
  return rc;
}

/* ------------------------------------------------------------------ interpolation */

static double
lagr1(double x, const double *xi, uint32_t mu, uint32_t m)
{
  double v = 1.0;
  uint32_t l;
  for (l = 0; l < mu; l++) v *= (x - xi[l]) / (xi[mu] - xi[l]);
  for (l = mu + 1; l < m; l++) v *= (x - xi[l]) / (xi[mu] - xi[l]);
  return v;
}

static double
dlagr1(double x, const double *xi, uint32_t mu, uint32_t m)
{
  double s = 0.0;
  uint32_t l, l2;
  for (l = 0; l < m; l++) {
    double tmp = 1.0;
    if (l == mu) continue;
    for (l2 = 0; l2 < m; l2++) {
      if (l2 == mu || l2 == l) continue;
      tmp *= (x - xi[l2]) / (xi[mu] - xi[l2]);
    }
    s += tmp / (xi[mu] - xi[l]);
  }
  return s;
}

/* 1D interpolation points of a box (Library/bem3d.c:5236) */
static void
box_points(const double *bmin, const double *bmax, const double *cheb, uint32_t m,
           double *px, double *py, double *pz)
{
  double a[3], b[3];
  uint32_t d, i;
  for (d = 0; d < 3; d++) {
    a[d] = bmin[d];
    b[d] = bmax[d];
    if (b[d] - a[d] < INTERPOLATION_EPS) {
      b[d] += INTERPOLATION_EPS;
      a[d] -= INTERPOLATION_EPS;
    }
  }
  for (i = 0; i < m; i++) {
    px[i] = (b[0] + a[0]) * 0.5 + (b[0] - a[0]) * 0.5 * cheb[i];
    py[i] = (b[1] + a[1]) * 0.5 + (b[1] - a[1]) * 0.5 * cheb[i];
    pz[i] = (b[2] + a[2]) * 0.5 + (b[2] - a[2]) * 0.5 * cheb[i];
  }
}

/* ------------------------------------------------------------------ H2 matrix */

typedef struct {
  uint32_t n;
  uint32_t *off, *size, *sons, *son0, *son1, *father;
  double *box;
  uint32_t nidx;
  const uint32_t *idx;
  /* per cluster: offset of its V (leaves) / E (non-root) in the storage */
  uint64_t *voff, *eoff;
  cplx *V, *E;
} ctree_t;

struct orc_h2 {
  op_t op;
  uint32_t m, k;
  double cheb[32];
  ctree_t rt, ct;
  uint32_t nb;
  uint32_t *brc, *bcc;
  uint8_t *badm;
  uint64_t *boff;   /* offset of each block's S or N */
  cplx *S, *N;
};

static void
ctree_free(ctree_t *c)
{
  free(c->off); free(c->size); free(c->sons); free(c->son0); free(c->son1); free(c->father);
  free(c->box); free(c->voff); free(c->eoff); free(c->V); free(c->E);
}

static int
ctree_init(ctree_t *c, uint32_t nc, const uint32_t *rec, const double *box, uint32_t n,
           const uint32_t *idx)
{
  uint32_t i, *stack, sp = 0;
  memset(c, 0, sizeof(*c));
  c->n = nc;
  c->nidx = n;
  c->idx = idx;
  c->off = malloc(4 * nc); c->size = malloc(4 * nc); c->sons = malloc(4 * nc);
  c->son0 = malloc(4 * nc); c->son1 = malloc(4 * nc); c->father = malloc(4 * nc);
  c->box = malloc(sizeof(double) * 6 * nc);
  c->voff = calloc(nc, 8); c->eoff = calloc(nc, 8);
  stack = malloc(4 * (nc + 1));
  if (!c->off || !c->size || !c->sons || !c->son0 || !c->son1 || !c->father || !c->box
      || !c->voff || !c->eoff || !stack) {
    free(stack);
    return -1;
  }
  memcpy(c->box, box, sizeof(double) * 6 * nc);
  for (i = 0; i < nc; i++) {
    c->off[i] = rec[3 * i];
    c->size[i] = rec[3 * i + 1];
    c->sons[i] = rec[3 * i + 2];
    c->son0[i] = c->son1[i] = c->father[i] = UINT32_MAX;
  }
  for (i = 0; i < nc; i++) {
    if (i > 0) {
      while (sp > 0) {
        uint32_t f = stack[sp - 1];
        if ((c->son0[f] != UINT32_MAX) + (c->son1[f] != UINT32_MAX) < c->sons[f]) break;
        sp--;
      }
      if (sp == 0) { free(stack); return -1; }
      if (c->son0[stack[sp - 1]] == UINT32_MAX) c->son0[stack[sp - 1]] = i;
      else c->son1[stack[sp - 1]] = i;
      c->father[i] = stack[sp - 1];
    }
    if (c->sons[i]) stack[sp++] = i;
  }
  free(stack);
  return 0;
}

/* Leaf basis of cluster c: V[i, nu] (size x k, column-major), row basis or column basis
 * (dn selects the normal-derivative version: the double layer's column side, the adjoint double
 * layer's row side). */
static void
leaf_basis(const orc_h2 *h, const ctree_t *c, uint32_t cid, int linear, int dn, cplx *V)
{
  const op_t *o = &h->op;
  uint32_t m = h->m, k = h->k, size = c->size[cid], jx, jy, jz, q, i, nu;
  const uint32_t *idx = c->idx + c->off[cid];
  double px[32], py[32], pz[32];
  box_points(c->box + 6 * cid, c->box + 6 * cid + 3, h->cheb, m, px, py, pz);
  for (i = 0; i < size * k; i++)
    V[i] = 0.0;
  if (!linear) {
    for (i = 0; i < size; i++) {
      uint32_t tt = idx[i];
      const uint32_t *tv = o->t + 3 * (size_t) tt;
      const double *A = o->x + 3 * (size_t) tv[0], *B = o->x + 3 * (size_t) tv[1],
                   *C = o->x + 3 * (size_t) tv[2], *nt = o->n + 3 * (size_t) tt;
      nu = 0;
      for (jx = 0; jx < m; jx++)
        for (jy = 0; jy < m; jy++)
          for (jz = 0; jz < m; jz++, nu++) {
            double sum = 0.0;
            for (q = 0; q < o->ns; q++) {
              double tx = o->xs[q], sx = o->ys[q], X[3];
              int d;
              for (d = 0; d < 3; d++)
                X[d] = A[d] * (1.0 - tx) + B[d] * (tx - sx) + C[d] * sx;
              if (!dn) {
                sum += o->ws[q] * (lagr1(X[0], px, jx, m) * lagr1(X[1], py, jy, m)
                                   * lagr1(X[2], pz, jz, m));
              }
              else {
                double lx = lagr1(X[0], px, jx, m), ly = lagr1(X[1], py, jy, m),
                       lz = lagr1(X[2], pz, jz, m);
                double g0 = dlagr1(X[0], px, jx, m) * ly * lz, g1 = lx * dlagr1(X[1], py, jy, m) * lz,
                       g2 = lx * ly * dlagr1(X[2], pz, jz, m);
                sum += o->ws[q] * (nt[0] * g0 + nt[1] * g1 + nt[2] * g2);
              }
            }
            V[i + (size_t) nu * size] = o->g[tt] * sum;
          }
    }
  }
  else {
    /* vertex-local lookup */
    int32_t *loc = malloc(sizeof(int32_t) * o->nv);
    uint8_t *seen = calloc(o->nt, 1);
    for (i = 0; i < o->nv; i++) loc[i] = -1;
    for (i = 0; i < size; i++) loc[idx[i]] = (int32_t) i;
    for (i = 0; i < size; i++) {
      uint32_t v = idx[i], a;
      for (a = o->v2t_off[v]; a < o->v2t_off[v + 1]; a++) {
        uint32_t ss = o->v2t[a], l;
        const uint32_t *sv;
        const double *A, *B, *C, *ns;
        if (seen[ss]) continue;
        seen[ss] = 1;
        sv = o->t + 3 * (size_t) ss;
        A = o->x + 3 * (size_t) sv[0]; B = o->x + 3 * (size_t) sv[1]; C = o->x + 3 * (size_t) sv[2];
        ns = o->n + 3 * (size_t) ss;
        nu = 0;
        for (jx = 0; jx < m; jx++)
          for (jy = 0; jy < m; jy++)
            for (jz = 0; jz < m; jz++, nu++) {
              double quad[64 * 64];
              for (q = 0; q < o->ns; q++) {
                double tx = o->xs[q], sx = o->ys[q], X[3];
                int d;
                for (d = 0; d < 3; d++)
                  X[d] = A[d] * (1.0 - tx) + B[d] * (tx - sx) + C[d] * sx;
                if (!dn)
                  quad[q] = lagr1(X[0], px, jx, m) * lagr1(X[1], py, jy, m) * lagr1(X[2], pz, jz, m);
                else {
                  double lx = lagr1(X[0], px, jx, m), ly = lagr1(X[1], py, jy, m),
                         lz = lagr1(X[2], pz, jz, m);
                  quad[q] = ns[0] * dlagr1(X[0], px, jx, m) * ly * lz
                            + ns[1] * lx * dlagr1(X[1], py, jy, m) * lz
                            + ns[2] * lx * ly * dlagr1(X[2], pz, jz, m);
                }
              }
              for (l = 0; l < 3; l++) {
                int32_t li = loc[sv[l]];
                double sum = 0.0;
                if (li < 0) continue;
                for (q = 0; q < o->ns; q++)
                  sum += (o->ws[q] * nodal(1, l, o->xs[q], o->ys[q])) * quad[q];
                V[li + (size_t) nu * size] += sum * o->g[ss];
              }
            }
      }
    }
    free(loc);
    free(seen);
  }
}

/* Transfer matrix of son s: E[i, nu] = L^father_nu(xi^son_i) (k x k). */
static void
transfer(const orc_h2 *h, const ctree_t *c, uint32_t son, cplx *E)
{
  uint32_t m = h->m, k = h->k, f = c->father[son], i, jx, jy, jz, nu = 0;
  double fx[32], fy[32], fz[32], sx[32], sy[32], sz[32];
  box_points(c->box + 6 * f, c->box + 6 * f + 3, h->cheb, m, fx, fy, fz);
  box_points(c->box + 6 * son, c->box + 6 * son + 3, h->cheb, m, sx, sy, sz);
  for (jx = 0; jx < m; jx++)
    for (jy = 0; jy < m; jy++)
      for (jz = 0; jz < m; jz++, nu++) {
        uint32_t a, b, cc;
        i = 0;
        for (a = 0; a < m; a++)
          for (b = 0; b < m; b++)
            for (cc = 0; cc < m; cc++, i++)
              E[i + (size_t) nu * k] = lagr1(sx[a], fx, jx, m) * lagr1(sy[b], fy, jy, m)
                                       * lagr1(sz[cc], fz, jz, m);
      }
}

static void
coupling(const orc_h2 *h, uint32_t r, uint32_t c, cplx *S)
{
  uint32_t m = h->m, k = h->k, i, j;
  double rx[32], ry[32], rz[32], cx[32], cy[32], cz[32];
  double (*X)[3] = malloc(sizeof(double) * 3 * k), (*Y)[3] = malloc(sizeof(double) * 3 * k);
  op_t slp = h->op;
  slp.layer = 0;
  box_points(h->rt.box + 6 * r, h->rt.box + 6 * r + 3, h->cheb, m, rx, ry, rz);
  box_points(h->ct.box + 6 * c, h->ct.box + 6 * c + 3, h->cheb, m, cx, cy, cz);
  {
    uint32_t a, b, d, p = 0;
    for (a = 0; a < m; a++)
      for (b = 0; b < m; b++)
        for (d = 0; d < m; d++, p++) {
          X[p][0] = rx[a]; X[p][1] = ry[b]; X[p][2] = rz[d];
          Y[p][0] = cx[a]; Y[p][1] = cy[b]; Y[p][2] = cz[d];
        }
  }
  for (j = 0; j < k; j++)
    for (i = 0; i < k; i++)
      S[i + (size_t) j * k] = KCONST * kernel(&slp, X[i], Y[j], NULL, NULL);
  free(X);
  free(Y);
}

static int
build_basis(orc_h2 *h, ctree_t *c, int linear, int dn)
{
  uint64_t vtot = 0, etot = 0;
  uint32_t i;
  for (i = 0; i < c->n; i++) {
    if (c->sons[i] == 0) { c->voff[i] = vtot; vtot += (uint64_t) c->size[i] * h->k; }
    if (i > 0) { c->eoff[i] = etot; etot += (uint64_t) h->k * h->k; }
  }
  c->V = malloc(sizeof(cplx) * (vtot + 1));
  c->E = malloc(sizeof(cplx) * (etot + 1));
  if (!c->V || !c->E) return -1;
  for (i = 0; i < c->n; i++) {
    if (c->sons[i] == 0) leaf_basis(h, c, i, linear, dn, c->V + c->voff[i]);
    if (i > 0) transfer(h, c, i, c->E + c->eoff[i]);
  }
  return 0;
}

orc_h2 *
orc_h2_new(uint32_t nv, const double *x, uint32_t nt, const uint32_t *t, const double *n,
           const double *g, int pde, int layer, int row_basis, int col_basis, uint32_t q,
           uint32_t q2, double k_re, double k_im, double alpha_re, double alpha_im, uint32_t m,
           uint32_t rnc, const uint32_t *rrec, const double *rbox, uint32_t rn,
           const uint32_t *ridx, uint32_t cnc, const uint32_t *crec, const double *cbox,
           uint32_t cn, const uint32_t *cidx, uint32_t nb, const uint32_t *brc,
           const uint32_t *bcc, const uint8_t *badm)
{
  orc_h2 *h = calloc(1, sizeof(orc_h2));
  uint64_t stot = 0, ntot = 0;
  uint32_t i, b;
  if (!h || m < 1 || m > 32) { free(h); return NULL; }
  if (op_init(&h->op, nv, x, nt, t, n, g, pde, layer, row_basis, col_basis, q, q2, k_re, k_im,
              alpha_re, alpha_im)) goto fail;
  h->m = m;
  h->k = m * m * m;
  for (i = 0; i < m; i++)
    h->cheb[i] = cos(M_PI * (2.0 * i * (1.0 / (2.0 * m)) + (1.0 / (2.0 * m))));
  if (ctree_init(&h->rt, rnc, rrec, rbox, rn, ridx) || ctree_init(&h->ct, cnc, crec, cbox, cn, cidx))
    goto fail;
  h->nb = nb;
  h->brc = malloc(4 * nb); h->bcc = malloc(4 * nb); h->badm = malloc(nb);
  h->boff = malloc(8 * nb);
  if (!h->brc || !h->bcc || !h->badm || !h->boff) goto fail;
  memcpy(h->brc, brc, 4 * nb); memcpy(h->bcc, bcc, 4 * nb); memcpy(h->badm, badm, nb);
  /* row basis: normal derivative for the adjoint double layer operator; column basis: normal
   * derivative for the double layer operator (assemble_bem3d_dn_lagrange_*) */
  if (build_basis(h, &h->rt, row_basis == ORC_BASIS_LINEAR, layer == 2)
      || build_basis(h, &h->ct, col_basis == ORC_BASIS_LINEAR, layer == 1)) goto fail;
  for (b = 0; b < nb; b++) {
    if (badm[b]) { h->boff[b] = stot; stot += (uint64_t) h->k * h->k; }
    else { h->boff[b] = ntot; ntot += (uint64_t) h->rt.size[brc[b]] * h->ct.size[bcc[b]]; }
  }
  h->S = malloc(sizeof(cplx) * (stot + 1));
  h->N = malloc(sizeof(cplx) * (ntot + 1));
  if (!h->S || !h->N) goto fail;
  for (b = 0; b < nb; b++) {
    uint32_t r = brc[b], c = bcc[b];
    if (badm[b]) {
      coupling(h, r, c, h->S + h->boff[b]);
    }
    else {
      uint32_t rows = h->rt.size[r], cols = h->ct.size[c];
      double *tmp = malloc(sizeof(double) * 2 * ((size_t) rows * cols + 1));
      uint64_t e;
      if (!tmp) goto fail;
      op_nearfield(&h->op, h->rt.idx + h->rt.off[r], rows, h->ct.idx + h->ct.off[c], cols, 0, tmp,
                   rows);
      for (e = 0; e < (uint64_t) rows * cols; e++)
        h->N[h->boff[b] + e] = pde == 1 ? tmp[2 * e] + tmp[2 * e + 1] * I : tmp[e];
      free(tmp);
    }
  }
  return h;
fail:
  orc_h2_del(h);
  return NULL;
}

void
orc_h2_del(orc_h2 *h)
{
  if (!h) return;
  op_free(&h->op);
  ctree_free(&h->rt);
  ctree_free(&h->ct);
  free(h->brc); free(h->bcc); free(h->badm); free(h->boff); free(h->S); free(h->N);
  free(h);
}

int
orc_h2_export(const orc_h2 *h, int part, uint32_t count, double *out, uint64_t *ndoubles)
{
  int cx = h->op.pde == 1;
  uint64_t pos = 0;
  uint32_t i, got = 0;
  const ctree_t *c = (part == 0 || part == 1) ? &h->rt : &h->ct;
#define EMIT(src, len)                                                           \
  do {                                                                         \
    uint64_t e_;                                                               \
    for (e_ = 0; e_ < (len); e_++) {                                           \
      if (out) {                                                               \
        if (cx) { out[2 * (pos + e_)] = creal((src)[e_]); out[2 * (pos + e_) + 1] = cimag((src)[e_]); } \
        else out[pos + e_] = creal((src)[e_]);                                 \
      }                                                                        \
    }                                                                          \
    pos += (len);                                                              \
  } while (0)
  if (part == 0 || part == 2) {
    for (i = 0; i < c->n && got < count; i++)
      if (c->sons[i] == 0) { EMIT(c->V + c->voff[i], (uint64_t) c->size[i] * h->k); got++; }
  }
  else if (part == 1 || part == 3) {
    for (i = 1; i < c->n && got < count; i++) { EMIT(c->E + c->eoff[i], (uint64_t) h->k * h->k); got++; }
  }
  else if (part == 4 || part == 5) {
    for (i = 0; i < h->nb && got < count; i++) {
      if ((part == 4) != (h->badm[i] != 0)) continue;
      if (part == 4) EMIT(h->S + h->boff[i], (uint64_t) h->k * h->k);
      else EMIT(h->N + h->boff[i], (uint64_t) h->rt.size[h->brc[i]] * h->ct.size[h->bcc[i]]);
      got++;
    }
  }
  else return -1;
#undef EMIT
  *ndoubles = cx ? 2 * pos : pos;
  return 0;
}

/* forward transform on cluster i (recursive), xt = k coefficients per cluster */
static void
forward(const orc_h2 *h, const ctree_t *c, uint32_t i, const cplx *x, cplx *xt)
{
  uint32_t k = h->k, a, b;
  cplx *xc = xt + (size_t) i * k;
  for (a = 0; a < k; a++) xc[a] = 0.0;
  if (c->sons[i]) {
    uint32_t s[2] = {c->son0[i], c->son1[i]}, j;
    for (j = 0; j < 2; j++) {
      const cplx *E = c->E + c->eoff[s[j]], *xs = xt + (size_t) s[j] * k;
      forward(h, c, s[j], x, xt);
      /* xc += E^H xs  (mvm with trans) */
      for (b = 0; b < k; b++) {
        cplx sum = 0.0;
        for (a = 0; a < k; a++) sum += conj(E[a + (size_t) b * k]) * xs[a];
        xc[b] += sum;
      }
    }
  }
  else {
    const cplx *V = c->V + c->voff[i];
    uint32_t size = c->size[i];
    for (b = 0; b < k; b++) {
      cplx sum = 0.0;
      for (a = 0; a < size; a++) sum += conj(V[a + (size_t) b * size]) * x[c->idx[c->off[i] + a]];
      xc[b] += sum;
    }
  }
}

static void
backward(const orc_h2 *h, const ctree_t *c, uint32_t i, cplx *yt, cplx *y)
{
  uint32_t k = h->k, a, b;
  cplx *yc = yt + (size_t) i * k;
  if (c->sons[i]) {
    uint32_t s[2] = {c->son0[i], c->son1[i]}, j;
    for (j = 0; j < 2; j++) {
      const cplx *E = c->E + c->eoff[s[j]];
      cplx *ys = yt + (size_t) s[j] * k;
      for (b = 0; b < k; b++)
        for (a = 0; a < k; a++) ys[a] += E[a + (size_t) b * k] * yc[b];
      backward(h, c, s[j], yt, y);
    }
  }
  else {
    const cplx *V = c->V + c->voff[i];
    uint32_t size = c->size[i];
    for (a = 0; a < size; a++) {
      cplx sum = 0.0;
      for (b = 0; b < k; b++) sum += V[a + (size_t) b * size] * yc[b];
      y[c->idx[c->off[i] + a]] += sum;
    }
  }
}

static void
h2_apply(const orc_h2 *h, cplx alpha, const cplx *x, cplx *y)
{
  uint32_t k = h->k, b, i, j;
  cplx *xt = calloc((size_t) h->ct.n * k, sizeof(cplx));
  cplx *yt = calloc((size_t) h->rt.n * k, sizeof(cplx));
  forward(h, &h->ct, 0, x, xt);
  for (b = 0; b < h->nb; b++) {
    uint32_t r = h->brc[b], c = h->bcc[b];
    if (h->badm[b]) {
      const cplx *S = h->S + h->boff[b];
      for (j = 0; j < k; j++)
        for (i = 0; i < k; i++)
          yt[(size_t) r * k + i] += alpha * S[i + (size_t) j * k] * xt[(size_t) c * k + j];
    }
    else {
      const cplx *N = h->N + h->boff[b];
      uint32_t rows = h->rt.size[r], cols = h->ct.size[c];
      for (j = 0; j < cols; j++) {
        cplx xj = x[h->ct.idx[h->ct.off[c] + j]];
        for (i = 0; i < rows; i++)
          y[h->rt.idx[h->rt.off[r] + i]] += alpha * N[i + (size_t) j * rows] * xj;
      }
    }
  }
  backward(h, &h->rt, 0, yt, y);
  free(xt);
  free(yt);
}

int
orc_h2_addeval(const orc_h2 *h, double alpha_re, double alpha_im, const double *x, double *y)
{
  uint32_t nr = h->rt.nidx, nc = h->ct.nidx, i;
  int cx = h->op.pde == 1;
  cplx *xv = malloc(sizeof(cplx) * nc), *yv = malloc(sizeof(cplx) * nr);
  if (!xv || !yv) { free(xv); free(yv); return -1; }
  for (i = 0; i < nc; i++) xv[i] = cx ? x[2 * i] + x[2 * i + 1] * I : x[i];
  for (i = 0; i < nr; i++) yv[i] = 0.0;
  h2_apply(h, alpha_re + alpha_im * I, xv, yv);
  for (i = 0; i < nr; i++) {
    if (cx) { y[2 * i] += creal(yv[i]); y[2 * i + 1] += cimag(yv[i]); }
    else y[i] += creal(yv[i]);
  }
  free(xv);
  free(yv);
  return 0;
}

/* ------------------------------------------------------------------ GMRES */

typedef struct {
  uint32_t nterms;
  orc_h2 *const *ops;
  const cplx *coef;
} combo_t;

static void
combo_apply(const combo_t *A, cplx alpha, const cplx *x, cplx *y)
{
  uint32_t i;
  for (i = 0; i < A->nterms; i++) h2_apply(A->ops[i], alpha * A->coef[i], x, y);
}

static double
sign1_abs(cplx v, cplx *sgn)
{
  double a = cabs(v);
  *sgn = (a == 0.0) ? 1.0 : v / a;
  return a;
}

/* Householder QR of the columns [col0, col0+ncols) of qr restricted to rows >= row0. */
static void
qr_cols(cplx *qr, uint32_t n, uint32_t row0, uint32_t col, cplx *tau)
{
  uint32_t i;
  double norm2 = 0.0, norm;
  cplx *a = qr + (size_t) col * n, diag, s, gamma;
  for (i = row0; i < n; i++) norm2 += creal(a[i] * conj(a[i]));
  norm = sqrt(norm2);
  if (norm2 <= 1e-300) { *tau = 0.0; return; }
  diag = a[row0];
  {
    double adiag = sign1_abs(diag, &s) + norm, beta = 1.0 / (norm2 + cabs(diag) * norm);
    beta *= adiag * adiag;
    gamma = conj(s) / adiag;
    for (i = row0 + 1; i < n; i++) a[i] *= gamma;
    *tau = beta;
    a[row0] = -s * norm;
  }
}

/* apply reflectors 0..refl-1 (qtrans) or refl-1..0 to x */
static void
qr_apply(const cplx *qr, uint32_t n, const cplx *tau, uint32_t refl, int qtrans, cplx *x)
{
  uint32_t k, i;
  if (qtrans) {
    for (k = 0; k < refl; k++) {
      cplx beta = conj(tau[k]), gamma;
      const cplx *v = qr + (size_t) k * n;
      if (beta == 0.0) continue;
      gamma = x[k];
      for (i = k + 1; i < n; i++) gamma += conj(v[i]) * x[i];
      gamma *= beta;
      x[k] -= gamma;
      for (i = k + 1; i < n; i++) x[i] -= gamma * v[i];
    }
  }
  else {
    for (k = refl; k-- > 0;) {
      cplx beta = tau[k], gamma;
      const cplx *v = qr + (size_t) k * n;
      if (beta == 0.0) continue;
      gamma = x[k];
      for (i = k + 1; i < n; i++) gamma += conj(v[i]) * x[i];
      gamma *= beta;
      x[k] -= gamma;
      for (i = k + 1; i < n; i++) x[i] -= gamma * v[i];
    }
  }
}

/* Givens rotations of Library/krylov.c:551/587, one number rho per rotation.  g_unitary = 0
 * restates the reference's complex form ((a, b) -> (c a + s b, c b - s a), s = c b / a), which
 * is not unitary for complex entries; g_unitary = 1 uses s = c conj(b / a) and
 * (a, b) -> (c a + s b, conj(c) b - conj(s) a), unitary, for checking the library's
 * H2B_SOLVE_UNITARY mode.  Both coincide for real entries. */
static int g_unitary = 0;

static cplx
findapply_givens(cplx *a, cplx *b)
{
  cplx aa = *a, bb = *b, s, c, t, rho;
  double a2 = creal(aa * conj(aa)), b2 = creal(bb * conj(bb));
  if (b2 < a2 || (g_unitary && b2 == a2 && a2 > 0.0)) {
    t = bb / aa; c = 1.0 / sqrt(creal(t * conj(t)) + 1.0); s = (g_unitary ? conj(t) : t) * c;
    rho = s;
  }
  else if (a2 < b2) {
    t = aa / bb; s = 1.0 / sqrt(creal(t * conj(t)) + 1.0); c = (g_unitary ? conj(t) : t) * s;
    rho = 1.0 / c;
  }
  else { c = 1.0; s = 0.0; rho = g_unitary ? 0.0 : 1.0; }
  *a = c * aa + s * bb;
  *b = 0.0;
  return rho;
}

static void
apply_givens(cplx rho, cplx *a, cplx *b)
{
  cplx aa = *a, bb = *b, s, c;
  double r2 = creal(rho * conj(rho));
  if (r2 < 1.0) { s = rho; c = sqrt(1.0 - creal(s * conj(s))); }
  else if (r2 > 1.0) { c = 1.0 / rho; s = sqrt(1.0 - creal(c * conj(c))); }
  else { c = 1.0; s = 0.0; }
  *a = c * aa + s * bb;
  *b = g_unitary ? conj(c) * bb - conj(s) * aa : c * bb - s * aa;
}

typedef struct {
  uint32_t n, kmax, k;
  cplx *qr, *tau, *rhat, *q;
} gm_t;

static void
gm_init(const combo_t *A, const cplx *b, cplx *x, gm_t *g)
{
  uint32_t i, n = g->n;
  cplx *r = g->qr;
  for (i = 0; i < n; i++) r[i] = b[i];
  combo_apply(A, -1.0, x, r);
  qr_cols(g->qr, n, 0, 0, &g->tau[0]);
  for (i = 0; i < n; i++) g->q[i] = 0.0;
  g->q[0] = 1.0;
  qr_apply(g->qr, n, g->tau, 1, 0, g->q);
  for (i = 0; i < g->kmax; i++) g->rhat[i] = 0.0;
  for (i = g->kmax; i < n; i++) g->rhat[i] = 0.0;
  g->rhat[0] = g->qr[0];
  g->k = 0;
}

static void
gm_step(const combo_t *A, gm_t *g)
{
  uint32_t k = g->k, n = g->n, i;
  cplx *a, rho;
  if (k + 1 >= g->kmax) return;
  a = g->qr + (size_t) (k + 1) * n;
  for (i = 0; i < n; i++) a[i] = 0.0;
  combo_apply(A, 1.0, g->q, a);
  qr_apply(g->qr, n, g->tau, k + 1, 1, a);
  qr_cols(g->qr, n, k + 1, k + 1, &g->tau[k + 1]);
  for (i = 0; i < n; i++) g->q[i] = 0.0;
  g->q[k + 1] = 1.0;
  qr_apply(g->qr, n, g->tau, k + 2, 0, g->q);
  for (i = 0; i < k; i++) {
    rho = g->qr[(i + 1) + (size_t) (i + 1) * n];
    apply_givens(rho, &g->qr[i + (size_t) (k + 1) * n], &g->qr[(i + 1) + (size_t) (k + 1) * n]);
  }
  rho = findapply_givens(&g->qr[k + (size_t) (k + 1) * n], &g->qr[(k + 1) + (size_t) (k + 1) * n]);
  g->qr[(k + 1) + (size_t) (k + 1) * n] = rho;
  apply_givens(rho, &g->rhat[k], &g->rhat[k + 1]);
  g->k = k + 1;
}

static void
gm_finish(const combo_t *A, const cplx *b, cplx *x, gm_t *g)
{
  uint32_t k = g->k, n = g->n, i, j;
  /* upper triangular solve with R = qr[0..k-1, 1..k] */
  for (j = k; j-- > 0;) {
    cplx s = g->rhat[j];
    for (i = j + 1; i < k; i++) s -= g->qr[j + (size_t) (i + 1) * n] * g->rhat[i];
    g->rhat[j] = s / g->qr[j + (size_t) (j + 1) * n];
  }
  for (i = k; i < n; i++) g->rhat[i] = 0.0;
  qr_apply(g->qr, n, g->tau, k, 0, g->rhat);
  for (i = 0; i < n; i++) x[i] += g->rhat[i];
  gm_init(A, b, x, g);
}

int
orc_gmres_unitary(uint32_t nterms, orc_h2 *const *ops, const double *coef, const double *b,
                  double *x, double eps, uint32_t maxiter, uint32_t kmax)
{
  int it;
  g_unitary = 1;
  it = orc_gmres(nterms, ops, coef, b, x, eps, maxiter, kmax);
  g_unitary = 0;
  return it;
}

int
orc_gmres(uint32_t nterms, orc_h2 *const *ops, const double *coef, const double *b, double *x,
          double eps, uint32_t maxiter, uint32_t kmax)
{
  combo_t A;
  gm_t g;
  cplx cf[16], *bv, *xv;
  uint32_t n, i, iter = 0;
  int cx;
  double norm = 0.0, err;
  if (nterms < 1 || nterms > 16 || kmax < 2) return -1;
  n = ops[0]->rt.nidx;
  cx = ops[0]->op.pde == 1;
  for (i = 0; i < nterms; i++) cf[i] = coef[2 * i] + coef[2 * i + 1] * I;
  A.nterms = nterms;
  A.ops = ops;
  A.coef = cf;
  g.n = n;
  g.kmax = kmax;
  g.qr = calloc((size_t) n * kmax, sizeof(cplx));
  g.tau = calloc(kmax, sizeof(cplx));
  g.rhat = calloc(n > kmax ? n : kmax, sizeof(cplx));
  g.q = calloc(n, sizeof(cplx));
  bv = malloc(sizeof(cplx) * n);
  xv = malloc(sizeof(cplx) * n);
  for (i = 0; i < n; i++) {
    bv[i] = cx ? b[2 * i] + b[2 * i + 1] * I : b[i];
    xv[i] = cx ? x[2 * i] + x[2 * i + 1] * I : x[i];
    norm += creal(bv[i] * conj(bv[i]));
  }
  norm = sqrt(norm);
  gm_init(&A, bv, xv, &g);
  err = cabs(g.rhat[g.k]);
  while (err > eps * norm && iter + 1 != maxiter) {
    if (g.k + 1 >= kmax) gm_finish(&A, bv, xv, &g);
    gm_step(&A, &g);
    err = cabs(g.rhat[g.k]);
    iter++;
    if (getenv("ORC_GMRES_TRACE"))
      fprintf(stderr, "gmres %u %.17e\n", iter, err / (eps * norm));
  }
  gm_finish(&A, bv, xv, &g);
  for (i = 0; i < n; i++) {
    if (cx) { x[2 * i] = creal(xv[i]); x[2 * i + 1] = cimag(xv[i]); }
    else x[i] = creal(xv[i]);
  }
  free(g.qr); free(g.tau); free(g.rhat); free(g.q); free(bv); free(xv);
  return (int) iter;
}

/* ------------------------------------------------------------------ RHS and errors */

static double
harmonic(const double *X, const double *z)
{
  double d0 = X[0] - z[0], d1 = X[1] - z[1], d2 = X[2] - z[2];
  return 1.0 / sqrt(d0 * d0 + d1 * d1 + d2 * d2);
}

static double
harmonic_dn(const double *X, const double *nn, const double *z)
{
  double d0 = X[0] - z[0], d1 = X[1] - z[1], d2 = X[2] - z[2];
  double r2 = d0 * d0 + d1 * d1 + d2 * d2;
  return -(d0 * nn[0] + d1 * nn[1] + d2 * nn[2]) / (r2 * sqrt(r2));
}

static void
mass_apply(uint32_t nv, uint32_t nt, const uint32_t *t, const double *g, const double *x,
           double *y)
{
  uint32_t i, j, k;
  for (i = 0; i < nv; i++) y[i] = 0.0;
  for (i = 0; i < nt; i++)
    for (j = 0; j < 3; j++)
      for (k = 0; k < 3; k++)
        y[t[3 * i + j]] += x[t[3 * i + k]] * g[i] * (j == k ? 1.0 / 12.0 : 1.0 / 24.0);
}

int
orc_project_l2_harmonic(uint32_t nv, const double *x, uint32_t nt, const uint32_t *t,
                        const double *g, uint32_t q, const double z[3], double *w)
{
  double xs[4096], ys[4096], ws[4096];
  double *v = calloc(nv, sizeof(double)), *r = malloc(8 * nv), *p = malloc(8 * nv),
         *a = malloc(8 * nv);
  uint32_t i, l, qq, ns = q * q, iter;
  double norm = 0.0, rr;
  if (!v || !r || !p || !a || single_rule(q, xs, ys, ws)) return -1;
  for (i = 0; i < nt; i++) {
    const uint32_t *tv = t + 3 * (size_t) i;
    const double *A = x + 3 * (size_t) tv[0], *B = x + 3 * (size_t) tv[1], *C = x + 3 * (size_t) tv[2];
    for (l = 0; l < 3; l++) {
      double sum = 0.0;
      for (qq = 0; qq < ns; qq++) {
        double tx = xs[qq], sx = ys[qq], X[3];
        int d;
        for (d = 0; d < 3; d++) X[d] = A[d] * (1.0 - tx) + B[d] * (tx - sx) + C[d] * sx;
        sum += (ws[qq] * nodal(1, l, tx, sx)) * harmonic(X, z);
      }
      v[tv[l]] += sum * g[i];
    }
  }
  /* CG on the mass matrix, start vector 0, to 1e-15 relative, at most 500 steps */
  for (i = 0; i < nv; i++) { w[i] = 0.0; r[i] = v[i]; p[i] = v[i]; norm += v[i] * v[i]; }
  norm = sqrt(norm);
  rr = norm * norm;
  for (iter = 0; sqrt(rr) > 1e-15 * norm && iter + 1 < 500; iter++) {
    double pa = 0.0, alpha, rr2 = 0.0;
    mass_apply(nv, nt, t, g, p, a);
    for (i = 0; i < nv; i++) pa += p[i] * a[i];
    alpha = rr / pa;
    for (i = 0; i < nv; i++) { w[i] += alpha * p[i]; r[i] -= alpha * a[i]; rr2 += r[i] * r[i]; }
    for (i = 0; i < nv; i++) p[i] = r[i] + (rr2 / rr) * p[i];
    rr = rr2;
  }
  free(v); free(r); free(p); free(a);
  return 0;
}

int
orc_l2_error_harmonic(uint32_t nv, const double *x, uint32_t nt, const uint32_t *t,
                      const double *n, const double *g, uint32_t q, const double z[3],
                      const double *u, double *err, double *norm)
{
  double xs[4096], ys[4096], ws[4096], e = 0.0, nn = 0.0;
  uint32_t i, qq, ns = q * q;
  (void) nv;
  if (single_rule(q, xs, ys, ws)) return -1;
  for (i = 0; i < nt; i++) {
    const uint32_t *tv = t + 3 * (size_t) i;
    const double *A = x + 3 * (size_t) tv[0], *B = x + 3 * (size_t) tv[1], *C = x + 3 * (size_t) tv[2];
    double se = 0.0, sn = 0.0;
    for (qq = 0; qq < ns; qq++) {
      double tx = xs[qq], sx = ys[qq], X[3], f, bf;
      int d;
      for (d = 0; d < 3; d++) X[d] = A[d] * (1.0 - tx) + B[d] * (tx - sx) + C[d] * sx;
      f = harmonic_dn(X, n + 3 * (size_t) i, z);
      bf = u[tv[0]] * (1.0 - tx) + u[tv[1]] * (tx - sx) + u[tv[2]] * sx;
      se += ws[qq] * (f - bf) * (f - bf);
      sn += ws[qq] * f * f;
    }
    e += g[i] * se;
    nn += g[i] * sn;
  }
  *err = sqrt(e);
  *norm = sqrt(nn);
  return 0;
}

/* Dirichlet datum of the point source f(x) = e^{ik|x - z|} / |x - z| tested with the constant
 * (b per triangle) or linear basis (b per vertex), by the single-triangle rule:
 * integrate_bem3d_c_avector / integrate_bem3d_l_avector (Library/bem3d.c:8579 / :8631) with
 * rhs_dirichlet_point_helmholtzbem3d (Library/helmholtzbem3d.c:1521).  b interleaved complex. */
int
orc_integrate_point_source(uint32_t nv, const double *x, uint32_t nt, const uint32_t *t,
                           const double *g, uint32_t q, int linear, const double z[3], double k,
                           double *b)
{
  double xs[4096], ys[4096], ws[4096];
  uint32_t i, l, qq, ns = q * q, n = linear ? nv : nt;
  if (single_rule(q, xs, ys, ws)) return -1;
  for (i = 0; i < 2 * n; i++) b[i] = 0.0;
  for (i = 0; i < nt; i++) {
    const uint32_t *tv = t + 3 * (size_t) i;
    const double *A = x + 3 * (size_t) tv[0], *B = x + 3 * (size_t) tv[1], *C = x + 3 * (size_t) tv[2];
    for (l = 0; l < (linear ? 3u : 1u); l++) {
      cplx sum = 0.0;
      for (qq = 0; qq < ns; qq++) {
        double tx = xs[qq], sx = ys[qq], X[3], r;
        int d;
        for (d = 0; d < 3; d++) X[d] = A[d] * (1.0 - tx) + B[d] * (tx - sx) + C[d] * sx;
        r = sqrt((X[0] - z[0]) * (X[0] - z[0]) + (X[1] - z[1]) * (X[1] - z[1]) +
                 (X[2] - z[2]) * (X[2] - z[2]));
        sum += (linear ? ws[qq] * nodal(1, l, tx, sx) : ws[qq]) * cexp(I * k * r) / r;
      }
      sum *= g[i];
      {
        const uint32_t o = linear ? tv[l] : i;
        b[2 * o] += creal(sum);
        b[2 * o + 1] += cimag(sum);
      }
    }
  }
  return 0;
}

/* Brakhage-Werner potential of the density w (constant: per triangle, linear: per vertex;
 * interleaved complex) at npoints points: sum over triangles of
 * 1/(4 pi) g_t sum_q w(y_q) e^{ikr} / r^3 ((1 - ikr) d.n - i eta r^2), d = x - y_q, r = |d|:
 * eval_brakhage_werner_c / _l (Tests/test_helmholtzbem3d.c:68 / :134). */
int
orc_eval_brakhage_werner(uint32_t nv, const double *x, uint32_t nt, const uint32_t *t,
                         const double *n, const double *g, uint32_t q, int linear, double k_re,
                         double k_im, double eta_re, double eta_im, const double *w,
                         uint32_t npoints, const double *pts, double *u)
{
  double xs[4096], ys[4096], ws[4096];
  const cplx k = k_re + I * k_im, eta = eta_re + I * eta_im;
  uint32_t p, i, l, qq, ns = q * q;
  (void) nv;
  if (single_rule(q, xs, ys, ws)) return -1;
  for (p = 0; p < npoints; p++) {
    const double *P = pts + 3 * (size_t) p;
    cplx res = 0.0;
    for (i = 0; i < nt; i++) {
      const uint32_t *tv = t + 3 * (size_t) i;
      const double *A = x + 3 * (size_t) tv[0], *B = x + 3 * (size_t) tv[1],
                   *C = x + 3 * (size_t) tv[2], *N = n + 3 * (size_t) i;
      cplx sum = 0.0;
      for (qq = 0; qq < ns; qq++) {
        double tx = xs[qq], sx = ys[qq], d[3], r2, r, dn;
        cplx wy = 0.0;
        int e;
        for (e = 0; e < 3; e++) d[e] = P[e] - (A[e] * (1.0 - tx) + B[e] * (tx - sx) + C[e] * sx);
        r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        r = sqrt(r2);
        dn = d[0] * N[0] + d[1] * N[1] + d[2] * N[2];
        if (linear) {
          for (l = 0; l < 3; l++)
            wy += ws[qq] * nodal(1, l, tx, sx) * (w[2 * tv[l]] + I * w[2 * tv[l] + 1]);
        } else {
          wy = ws[qq] * (w[2 * i] + I * w[2 * i + 1]);
        }
        sum += wy * cexp(I * k * r) / (r2 * r) * ((1.0 - I * k * r) * dn - I * eta * r2);
      }
      res += sum * g[i];
    }
    res *= 0.0795774715459476679; /* 1 / (4 pi) */
    u[2 * p] = creal(res);
    u[2 * p + 1] = cimag(res);
  }
  return 0;
}
