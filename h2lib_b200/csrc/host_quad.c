/* Host-side quadrature tables for the B200 nearfield kernels.
 *
 * Gauss-Legendre nodes on [0,1] are computed by Newton's method on the Legendre three-term
 * recurrence (Golub-Welsch is what the reference uses, Library/gaussquad.c:11; both give the
 * nodes to ~1 ulp, ascending).
 *
 * The Sauter-Schwab rules restate Library/singquad2d.c: the distant tensor rule (:50, q^4 points),
 * vertex-adjacent (:80, 2 q2^4), edge-adjacent (:129, 6 q2^4), identical (:206, 6 q2^4) and the
 * single-triangle rule (:25, q^2).  Point coordinates use the reference's parametrisation of the
 * unit triangle by (t, s) with 0 <= s <= t <= 1 and point = A(1-t) + B(t-s) + C s, so that the
 * vertex permutation chosen per pair (select_quadrature_singquad2d, :549) applies unchanged.
 * Basis weighting restates weight_basisfunc_{ll,cl,lc,l}_singquad2d (:456-530): weight row
 * (i + 3 j) = raw weight * phi_i(row point) * phi_j(column point) with the linear nodal functions
 * phi_0 = 1-t, phi_1 = t-s, phi_2 = s; a constant basis contributes the factor 1.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "h2b200_internal.h"

int
h2b_gauss_legendre01(uint32_t m, double *x, double *w)
{
  uint32_t i, it, k;
  if (m == 0 || m > 64) {
    h2b_set_error("h2b_gauss_legendre01: order %u out of range [1,64]", m);
    return H2B_ERR_ARG;
  }
  for (i = 0; i < m; i++) {
    /* i-th root from the top, refined by Newton on P_m */
    double z = cos(M_PI * (i + 0.75) / (m + 0.5)), p0, p1, dp = 1.0;
    for (it = 0; it < 100; it++) {
      double z1;
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
      z1 = z;
      z = z1 - p1 / dp;
      if (fabs(z - z1) <= 1e-16)
        break;
    }
    /* recompute at the converged node */
    p0 = 1.0;
    p1 = z;
    for (k = 2; k <= m; k++) {
      double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    dp = (m == 1) ? 1.0 : m * (z * p1 - p0) / (z * z - 1.0);
    /* node in ascending order on [0,1] */
    x[m - 1 - i] = 0.5 + 0.5 * z;
    w[m - 1 - i] = 0.5 * 2.0 / ((1.0 - z * z) * dp * dp);
  }
  if (m == 1) {
    x[0] = 0.5;
    w[0] = 1.0;
  }
  return H2B_OK;
}

static int
rule_alloc(h2b_rule *r, uint32_t n)
{
  r->n = n;
  r->x0 = (double *) calloc(n, sizeof(double));
  r->x1 = (double *) calloc(n, sizeof(double));
  r->y0 = (double *) calloc(n, sizeof(double));
  r->y1 = (double *) calloc(n, sizeof(double));
  r->w = (double *) calloc((size_t) 10 * n, sizeof(double));
  return (r->x0 && r->x1 && r->y0 && r->y1 && r->w) ? 0 : -1;
}

static void
rule_free(h2b_rule *r)
{
  free(r->x0); free(r->x1); free(r->y0); free(r->y1); free(r->w);
  memset(r, 0, sizeof(*r));
}

static inline void
put(h2b_rule *r, uint32_t p, double w, double x0, double x1, double y0, double y1)
{
  r->w[9 * (size_t) r->n + p] = w;
  r->x0[p] = x0;
  r->x1[p] = x1;
  r->y0[p] = y0;
  r->y1[p] = y1;
}

/* Distant pairs: tensor Gauss rule on both triangles (Duffy map of the square). */
static void
build_dist(h2b_rule *r, uint32_t q, const double *g, const double *gw)
{
  uint32_t i, j, k, l, p = 0;
  for (i = 0; i < q; i++)
    for (j = 0; j < q; j++)
      for (k = 0; k < q; k++)
        for (l = 0; l < q; l++)
          put(r, p++, gw[i] * gw[j] * gw[k] * gw[l] * g[i] * g[k],
              g[i], g[i] * g[j], g[k], g[k] * g[l]);
}

/* Common vertex (at local vertex 0 of both triangles): two sub-simplices. */
static void
build_vert(h2b_rule *r, uint32_t q, const double *g, const double *gw)
{
  uint32_t i, j, k, l, p = 0;
  for (i = 0; i < q; i++)
    for (j = 0; j < q; j++)
      for (k = 0; k < q; k++)
        for (l = 0; l < q; l++) {
          double e1 = g[i], e2 = g[j], e3 = g[k], xi = g[l];
          double w = gw[i] * gw[j] * gw[k] * gw[l] * xi * xi * xi * e1;
          put(r, p++, w, xi, e2 * xi, e1 * xi, e1 * e3 * xi);
          put(r, p++, w, e1 * xi, e1 * e3 * xi, xi, e2 * xi);
        }
}

/* Common edge (local vertices 0,1 of both triangles): six sub-simplices. */
static void
build_edge(h2b_rule *r, uint32_t q, const double *g, const double *gw)
{
  uint32_t i, j, k, l, p = 0;
  for (i = 0; i < q; i++)
    for (j = 0; j < q; j++)
      for (k = 0; k < q; k++)
        for (l = 0; l < q; l++) {
          double e1 = g[i], e2 = g[j], x1 = g[k];
          double x2 = g[l] * (1.0 - x1);
          double w = gw[i] * gw[j] * gw[k] * (gw[l] * (1.0 - x1)) * x1 * x1 * e1;
          put(r, p++, w, x1 + x2, x1 * e1 * e2, x1 * (1.0 - e1) + x2, x1 * (1.0 - e1));
          put(r, p++, w, x1 + x2, x1 * e1, x1 * (1.0 - e1 * e2) + x2, x1 * (1.0 - e1 * e2));
          put(r, p++, w, x1 + x2, x1, x1 * e1 + x2, x1 * e1 * e2);
          put(r, p++, w, x1 * (1.0 - e1 + e1 * e2) + x2, x1 * e1 * e2, x1 + x2, x1);
          put(r, p++, w, x1 * e1 * e2 + x2, x1 * e1 * e2, x1 + x2, x1 * e1);
          put(r, p++, w, x1 * e1 + x2, x1 * e1, x1 + x2, x1 * e1 * e2);
        }
}

/* Identical triangles: six sub-simplices. */
static void
build_id(h2b_rule *r, uint32_t q, const double *g, const double *gw)
{
  uint32_t i, j, k, l, p = 0;
  for (i = 0; i < q; i++)
    for (j = 0; j < q; j++)
      for (k = 0; k < q; k++)
        for (l = 0; l < q; l++) {
          double eta = g[i], x1 = g[j];
          double x2 = g[k] * (1.0 - x1);
          double x3 = g[l] * (1.0 - x1 - x2);
          double w = gw[i] * gw[j] * (gw[k] * (1.0 - x1)) * (gw[l] * (1.0 - x1 - x2)) * x1;
          double a = x1 * (1.0 - eta);
          put(r, p++, w, x1 + x2 + x3, x1 + x2, a + x2 + x3, x2);
          put(r, p++, w, a + x2 + x3, a + x2, x1 + x2 + x3, x2);
          put(r, p++, w, x1 + x2 + x3, x1 * eta + x2, x2 + x3, x2);
          put(r, p++, w, a + x2 + x3, x2, x1 + x2 + x3, x1 + x2);
          put(r, p++, w, x1 + x2 + x3, x2, a + x2 + x3, a + x2);
          put(r, p++, w, x2 + x3, x2, x1 + x2 + x3, x1 * eta + x2);
        }
}

static inline double
nodal(int basis, int i, double t, double s)
{
  if (basis != H2B_BASIS_LINEAR)
    return 1.0;
  return i == 0 ? 1.0 - t : (i == 1 ? t - s : s);
}

/* Rows 0..8 of w: raw weight times the row/column basis factors. */
static void
weight_rule(h2b_rule *r, int row_basis, int col_basis)
{
  uint32_t p, i, j, n = r->n;
  for (j = 0; j < 3; j++)
    for (i = 0; i < 3; i++)
      for (p = 0; p < n; p++)
        r->w[(i + 3 * j) * (size_t) n + p] = r->w[9 * (size_t) n + p]
            * nodal(row_basis, (int) i, r->x0[p], r->x1[p])
            * nodal(col_basis, (int) j, r->y0[p], r->y1[p]);
}

int
h2b_quad_build(uint32_t q, uint32_t q2, int row_basis, int col_basis, h2b_quad *out)
{
  double g[64], gw[64], g2[64], gw2[64];
  uint32_t n2 = q2 * q2 * q2 * q2, i, j, p;
  memset(out, 0, sizeof(*out));
  if (q < 1 || q > 16 || q2 < 1 || q2 > 16) {
    h2b_set_error("quadrature orders q=%u q2=%u out of range [1,16]", q, q2);
    return H2B_ERR_ARG;
  }
  if (h2b_gauss_legendre01(q, g, gw) || h2b_gauss_legendre01(q2, g2, gw2))
    return H2B_ERR_ARG;
  out->q = q;
  out->q2 = q2;
  if (rule_alloc(&out->rule[H2B_RULE_DIST], q * q * q * q)
      || rule_alloc(&out->rule[H2B_RULE_VERT], 2 * n2)
      || rule_alloc(&out->rule[H2B_RULE_EDGE], 6 * n2)
      || rule_alloc(&out->rule[H2B_RULE_ID], 6 * n2)) {
    h2b_quad_free(out);
    h2b_set_error("h2b_quad_build: out of host memory");
    return H2B_ERR_NOMEM;
  }
  build_dist(&out->rule[H2B_RULE_DIST], q, g, gw);
  build_vert(&out->rule[H2B_RULE_VERT], q2, g2, gw2);
  build_edge(&out->rule[H2B_RULE_EDGE], q2, g2, gw2);
  build_id(&out->rule[H2B_RULE_ID], q2, g2, gw2);
  for (i = 0; i < 4; i++)
    weight_rule(&out->rule[i], row_basis, col_basis);

  /* single-triangle rule, Library/singquad2d.c:25 */
  out->ns = q * q;
  out->xs = (double *) calloc(out->ns, sizeof(double));
  out->ys = (double *) calloc(out->ns, sizeof(double));
  out->ws = (double *) calloc((size_t) 4 * out->ns, sizeof(double));
  if (!out->xs || !out->ys || !out->ws) {
    h2b_quad_free(out);
    h2b_set_error("h2b_quad_build: out of host memory");
    return H2B_ERR_NOMEM;
  }
  p = 0;
  for (i = 0; i < q; i++)
    for (j = 0; j < q; j++) {
      out->ws[3 * out->ns + p] = gw[i] * gw[j] * g[i];
      out->xs[p] = g[i];
      out->ys[p] = g[i] * g[j];
      p++;
    }
  for (i = 0; i < 3; i++)
    for (p = 0; p < out->ns; p++)
      out->ws[i * out->ns + p] = out->ws[3 * out->ns + p]
          * nodal(H2B_BASIS_LINEAR, (int) i, out->xs[p], out->ys[p]);
  return H2B_OK;
}

/* Reduced edge / identical rule.  With the shared vertices first in both triangles (the
 * permutation of select_quadrature_singquad2d), X - Y depends on fewer variables than the rule
 * has: for a common edge (A, B shared) X - Y = (x0 - y0)(B - A) + x1 (C_t - B) - y1 (C_s - B),
 * and in each sub-simplex of build_edge x0 - y0, x1 and y1 do not depend on the innermost Gauss
 * variable (xi2, loop l); for identical triangles X - Y = (x0 - y0)(B - A) + (x1 - y1)(C - B),
 * and x0 - y0, x1 - y1 depend on neither xi2 nor xi3 (loops k, l).  The points that differ only
 * in those variables therefore share one kernel value, so they become one point whose
 * basis-weighted weights are the sums of theirs: q2 (edge) or q2^2 (identical) times fewer
 * kernel evaluations for the same quadrature sum (summed in another order).
 * Output: n' points; abc[0..n'), abc[n'..2n'), abc[2n'..3n') = (a, b, c) with
 * X - Y = (A_t - A_s) + a (B_t - A_t) + b (C_t - B_t) - c (C_s - B_s); w9[(i + 3 j) n' + g] the
 * summed weight rows 0..8.  Points are ordered as build_edge / build_id order them: six
 * sub-simplices innermost, then l, k, j, i. */
int
h2b_quad_reduce(const h2b_rule *r, int which, uint32_t q2, uint32_t *n_out, double **abc,
                double **w9)
{
  const uint32_t merge = which == H2B_RULE_EDGE ? q2 : q2 * q2;
  uint32_t n, p, g, i;
  *abc = NULL;
  *w9 = NULL;
  if ((which != H2B_RULE_EDGE && which != H2B_RULE_ID) || r->n % (6 * merge)) {
    h2b_set_error("h2b_quad_reduce: rule %d cannot be reduced", which);
    return H2B_ERR_ARG;
  }
  n = r->n / merge;
  *abc = (double *) calloc(3 * (size_t) n, sizeof(double));
  *w9 = (double *) calloc(9 * (size_t) n, sizeof(double));
  if (!*abc || !*w9) {
    free(*abc);
    free(*w9);
    *abc = *w9 = NULL;
    h2b_set_error("h2b_quad_reduce: out of host memory");
    return H2B_ERR_NOMEM;
  }
  for (p = 0; p < r->n; p++) {
    const uint32_t s = p % 6, rest = p / 6, m = rest % merge, outer = rest / merge;
    g = outer * 6 + s;
    if (m == 0) {  /* the group's first point defines its kernel argument */
      (*abc)[g] = r->x0[p] - r->y0[p];
      if (which == H2B_RULE_EDGE) {
        (*abc)[n + g] = r->x1[p];
        (*abc)[2 * (size_t) n + g] = r->y1[p];
      }
      else {
        (*abc)[n + g] = r->x1[p] - r->y1[p];
        (*abc)[2 * (size_t) n + g] = 0.0;
      }
    }
    for (i = 0; i < 9; i++)
      (*w9)[i * (size_t) n + g] += r->w[i * (size_t) r->n + p];
  }
  *n_out = n;
  return H2B_OK;
}

/* Common-vertex rule in tensor form.  build_vert's points with the same (eta1, xi, sub-simplex)
 * form a q2 x q2 tensor product: in sub-simplex 0 the row point (xi, eta2 xi) runs over eta2 and
 * the column point (eta1 xi, eta1 eta3 xi) over eta3, in sub-simplex 1 the roles swap, and the
 * weight gw_i gw_j gw_k gw_l xi^3 eta1 factors into a group part, a row-point part and a
 * column-point part.  A group therefore needs q2 row points and q2 column points instead of
 * q2^2 point pairs, and the pair sum can be taken column side first (as for distant pairs).
 * Output (ngroups = 2 q2^2 groups, each array ngroups long, group g = (i q2 + l) 2 + s):
 *   row points a < q2:    x0, x1, then NR weights G w_a phi_r(x)   (NR = 3 linear, 1 constant)
 *   column points b < q2: y0, y1, then NC weights w_b phi_c(y)
 * i.e. (2 + NR) q2 + (2 + NC) q2 arrays. */
int
h2b_quad_vert_tensor(uint32_t q2, int row_basis, int col_basis, uint32_t *ngroups, double **out)
{
  double g[64], gw[64];
  const uint32_t NR = row_basis == H2B_BASIS_LINEAR ? 3 : 1, NC = col_basis == H2B_BASIS_LINEAR ? 3 : 1;
  const uint32_t G = 2 * q2 * q2, rstride = 2 + NR, cstride = 2 + NC;
  uint32_t i, l, s, a, r;
  double *o, *col;
  *out = NULL;
  if (h2b_gauss_legendre01(q2, g, gw))
    return H2B_ERR_ARG;
  o = (double *) calloc((size_t) (rstride + cstride) * q2 * G, sizeof(double));
  if (!o) {
    h2b_set_error("h2b_quad_vert_tensor: out of host memory");
    return H2B_ERR_NOMEM;
  }
  col = o + (size_t) rstride * q2 * G;
  for (i = 0; i < q2; i++)
    for (l = 0; l < q2; l++)
      for (s = 0; s < 2; s++) {
        const uint32_t grp = (i * q2 + l) * 2 + s;
        const double e1 = g[i], xi = g[l];
        const double wg = gw[i] * gw[l] * xi * xi * xi * e1;
        for (a = 0; a < q2; a++) {
          /* the point that varies with eta2 (index j) or eta3 (index k) */
          const double pa0 = xi, pa1 = g[a] * xi;                  /* (xi, eta xi) */
          const double pb0 = e1 * xi, pb1 = e1 * g[a] * xi;        /* (eta1 xi, eta1 eta xi) */
          const double x0 = s == 0 ? pa0 : pb0, x1 = s == 0 ? pa1 : pb1;
          const double y0 = s == 0 ? pb0 : pa0, y1 = s == 0 ? pb1 : pa1;
          double *rp = o + (size_t) a * rstride * G, *cp = col + (size_t) a * cstride * G;
          rp[grp] = x0;
          rp[G + grp] = x1;
          for (r = 0; r < NR; r++)
            rp[(2 + r) * (size_t) G + grp] = wg * gw[a] * nodal(row_basis, (int) r, x0, x1);
          cp[grp] = y0;
          cp[G + grp] = y1;
          for (r = 0; r < NC; r++)
            cp[(2 + r) * (size_t) G + grp] = gw[a] * nodal(col_basis, (int) r, y0, y1);
        }
      }
  *ngroups = G;
  *out = o;
  return H2B_OK;
}

/* Common-vertex rule with the radial Gauss sum folded into moments (Laplace kernels only).  In
 * h2b_quad_vert_tensor every row and column point of group (i, l, s) is xi = g[l] times a point
 * that does not depend on l: x = xi xh, y = xi yh.  With the shared vertex first in both
 * triangles, x - y = xi (xh - yh), so a kernel homogeneous of degree -p (p = 1 single layer,
 * p = 2 double layer and its adjoint) gives k(x - y) = xi^-p k(xh - yh), and the linear basis
 * functions are affine in xi: phi(xi xh) = phi(0) + xi (phi(xh) - phi(0)).  The sum over l then
 * needs only the moments M_e = sum_l gw[l] g[l]^e:
 *   sum_l gw[l] xi^(3-p) phi_r(xi xh) phi_c(xi yh)
 *     = phi_r0 phi_c0 M_(3-p) + (phi_r0 C + R phi_c0) M_(4-p) + R C M_(5-p),
 * R = phi_r(xh) - phi_r0, C = phi_c(yh) - phi_c0: one kernel evaluation per (i, s, a, b) instead
 * of q2 of them.  Same quadrature sum as the point rule, in another order.
 * Output: n = 2 q2^2 items k = (i 2 + s) q2 + a, arrays of n doubles each:
 *   row point a of group (i, s):    xh0, xh1, U_r (NR), V_r (NR)
 *       U_r = gw[i] eta1 gw[a] phi_r0,  V_r = gw[i] eta1 gw[a] R_r
 *   column point b of group (i, s) (index (i 2 + s) q2 + b):  yh0, yh1, then for p = 1 and p = 2
 *       A_c = gw[b] (phi_c0 M_(3-p) + C_c M_(4-p)),  B_c = gw[b] (phi_c0 M_(4-p) + C_c M_(5-p))
 *   (NC each, p = 1 first), i.e. (2 + 2 NR) + (2 + 4 NC) arrays;
 * the entry sum is  sum over (i, s, a, b) of  k_p(xh - yh) (U_r A_c + V_r B_c). */
int
h2b_quad_vert_merged(uint32_t q2, int row_basis, int col_basis, uint32_t *n_out, double **out)
{
  double g[64], gw[64], M[6] = {0, 0, 0, 0, 0, 0};
  const uint32_t NR = row_basis == H2B_BASIS_LINEAR ? 3 : 1, NC = col_basis == H2B_BASIS_LINEAR ? 3 : 1;
  const uint32_t n = 2 * q2 * q2, rs = 2 + 2 * NR, cs = 2 + 4 * NC;
  uint32_t i, l, s, a, r, p, e;
  double *o, *col;
  *out = NULL;
  if (h2b_gauss_legendre01(q2, g, gw))
    return H2B_ERR_ARG;
  for (e = 0; e < 6; e++)
    for (l = 0; l < q2; l++) {
      double pw = 1.0;
      for (p = 0; p < e; p++)
        pw *= g[l];
      M[e] += gw[l] * pw;
    }
  o = (double *) calloc((size_t) (rs + cs) * n, sizeof(double));
  if (!o) {
    h2b_set_error("h2b_quad_vert_merged: out of host memory");
    return H2B_ERR_NOMEM;
  }
  col = o + (size_t) rs * n;
  for (i = 0; i < q2; i++)
    for (s = 0; s < 2; s++) {
      const double e1 = g[i], wg = gw[i] * e1;
      for (a = 0; a < q2; a++) {
        const uint32_t k = (i * 2 + s) * q2 + a;
        /* (1, eta) and (eta1, eta1 eta): the tensor form's points divided by xi */
        const double pa0 = 1.0, pa1 = g[a], pb0 = e1, pb1 = e1 * g[a];
        const double x0 = s == 0 ? pa0 : pb0, x1 = s == 0 ? pa1 : pb1;
        const double y0 = s == 0 ? pb0 : pa0, y1 = s == 0 ? pb1 : pa1;
        o[k] = x0;
        o[n + k] = x1;
        for (r = 0; r < NR; r++) {
          const double f0 = nodal(row_basis, (int) r, 0.0, 0.0);
          o[(2 + r) * (size_t) n + k] = wg * gw[a] * f0;
          o[(2 + NR + r) * (size_t) n + k] = wg * gw[a] * (nodal(row_basis, (int) r, x0, x1) - f0);
        }
        col[k] = y0;
        col[n + k] = y1;
        for (p = 1; p <= 2; p++)
          for (r = 0; r < NC; r++) {
            const double f0 = nodal(col_basis, (int) r, 0.0, 0.0);
            const double C = nodal(col_basis, (int) r, y0, y1) - f0;
            const size_t base = 2 + (p - 1) * 2 * NC;
            col[(base + r) * n + k] = gw[a] * (f0 * M[3 - p] + C * M[4 - p]);
            col[(base + NC + r) * n + k] = gw[a] * (f0 * M[4 - p] + C * M[5 - p]);
          }
      }
    }
  *n_out = n;
  *out = o;
  return H2B_OK;
}

void
h2b_quad_free(h2b_quad *qd)
{
  int i;
  for (i = 0; i < 4; i++)
    rule_free(&qd->rule[i]);
  free(qd->xs);
  free(qd->ys);
  free(qd->ws);
  memset(qd, 0, sizeof(*qd));
}

int
h2b_quad_export(uint32_t q, uint32_t q2, int row_basis, int col_basis, int which,
                uint32_t *n, double *x0, double *x1, double *y0, double *y1, double *w10)
{
  h2b_quad qd;
  int rc = h2b_quad_build(q, q2, row_basis, col_basis, &qd);
  if (rc)
    return rc;
  if (which >= 0 && which < 4) {
    h2b_rule *r = &qd.rule[which];
    *n = r->n;
    if (x0) memcpy(x0, r->x0, sizeof(double) * r->n);
    if (x1) memcpy(x1, r->x1, sizeof(double) * r->n);
    if (y0) memcpy(y0, r->y0, sizeof(double) * r->n);
    if (y1) memcpy(y1, r->y1, sizeof(double) * r->n);
    if (w10) memcpy(w10, r->w, sizeof(double) * 10 * r->n);
  }
  else if (which == 4) {
    *n = qd.ns;
    if (x0) memcpy(x0, qd.xs, sizeof(double) * qd.ns);
    if (x1) memcpy(x1, qd.ys, sizeof(double) * qd.ns);
    if (w10) memcpy(w10, qd.ws, sizeof(double) * 4 * qd.ns);
  }
  else {
    h2b_quad_free(&qd);
    h2b_set_error("h2b_quad_export: rule index %d out of range [0,4]", which);
    return H2B_ERR_ARG;
  }
  h2b_quad_free(&qd);
  return H2B_OK;
}
