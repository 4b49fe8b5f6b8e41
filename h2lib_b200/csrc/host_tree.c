/* Host-side cluster trees and block trees, flattened for the device.
 *
 * Restates, in this project's own code:
 *   build_bem3d_const_clustergeometry / _linear_  Library/bem3d.c:811 / :850
 *        (characteristic point = triangle centroid / vertex; support box = triangle box /
 *         union of the boxes of the triangles around the vertex)
 *   build_adaptive_cluster                        Library/cluster.c:80
 *        (split the longest side of the point bounding box at its midpoint, in-place partition
 *         of the index array; leaves get the support box, inner clusters the union of the sons)
 *   admissible_max_cluster                        Library/block.c:52
 *        (max(diam_inf(t), diam_inf(s)) <= eta * dist_inf(t, s), using getdiam_max_cluster and
 *         getdist_max_cluster, Library/cluster.c:775 / :793)
 *   build_strict_block                            Library/block.c:258
 *        (inadmissible blocks are refined until both clusters are leaves)
 * The index permutation, the pre-order numbering of clusters and the son-major order of block
 * leaves match the reference, so that the device arrays can be compared with H2Lib's trees.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "h2b200_internal.h"

typedef struct {
  uint32_t n;
  double *x;        /* characteristic points, 3 per index */
  double *smin;     /* support boxes */
  double *smax;
} cgeom_t;

/* Growable pre-order cluster storage. */
typedef struct {
  h2b_ctree *t;
  uint32_t cap;
} cbuild_t;

static int
cbuild_push(cbuild_t *b)
{
  h2b_ctree *t = b->t;
  if (t->n == b->cap) {
    uint32_t cap = b->cap ? 2 * b->cap : 256;
#define GROW(f, k)                                                   \
  do {                                                               \
    void *p = realloc(t->f, sizeof(*t->f) * (size_t) (k) * cap);     \
    if (!p)                                                          \
      return -1;                                                     \
    t->f = p;                                                        \
  } while (0)
    GROW(off, 1); GROW(size, 1); GROW(sons, 1); GROW(son0, 1); GROW(son1, 1);
    GROW(father, 1); GROW(level, 1); GROW(bmin, 3); GROW(bmax, 3);
#undef GROW
    b->cap = cap;
  }
  return (int) t->n++;
}

static void
support_box(const cgeom_t *cg, const uint32_t *idx, uint32_t size, double *bmin, double *bmax)
{
  uint32_t i, d;
  for (d = 0; d < 3; d++) {
    bmin[d] = cg->smin[3 * (size_t) idx[0] + d];
    bmax[d] = cg->smax[3 * (size_t) idx[0] + d];
  }
  for (i = 1; i < size; i++)
    for (d = 0; d < 3; d++) {
      double lo = cg->smin[3 * (size_t) idx[i] + d], hi = cg->smax[3 * (size_t) idx[i] + d];
      if (lo < bmin[d]) bmin[d] = lo;
      if (hi > bmax[d]) bmax[d] = hi;
    }
}

static int
build_cluster(cbuild_t *b, const cgeom_t *cg, uint32_t *idx0, uint32_t off, uint32_t size,
              uint32_t clf, uint32_t father, uint32_t level)
{
  h2b_ctree *t = b->t;
  uint32_t *idx = idx0 + off;
  int id = cbuild_push(b);
  uint32_t d;
  if (id < 0)
    return -1;
  t->off[id] = off;
  t->size[id] = size;
  t->sons[id] = 0;
  t->son0[id] = t->son1[id] = UINT32_MAX;
  t->father[id] = father;
  t->level[id] = level;
  if (level + 1 > t->depth)
    t->depth = level + 1;

  if (size > clf) {
    double hmin[3], hmax[3], a, mid;
    uint32_t i, dir = 0, size0 = 0;
    for (d = 0; d < 3; d++)
      hmin[d] = hmax[d] = cg->x[3 * (size_t) idx[0] + d];
    for (i = 1; i < size; i++)
      for (d = 0; d < 3; d++) {
        double v = cg->x[3 * (size_t) idx[i] + d];
        if (v < hmin[d]) hmin[d] = v;
        if (v > hmax[d]) hmax[d] = v;
      }
    a = hmax[0] - hmin[0];
    for (d = 1; d < 3; d++)
      if (a < hmax[d] - hmin[d]) {
        a = hmax[d] - hmin[d];
        dir = d;
      }
    if (a > 0.0) {
      mid = (hmax[dir] + hmin[dir]) / 2.0;
      for (i = 0; i < size; i++)
        if (cg->x[3 * (size_t) idx[i] + dir] < mid) {
          uint32_t tmp = idx[i];
          idx[i] = idx[size0];
          idx[size0] = tmp;
          size0++;
        }
      if (size0 > 0 && size0 < size) {
        int s0, s1;
        t->sons[id] = 2;
        s0 = build_cluster(b, cg, idx0, off, size0, clf, (uint32_t) id, level + 1);
        if (s0 < 0)
          return -1;
        s1 = build_cluster(b, cg, idx0, off + size0, size - size0, clf, (uint32_t) id, level + 1);
        if (s1 < 0)
          return -1;
        t = b->t;
        t->son0[id] = (uint32_t) s0;
        t->son1[id] = (uint32_t) s1;
        for (d = 0; d < 3; d++) {
          t->bmin[3 * id + d] = fmin(t->bmin[3 * s0 + d], t->bmin[3 * s1 + d]);
          t->bmax[3 * id + d] = fmax(t->bmax[3 * s0 + d], t->bmax[3 * s1 + d]);
        }
        return id;
      }
      /* one side empty: leaf with the bounding box of its sons' union (= its own support) */
    }
  }
  support_box(cg, idx, size, t->bmin + 3 * (size_t) id, t->bmax + 3 * (size_t) id);
  return id;
}

static void
bbox3(const double *a, const double *b, const double *c, double *lo, double *hi)
{
  int d;
  for (d = 0; d < 3; d++) {
    lo[d] = fmin(a[d], fmin(b[d], c[d]));
    hi[d] = fmax(a[d], fmax(b[d], c[d]));
  }
}

int
h2b_ctree_build(uint32_t vertices, const double *x, uint32_t triangles, const uint32_t *t,
                int basis, uint32_t clf, h2b_ctree *out)
{
  cgeom_t cg;
  cbuild_t b;
  uint32_t i, n, d, k;
  memset(out, 0, sizeof(*out));
  if (clf < 1) {
    h2b_set_error("h2b_ctree_build: leaf size must be >= 1");
    return H2B_ERR_ARG;
  }
  n = (basis == H2B_BASIS_LINEAR) ? vertices : triangles;
  if (n == 0) {
    h2b_set_error("h2b_ctree_build: empty index set");
    return H2B_ERR_ARG;
  }
  cg.n = n;
  cg.x = (double *) malloc(sizeof(double) * 3 * n);
  cg.smin = (double *) malloc(sizeof(double) * 3 * n);
  cg.smax = (double *) malloc(sizeof(double) * 3 * n);
  out->idx = (uint32_t *) malloc(sizeof(uint32_t) * n);
  if (!cg.x || !cg.smin || !cg.smax || !out->idx) {
    free(cg.x); free(cg.smin); free(cg.smax); free(out->idx);
    h2b_set_error("h2b_ctree_build: out of host memory");
    return H2B_ERR_NOMEM;
  }
  out->nidx = n;
  for (i = 0; i < n; i++)
    out->idx[i] = i;

  if (basis == H2B_BASIS_LINEAR) {
    for (i = 0; i < vertices; i++)
      for (d = 0; d < 3; d++)
        cg.x[3 * i + d] = cg.smin[3 * i + d] = cg.smax[3 * i + d] = x[3 * (size_t) i + d];
    for (i = 0; i < triangles; i++) {
      const uint32_t *ti = t + 3 * (size_t) i;
      double lo[3], hi[3];
      bbox3(x + 3 * (size_t) ti[0], x + 3 * (size_t) ti[1], x + 3 * (size_t) ti[2], lo, hi);
      for (k = 0; k < 3; k++)
        for (d = 0; d < 3; d++) {
          double *smin = cg.smin + 3 * (size_t) ti[k], *smax = cg.smax + 3 * (size_t) ti[k];
          smin[d] = fmin(smin[d], lo[d]);
          smax[d] = fmax(smax[d], hi[d]);
        }
    }
  }
  else {
    for (i = 0; i < triangles; i++) {
      const uint32_t *ti = t + 3 * (size_t) i;
      const double *a = x + 3 * (size_t) ti[0], *bb = x + 3 * (size_t) ti[1],
                   *c = x + 3 * (size_t) ti[2];
      for (d = 0; d < 3; d++)
        cg.x[3 * i + d] = (a[d] + bb[d] + c[d]) / 3.0;
      bbox3(a, bb, c, cg.smin + 3 * (size_t) i, cg.smax + 3 * (size_t) i);
    }
  }

  b.t = out;
  b.cap = 0;
  if (build_cluster(&b, &cg, out->idx, 0, n, clf, UINT32_MAX, 0) < 0) {
    free(cg.x); free(cg.smin); free(cg.smax);
    h2b_ctree_free(out);
    h2b_set_error("h2b_ctree_build: out of host memory");
    return H2B_ERR_NOMEM;
  }
  free(cg.x); free(cg.smin); free(cg.smax);
  return H2B_OK;
}

void
h2b_ctree_free(h2b_ctree *t)
{
  free(t->off); free(t->size); free(t->sons); free(t->son0); free(t->son1);
  free(t->father); free(t->level); free(t->bmin); free(t->bmax); free(t->idx);
  memset(t, 0, sizeof(*t));
}

/* ---------------- block tree ---------------- */

static double
diam_max(const h2b_ctree *t, uint32_t c)
{
  double m = 0.0;
  int d;
  for (d = 0; d < 3; d++) {
    double v = t->bmax[3 * c + d] - t->bmin[3 * c + d];
    if (v > m) m = v;
  }
  return m;
}

static double
dist_max(const h2b_ctree *a, uint32_t i, const h2b_ctree *b, uint32_t j)
{
  double m = 0.0;
  int d;
  for (d = 0; d < 3; d++) {
    double v = 0.0;
    if (a->bmax[3 * i + d] < b->bmin[3 * j + d])
      v = b->bmin[3 * j + d] - a->bmax[3 * i + d];
    else if (b->bmax[3 * j + d] < a->bmin[3 * i + d])
      v = a->bmin[3 * i + d] - b->bmax[3 * j + d];
    if (v > m) m = v;
  }
  return m;
}

typedef struct {
  h2b_blist *l;
  uint32_t cap;
} bbuild_t;

static int
bpush(bbuild_t *b, uint32_t rc, uint32_t cc, uint8_t adm)
{
  h2b_blist *l = b->l;
  if (l->n == b->cap) {
    uint32_t cap = b->cap ? 2 * b->cap : 1024;
    void *p1 = realloc(l->rc, sizeof(uint32_t) * cap);
    void *p2 = p1 ? realloc(l->cc, sizeof(uint32_t) * cap) : NULL;
    void *p3 = p2 ? realloc(l->adm, cap) : NULL;
    if (p1) l->rc = p1;
    if (p2) l->cc = p2;
    if (!p3)
      return -1;
    l->adm = p3;
    b->cap = cap;
  }
  l->rc[l->n] = rc;
  l->cc[l->n] = cc;
  l->adm[l->n] = adm;
  l->n++;
  return 0;
}

static int
build_block(bbuild_t *b, const h2b_ctree *rt, uint32_t r, const h2b_ctree *ct, uint32_t c,
            double eta)
{
  double dist = dist_max(rt, r, ct, c);
  int adm = (diam_max(rt, r) <= eta * dist) && (diam_max(ct, c) <= eta * dist);
  uint32_t rs[2], cs[2], nr, nc, i, j;
  if (adm)
    return bpush(b, r, c, 1);
  if (rt->sons[r] == 0 && ct->sons[c] == 0)
    return bpush(b, r, c, 0);
  /* refine every side that has sons; sons enumerated column-major (column son outer) */
  nr = rt->sons[r] ? 2 : 1;
  nc = ct->sons[c] ? 2 : 1;
  rs[0] = rt->sons[r] ? rt->son0[r] : r;
  rs[1] = rt->son1[r];
  cs[0] = ct->sons[c] ? ct->son0[c] : c;
  cs[1] = ct->son1[c];
  for (j = 0; j < nc; j++)
    for (i = 0; i < nr; i++)
      if (build_block(b, rt, rs[i], ct, cs[j], eta))
        return -1;
  return 0;
}

int
h2b_blist_build(const h2b_ctree *rt, const h2b_ctree *ct, double eta, h2b_blist *out)
{
  bbuild_t b;
  memset(out, 0, sizeof(*out));
  b.l = out;
  b.cap = 0;
  if (build_block(&b, rt, 0, ct, 0, eta)) {
    h2b_blist_free(out);
    h2b_set_error("h2b_blist_build: out of host memory");
    return H2B_ERR_NOMEM;
  }
  return H2B_OK;
}

void
h2b_blist_free(h2b_blist *b)
{
  free(b->rc); free(b->cc); free(b->adm);
  memset(b, 0, sizeof(*b));
}
