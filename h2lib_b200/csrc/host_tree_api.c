/* C-ABI wrappers of the host-side trees (no GPU involved). */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "h2b200_tree.h"

int h2b_ctree_build(uint32_t vertices, const double *x, uint32_t triangles, const uint32_t *t,
                    int basis, uint32_t clf, h2b_ctree *out);
int h2b_blist_build(const h2b_ctree *rt, const h2b_ctree *ct, double eta, h2b_blist *out);

/* Block counts of a complete tree (also used by the device builder, devtree.cu). */
int h2b_tree_finish(h2b_tree *tr);

static int
finish_tree(h2b_tree *tr)
{
  uint32_t i;
  uint64_t near = 0, adm = 0;
  for (i = 0; i < tr->blocks.n; i++) {
    if (tr->blocks.adm[i])
      adm++;
    else
      near += (uint64_t) tr->row.size[tr->blocks.rc[i]] * tr->col.size[tr->blocks.cc[i]];
  }
  tr->near_entries = near;
  tr->admissible = adm;
  return H2B_OK;
}

static int ctree_append(h2b_ctree *dst, const h2b_ctree *src, uint32_t ioff);

int
h2b_tree_finish(h2b_tree *tr)
{
  return finish_tree(tr);
}

/* dst (empty) = a copy of src (also used by the device builder for equal bases). */
int h2b_ctree_copy(h2b_ctree *dst, const h2b_ctree *src);
int
h2b_ctree_copy(h2b_ctree *dst, const h2b_ctree *src)
{
  return ctree_append(dst, src, 0);
}

h2b_tree *
h2b_tree_new(uint32_t vertices, const double *x, uint32_t triangles, const uint32_t *t,
             int row_basis, int col_basis, uint32_t clf, double eta)
{
  h2b_tree *tr;
  if (!x || !t || vertices == 0 || triangles == 0) {
    h2b_set_error("h2b_tree_new: empty mesh");
    return NULL;
  }
  if ((row_basis != H2B_BASIS_CONSTANT && row_basis != H2B_BASIS_LINEAR)
      || (col_basis != H2B_BASIS_CONSTANT && col_basis != H2B_BASIS_LINEAR) || !(eta > 0.0)) {
    h2b_set_error("h2b_tree_new: invalid basis or eta");
    return NULL;
  }
  tr = (h2b_tree *) calloc(1, sizeof(h2b_tree));
  if (!tr) {
    h2b_set_error("h2b_tree_new: out of host memory");
    return NULL;
  }
  tr->row_basis = row_basis;
  tr->col_basis = col_basis;
  /* equal bases give equal trees: build the row tree once and copy it */
  if (h2b_ctree_build(vertices, x, triangles, t, row_basis, clf, &tr->row) != H2B_OK
      || (col_basis == row_basis ? ctree_append(&tr->col, &tr->row, 0)
                                 : h2b_ctree_build(vertices, x, triangles, t, col_basis, clf,
                                                   &tr->col)) != H2B_OK
      || h2b_blist_build(&tr->row, &tr->col, eta, &tr->blocks) != H2B_OK) {
    h2b_tree_del(tr);
    return NULL;
  }
  finish_tree(tr);
  return tr;
}

/* Append the clusters of `src` to `dst` with cluster ids shifted by dst->n, index positions by
 * dst->nidx and index values by `ioff`. */
static int
ctree_append(h2b_ctree *dst, const h2b_ctree *src, uint32_t ioff)
{
  const uint32_t c0 = dst->n, i0 = dst->nidx, n = dst->n + src->n, ni = dst->nidx + src->nidx;
  uint32_t i;
#define H2B_RE(f, type, cnt)                                                   \
  do {                                                                        \
    type *p_ = (type *) realloc(dst->f, sizeof(type) * (size_t) (cnt));      \
    if (!p_)                                                                  \
      return H2B_ERR_NOMEM;                                                   \
    dst->f = p_;                                                              \
  } while (0)
  H2B_RE(off, uint32_t, n); H2B_RE(size, uint32_t, n); H2B_RE(sons, uint32_t, n);
  H2B_RE(son0, uint32_t, n); H2B_RE(son1, uint32_t, n); H2B_RE(father, uint32_t, n);
  H2B_RE(level, uint32_t, n); H2B_RE(bmin, double, 3 * (size_t) n);
  H2B_RE(bmax, double, 3 * (size_t) n); H2B_RE(idx, uint32_t, ni);
#undef H2B_RE
  for (i = 0; i < src->n; i++) {
    dst->off[c0 + i] = src->off[i] + i0;
    dst->size[c0 + i] = src->size[i];
    dst->sons[c0 + i] = src->sons[i];
    dst->son0[c0 + i] = src->son0[i] == UINT32_MAX ? UINT32_MAX : src->son0[i] + c0;
    dst->son1[c0 + i] = src->son1[i] == UINT32_MAX ? UINT32_MAX : src->son1[i] + c0;
    dst->father[c0 + i] = src->father[i] == UINT32_MAX ? UINT32_MAX : src->father[i] + c0;
    dst->level[c0 + i] = src->level[i];
  }
  memcpy(dst->bmin + 3 * (size_t) c0, src->bmin, sizeof(double) * 3 * src->n);
  memcpy(dst->bmax + 3 * (size_t) c0, src->bmax, sizeof(double) * 3 * src->n);
  for (i = 0; i < src->nidx; i++)
    dst->idx[i0 + i] = src->idx[i] + ioff;
  dst->n = n;
  dst->nidx = ni;
  if (src->depth > dst->depth)
    dst->depth = src->depth;
  return H2B_OK;
}

/* One surface of a forest: its trees, built with local vertex ids, are filled in by a worker
 * thread; the surfaces are independent, so any number of threads gives the same forest. */
typedef struct {
  uint32_t surfaces;
  const uint32_t *vertex_off, *triangle_off, *t;
  const double *x;
  int row_basis, col_basis;
  uint32_t clf;
  double eta;
  h2b_tree *ones;
  int *rc;
  uint32_t next;
} forest_job;

static int
forest_one(forest_job *j, uint32_t m, uint32_t **tl, size_t *tcap)
{
  const uint32_t v0 = j->vertex_off[m], nv = j->vertex_off[m + 1] - v0;
  const uint32_t t0 = j->triangle_off[m], nt = j->triangle_off[m + 1] - t0;
  h2b_tree *one = &j->ones[m];
  size_t i;
  int rc;
  if (3 * (size_t) nt > *tcap) {
    uint32_t *p = (uint32_t *) realloc(*tl, sizeof(uint32_t) * 3 * (size_t) nt);
    if (!p)
      return H2B_ERR_NOMEM;
    *tl = p;
    *tcap = 3 * (size_t) nt;
  }
  for (i = 0; i < 3 * (size_t) nt; i++)
    (*tl)[i] = j->t[3 * (size_t) t0 + i] - v0;
  rc = h2b_ctree_build(nv, j->x + 3 * (size_t) v0, nt, *tl, j->row_basis, j->clf, &one->row);
  /* equal bases give equal trees, as in h2b_tree_new */
  if (rc == H2B_OK)
    rc = j->col_basis == j->row_basis
             ? ctree_append(&one->col, &one->row, 0)
             : h2b_ctree_build(nv, j->x + 3 * (size_t) v0, nt, *tl, j->col_basis, j->clf,
                               &one->col);
  if (rc == H2B_OK)
    rc = h2b_blist_build(&one->row, &one->col, j->eta, &one->blocks);
  return rc;
}

static void *
forest_worker(void *arg)
{
  forest_job *j = (forest_job *) arg;
  uint32_t *tl = NULL;
  size_t tcap = 0;
  for (;;) {
    const uint32_t m = __atomic_fetch_add(&j->next, 1u, __ATOMIC_RELAXED);
    if (m >= j->surfaces)
      break;
    j->rc[m] = forest_one(j, m, &tl, &tcap);
  }
  free(tl);
  return NULL;
}

/* Host threads for the per-surface builds: the online cores, at most 32 and one per surface. */
static uint32_t
forest_threads(uint32_t surfaces)
{
  long c = sysconf(_SC_NPROCESSORS_ONLN);
  uint32_t n = c > 0 ? (uint32_t) c : 1u;
  if (n > 32u)
    n = 32u;
  return n < surfaces ? n : surfaces;
}

/* Append surface m's trees (already built) to the forest. */
static int
forest_append(h2b_tree *tr, const h2b_tree *one, uint32_t v0, uint32_t t0)
{
  const uint32_t rc0 = tr->row.n, cc0 = tr->col.n, b0 = tr->blocks.n;
  const uint32_t nb = b0 + one->blocks.n;
  uint32_t i;
  uint32_t *prc, *pcc;
  uint8_t *padm;
  int rc = ctree_append(&tr->row, &one->row, tr->row_basis == H2B_BASIS_LINEAR ? v0 : t0);
  if (rc == H2B_OK)
    rc = ctree_append(&tr->col, &one->col, tr->col_basis == H2B_BASIS_LINEAR ? v0 : t0);
  if (rc != H2B_OK)
    return rc;
  prc = (uint32_t *) realloc(tr->blocks.rc, sizeof(uint32_t) * nb);
  if (prc)
    tr->blocks.rc = prc;
  pcc = prc ? (uint32_t *) realloc(tr->blocks.cc, sizeof(uint32_t) * nb) : NULL;
  if (pcc)
    tr->blocks.cc = pcc;
  padm = pcc ? (uint8_t *) realloc(tr->blocks.adm, nb) : NULL;
  if (padm)
    tr->blocks.adm = padm;
  if (!prc || !pcc || !padm)
    return H2B_ERR_NOMEM;
  for (i = 0; i < one->blocks.n; i++) {
    tr->blocks.rc[b0 + i] = one->blocks.rc[i] + rc0;
    tr->blocks.cc[b0 + i] = one->blocks.cc[i] + cc0;
    tr->blocks.adm[b0 + i] = one->blocks.adm[i];
  }
  tr->blocks.n = nb;
  return H2B_OK;
}

h2b_tree *
h2b_tree_new_forest(uint32_t surfaces, const uint32_t *vertex_off, const uint32_t *triangle_off,
                    const double *x, const uint32_t *t, int row_basis, int col_basis, uint32_t clf,
                    double eta)
{
  h2b_tree *tr;
  forest_job job;
  pthread_t *th = NULL;
  uint32_t m, i, nth, started = 0, bad = 0;
  int rc = H2B_OK;
  if (!vertex_off || !triangle_off || !x || !t || surfaces == 0) {
    h2b_set_error("h2b_tree_new_forest: empty input");
    return NULL;
  }
  if ((row_basis != H2B_BASIS_CONSTANT && row_basis != H2B_BASIS_LINEAR)
      || (col_basis != H2B_BASIS_CONSTANT && col_basis != H2B_BASIS_LINEAR) || !(eta > 0.0)) {
    h2b_set_error("h2b_tree_new_forest: invalid basis or eta");
    return NULL;
  }
  if (clf == 0) {
    h2b_set_error("h2b_tree_new_forest: leaf size must be >= 1");
    return NULL;
  }
  /* every surface is checked here, before any thread starts, so each error names its surface */
  for (m = 0; m < surfaces; m++) {
    const uint32_t v0 = vertex_off[m], nv = vertex_off[m + 1] - vertex_off[m];
    const uint32_t t0 = triangle_off[m], nt = triangle_off[m + 1] - triangle_off[m];
    if (vertex_off[m + 1] < vertex_off[m] || triangle_off[m + 1] < triangle_off[m] || nv == 0
        || nt == 0) {
      h2b_set_error("h2b_tree_new_forest: surface %u is empty or its offsets decrease", m);
      return NULL;
    }
    for (i = 0; i < 3 * nt; i++) {
      const uint32_t v = t[3 * (size_t) t0 + i];
      if (v < v0 || v >= v0 + nv) {
        h2b_set_error("h2b_tree_new_forest: triangle %u of surface %u has a vertex outside it",
                      t0 + i / 3, m);
        return NULL;
      }
    }
  }
  tr = (h2b_tree *) calloc(1, sizeof(h2b_tree));
  memset(&job, 0, sizeof(job));
  job.ones = (h2b_tree *) calloc(surfaces, sizeof(h2b_tree));
  job.rc = (int *) calloc(surfaces, sizeof(int));
  nth = forest_threads(surfaces);
  if (nth > 1)
    th = (pthread_t *) malloc(sizeof(pthread_t) * (nth - 1));
  if (!tr || !job.ones || !job.rc) {
    free(th);
    free(job.rc);
    free(job.ones);
    free(tr);
    h2b_set_error("h2b_tree_new_forest: out of host memory");
    return NULL;
  }
  tr->row_basis = row_basis;
  tr->col_basis = col_basis;
  job.surfaces = surfaces;
  job.vertex_off = vertex_off;
  job.triangle_off = triangle_off;
  job.t = t;
  job.x = x;
  job.row_basis = row_basis;
  job.col_basis = col_basis;
  job.clf = clf;
  job.eta = eta;
  /* the calling thread works too; a thread that cannot start leaves its share to the others */
  for (i = 0; th && i + 1 < nth; i++)
    if (pthread_create(&th[started], NULL, forest_worker, &job) == 0)
      started++;
  forest_worker(&job);
  for (i = 0; i < started; i++)
    pthread_join(th[i], NULL);
  free(th);
  for (m = 0; m < surfaces; m++) {
    if (rc == H2B_OK) {
      rc = job.rc[m];
      if (rc == H2B_OK)
        rc = forest_append(tr, &job.ones[m], vertex_off[m], triangle_off[m]);
      if (rc != H2B_OK)
        bad = m;
    }
    h2b_ctree_free(&job.ones[m].row);
    h2b_ctree_free(&job.ones[m].col);
    h2b_blist_free(&job.ones[m].blocks);
  }
  free(job.rc);
  free(job.ones);
  if (rc != H2B_OK) {
    h2b_tree_del(tr);
    if (rc == H2B_ERR_NOMEM)
      h2b_set_error("h2b_tree_new_forest: out of host memory at surface %u", bad);
    else
      h2b_set_error("h2b_tree_new_forest: the trees of surface %u failed (code %d)", bad, rc);
    return NULL;
  }
  finish_tree(tr);
  return tr;
}

/* Rebuild son/father/level links of a pre-order tree given only (off, size, sons). */
static int
link_tree(h2b_ctree *t)
{
  uint32_t *stack, sp = 0, i;
  stack = (uint32_t *) malloc(sizeof(uint32_t) * (t->n + 1));
  if (!stack)
    return H2B_ERR_NOMEM;
  t->depth = 0;
  for (i = 0; i < t->n; i++) {
    t->son0[i] = t->son1[i] = UINT32_MAX;
    t->father[i] = UINT32_MAX;
    t->level[i] = 0;
  }
  /* pre-order: the first son of i is i+1; the second son follows the first son's subtree */
  for (i = 0; i < t->n; i++) {
    if (i > 0) {
      /* pop completed fathers: a father is complete when all its sons have been seen */
      while (sp > 0) {
        uint32_t f = stack[sp - 1];
        uint32_t have = (t->son0[f] != UINT32_MAX) + (t->son1[f] != UINT32_MAX);
        if (have < t->sons[f])
          break;
        sp--;
      }
      if (sp == 0) {
        free(stack);
        return H2B_ERR_ARG;
      }
      {
        uint32_t f = stack[sp - 1];
        if (t->son0[f] == UINT32_MAX)
          t->son0[f] = i;
        else
          t->son1[f] = i;
        t->father[i] = f;
        t->level[i] = t->level[f] + 1;
      }
    }
    if (t->level[i] + 1 > t->depth)
      t->depth = t->level[i] + 1;
    if (t->sons[i] > 0) {
      if (t->sons[i] != 2) {
        free(stack);
        return H2B_ERR_ARG;
      }
      stack[sp++] = i;
    }
  }
  free(stack);
  return H2B_OK;
}

static int
copy_flat(h2b_ctree *t, uint32_t nc, const uint32_t *off, const uint32_t *size,
          const uint32_t *sons, const double *box, uint32_t n, const uint32_t *idx)
{
  uint32_t i;
  memset(t, 0, sizeof(*t));
  t->n = nc;
  t->nidx = n;
  t->off = malloc(sizeof(uint32_t) * nc);
  t->size = malloc(sizeof(uint32_t) * nc);
  t->sons = malloc(sizeof(uint32_t) * nc);
  t->son0 = malloc(sizeof(uint32_t) * nc);
  t->son1 = malloc(sizeof(uint32_t) * nc);
  t->father = malloc(sizeof(uint32_t) * nc);
  t->level = malloc(sizeof(uint32_t) * nc);
  t->bmin = malloc(sizeof(double) * 3 * nc);
  t->bmax = malloc(sizeof(double) * 3 * nc);
  t->idx = malloc(sizeof(uint32_t) * (n ? n : 1));
  if (!t->off || !t->size || !t->sons || !t->son0 || !t->son1 || !t->father || !t->level
      || !t->bmin || !t->bmax || !t->idx)
    return H2B_ERR_NOMEM;
  memcpy(t->off, off, sizeof(uint32_t) * nc);
  memcpy(t->size, size, sizeof(uint32_t) * nc);
  memcpy(t->sons, sons, sizeof(uint32_t) * nc);
  memcpy(t->idx, idx, sizeof(uint32_t) * n);
  for (i = 0; i < nc; i++) {
    memcpy(t->bmin + 3 * i, box + 6 * (size_t) i, sizeof(double) * 3);
    memcpy(t->bmax + 3 * i, box + 6 * (size_t) i + 3, sizeof(double) * 3);
    if ((uint64_t) off[i] + size[i] > n)
      return H2B_ERR_ARG;
  }
  return link_tree(t);
}

h2b_tree *
h2b_tree_new_flat(uint32_t row_clusters, const uint32_t *row_off, const uint32_t *row_size,
                  const uint32_t *row_sons, const double *row_box, uint32_t row_n,
                  const uint32_t *row_idx, uint32_t col_clusters, const uint32_t *col_off,
                  const uint32_t *col_size, const uint32_t *col_sons, const double *col_box,
                  uint32_t col_n, const uint32_t *col_idx, uint32_t blocks,
                  const uint32_t *block_rc, const uint32_t *block_cc, const uint8_t *block_adm)
{
  h2b_tree *tr;
  uint32_t i;
  if (!row_clusters || !col_clusters || !blocks || !row_off || !row_size || !row_sons
      || !row_box || !row_idx || !col_off || !col_size || !col_sons || !col_box || !col_idx
      || !block_rc || !block_cc || !block_adm) {
    h2b_set_error("h2b_tree_new_flat: empty tree or NULL array");
    return NULL;
  }
  tr = (h2b_tree *) calloc(1, sizeof(h2b_tree));
  if (!tr) {
    h2b_set_error("h2b_tree_new_flat: out of host memory");
    return NULL;
  }
  tr->row_basis = tr->col_basis = 0;
  if (copy_flat(&tr->row, row_clusters, row_off, row_size, row_sons, row_box, row_n, row_idx)
      || copy_flat(&tr->col, col_clusters, col_off, col_size, col_sons, col_box, col_n,
                   col_idx)) {
    h2b_tree_del(tr);
    h2b_set_error("h2b_tree_new_flat: malformed cluster tree (pre-order, 0 or 2 sons)");
    return NULL;
  }
  tr->blocks.n = blocks;
  tr->blocks.rc = malloc(sizeof(uint32_t) * blocks);
  tr->blocks.cc = malloc(sizeof(uint32_t) * blocks);
  tr->blocks.adm = malloc(blocks);
  if (!tr->blocks.rc || !tr->blocks.cc || !tr->blocks.adm) {
    h2b_tree_del(tr);
    h2b_set_error("h2b_tree_new_flat: out of host memory");
    return NULL;
  }
  for (i = 0; i < blocks; i++) {
    if (block_rc[i] >= row_clusters || block_cc[i] >= col_clusters) {
      h2b_tree_del(tr);
      h2b_set_error("h2b_tree_new_flat: block %u references a missing cluster", i);
      return NULL;
    }
    tr->blocks.rc[i] = block_rc[i];
    tr->blocks.cc[i] = block_cc[i];
    tr->blocks.adm[i] = block_adm[i] ? 1 : 0;
    if (!block_adm[i] && (tr->row.sons[block_rc[i]] || tr->col.sons[block_cc[i]])) {
      /* strict block trees only: nearfield blocks between leaves */
      h2b_tree_del(tr);
      h2b_set_error("h2b_tree_new_flat: inadmissible block %u is not a leaf-leaf block", i);
      return NULL;
    }
  }
  finish_tree(tr);
  return tr;
}

void
h2b_tree_del(h2b_tree *tree)
{
  if (!tree)
    return;
  h2b_ctree_free(&tree->row);
  h2b_ctree_free(&tree->col);
  h2b_blist_free(&tree->blocks);
  free(tree);
}

int
h2b_tree_info(const h2b_tree *tree, uint64_t info[8])
{
  if (!tree || !info) {
    h2b_set_error("h2b_tree_info: NULL argument");
    return H2B_ERR_ARG;
  }
  info[0] = tree->row.n;
  info[1] = tree->col.n;
  info[2] = tree->row.nidx;
  info[3] = tree->col.nidx;
  info[4] = tree->blocks.n;
  info[5] = tree->admissible;
  info[6] = tree->near_entries;
  info[7] = (uint64_t) tree->row.depth | ((uint64_t) tree->col.depth << 32);
  return H2B_OK;
}

int
h2b_tree_export_clusters(const h2b_tree *tree, int which, uint32_t *rec, double *box,
                         uint32_t *idx)
{
  const h2b_ctree *t;
  uint32_t i;
  if (!tree || (which != 0 && which != 1)) {
    h2b_set_error("h2b_tree_export_clusters: bad argument");
    return H2B_ERR_ARG;
  }
  t = which ? &tree->col : &tree->row;
  for (i = 0; i < t->n; i++) {
    if (rec) {
      rec[3 * i] = t->off[i];
      rec[3 * i + 1] = t->size[i];
      rec[3 * i + 2] = t->sons[i];
    }
    if (box) {
      memcpy(box + 6 * (size_t) i, t->bmin + 3 * (size_t) i, sizeof(double) * 3);
      memcpy(box + 6 * (size_t) i + 3, t->bmax + 3 * (size_t) i, sizeof(double) * 3);
    }
  }
  if (idx)
    memcpy(idx, t->idx, sizeof(uint32_t) * t->nidx);
  return H2B_OK;
}

int
h2b_tree_export_blocks(const h2b_tree *tree, uint32_t *rec)
{
  uint32_t i;
  if (!tree || !rec) {
    h2b_set_error("h2b_tree_export_blocks: NULL argument");
    return H2B_ERR_ARG;
  }
  for (i = 0; i < tree->blocks.n; i++) {
    uint32_t r = tree->blocks.rc[i], c = tree->blocks.cc[i];
    rec[5 * i] = tree->row.off[r];
    rec[5 * i + 1] = tree->row.size[r];
    rec[5 * i + 2] = tree->col.off[c];
    rec[5 * i + 3] = tree->col.size[c];
    rec[5 * i + 4] = tree->blocks.adm[i];
  }
  return H2B_OK;
}
