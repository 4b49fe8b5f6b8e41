/* Golden-vector generator: runs the unmodified H2Lib reference (compiled from its own sources into
 * oracle/_ref/libh2ref_{real,complex}.so by oracle/Makefile) on the synthetic inputs the tests use,
 * and writes raw arrays plus a manifest into an output directory.  make_golden.py drives it and
 * packs the arrays into the committed .npz fixtures.
 *
 * Built twice: without USE_COMPLEX (Laplace, real field) and with it (Helmholtz, complex field).
 *
 * Usage: gen_golden <outdir> <section> [...]
 * Sections (real build):    quad sphere8 sphere4 h2small config2 cube adlp green
 * Sections (complex build): helm_sphere4 helm_h2small config3 config3_k8 helm_gmres helm_adlp
 *                           helm_point
 * The complex build also links the reference's Tests/test_helmholtzbem3d.c (its main renamed) for
 * that test's evaluation of the exterior field.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "basic.h"
#include "bem3d.h"
#include "block.h"
#include "cluster.h"
#include "clusterbasis.h"
#include "gaussquad.h"
#include "h2matrix.h"
#include "krylovsolvers.h"
#include "laplacebem3d.h"
#include "macrosurface3d.h"
#include "singquad2d.h"
#include "surface3d.h"
#ifdef USE_COMPLEX
#include "helmholtzbem3d.h"
#endif

static const char *outdir;
static FILE *manifest;

/* ---------- raw array writer ---------- */

static void
dump(const char *name, const char *dtype, size_t esize, const void *data, int ndim,
     size_t d0, size_t d1)
{
  char path[4096];
  size_t n = (ndim == 1 ? d0 : d0 * d1);
  FILE *f;

  snprintf(path, sizeof(path), "%s/%s.bin", outdir, name);
  f = fopen(path, "wb");
  if (!f) {
    perror(path);
    exit(1);
  }
  if (n > 0 && fwrite(data, esize, n, f) != n) {
    perror(path);
    exit(1);
  }
  fclose(f);
  if (ndim == 1)
    fprintf(manifest, "%s %s %zu\n", name, dtype, d0);
  else
    fprintf(manifest, "%s %s %zu %zu\n", name, dtype, d0, d1);
  fflush(manifest);
}

static void
dump_real(const char *name, const real *v, int ndim, size_t d0, size_t d1)
{
  dump(name, "f8", sizeof(real), v, ndim, d0, d1);
}

static void
dump_uint(const char *name, const uint *v, int ndim, size_t d0, size_t d1)
{
  dump(name, "u4", sizeof(uint), v, ndim, d0, d1);
}

static void
dump_scalar(const char *name, double v)
{
  dump(name, "f8", sizeof(double), &v, 1, 1, 0);
}

/* Matrix stored column-major with ld: written as (cols, rows) C-order == column-major contiguous. */
static void
dump_amatrix(const char *name, pcamatrix A)
{
  size_t rows = A->rows, cols = A->cols, j;
  field *buf = (field *) malloc(sizeof(field) * (rows * cols + 1));

  for (j = 0; j < cols; j++)
    memcpy(buf + j * rows, A->a + j * A->ld, sizeof(field) * rows);
#ifdef USE_COMPLEX
  dump(name, "c16", sizeof(field), buf, 2, cols, rows);
#else
  dump(name, "f8", sizeof(field), buf, 2, cols, rows);
#endif
  free(buf);
}

static void
dump_avector(const char *name, pcavector v)
{
#ifdef USE_COMPLEX
  dump(name, "c16", sizeof(field), v->v, 1, v->dim, 0);
#else
  dump(name, "f8", sizeof(field), v->v, 1, v->dim, 0);
#endif
}

static void
dump_mesh(const char *prefix, pcsurface3d gr)
{
  char name[256];

  snprintf(name, sizeof(name), "%s_x", prefix);
  dump_real(name, &gr->x[0][0], 2, gr->vertices, 3);
  snprintf(name, sizeof(name), "%s_t", prefix);
  dump_uint(name, &gr->t[0][0], 2, gr->triangles, 3);
  snprintf(name, sizeof(name), "%s_n", prefix);
  dump_real(name, &gr->n[0][0], 2, gr->triangles, 3);
  snprintf(name, sizeof(name), "%s_g", prefix);
  dump_real(name, gr->g, 1, gr->triangles, 0);
  snprintf(name, sizeof(name), "%s_h", prefix);
  {
    real h[2] = { gr->hmin, gr->hmax };
    dump_real(name, h, 1, 2, 0);
  }
}

/* Deterministic test vector (stored in the fixture, so no bitwise libm agreement is needed). */
static void
seeded_avector(pavector x, uint salt)
{
  uint i;
  for (i = 0; i < x->dim; i++) {
    real re = sin(0.37 * i + 0.1 * salt) + 0.5 * cos(1.3 * i + 0.7);
#ifdef USE_COMPLEX
    real im = cos(0.21 * i + 0.3 * salt) - 0.25 * sin(2.1 * i);
    x->v[i] = re + im * I;
#else
    x->v[i] = re;
#endif
  }
}

/* ---------- cluster / block tree flattening ---------- */

typedef struct {
  uint n, cap;
  uint *rec;   /* per cluster: offset, size, sons */
  real *box;   /* per cluster: bmin[3], bmax[3] */
} ctree_t;

static void
flatten_cluster(pccluster t, const uint *root_idx, ctree_t *ct)
{
  uint i;
  if (ct->n == ct->cap) {
    ct->cap = ct->cap ? 2 * ct->cap : 256;
    ct->rec = realloc(ct->rec, sizeof(uint) * 3 * ct->cap);
    ct->box = realloc(ct->box, sizeof(real) * 6 * ct->cap);
  }
  ct->rec[3 * ct->n + 0] = (uint) (t->idx - root_idx);
  ct->rec[3 * ct->n + 1] = t->size;
  ct->rec[3 * ct->n + 2] = t->sons;
  for (i = 0; i < 3; i++) {
    ct->box[6 * ct->n + i] = t->bmin[i];
    ct->box[6 * ct->n + 3 + i] = t->bmax[i];
  }
  ct->n++;
  for (i = 0; i < t->sons; i++)
    flatten_cluster(t->son[i], root_idx, ct);
}

static void
dump_cluster(const char *prefix, pccluster root)
{
  ctree_t ct = { 0, 0, NULL, NULL };
  char name[256];

  flatten_cluster(root, root->idx, &ct);
  snprintf(name, sizeof(name), "%s_ctree", prefix);
  dump_uint(name, ct.rec, 2, ct.n, 3);
  snprintf(name, sizeof(name), "%s_cbox", prefix);
  dump_real(name, ct.box, 2, ct.n, 6);
  snprintf(name, sizeof(name), "%s_idx", prefix);
  dump_uint(name, root->idx, 1, root->size, 0);
  free(ct.rec);
  free(ct.box);
}

typedef struct {
  uint n, cap;
  uint *rec;   /* per leaf block: rc offset, rc size, cc offset, cc size, admissible */
} btree_t;

static void
flatten_block(pcblock b, const uint *ridx0, const uint *cidx0, btree_t *bt)
{
  uint i, j;
  if (b->son == NULL) {
    if (bt->n == bt->cap) {
      bt->cap = bt->cap ? 2 * bt->cap : 1024;
      bt->rec = realloc(bt->rec, sizeof(uint) * 5 * bt->cap);
    }
    bt->rec[5 * bt->n + 0] = (uint) (b->rc->idx - ridx0);
    bt->rec[5 * bt->n + 1] = b->rc->size;
    bt->rec[5 * bt->n + 2] = (uint) (b->cc->idx - cidx0);
    bt->rec[5 * bt->n + 3] = b->cc->size;
    bt->rec[5 * bt->n + 4] = b->a ? 1 : 0;
    bt->n++;
    return;
  }
  for (j = 0; j < b->csons; j++)
    for (i = 0; i < b->rsons; i++)
      flatten_block(b->son[i + j * b->rsons], ridx0, cidx0, bt);
}

static void
dump_block(const char *prefix, pcblock b, pccluster rroot, pccluster croot)
{
  btree_t bt = { 0, 0, NULL };
  char name[256];

  flatten_block(b, rroot->idx, croot->idx, &bt);
  snprintf(name, sizeof(name), "%s_blocks", prefix);
  dump_uint(name, bt.rec, 2, bt.n, 5);
  free(bt.rec);
}

/* Leaf bases V and transfer matrices E of a cluster basis, pre-order, concatenated. */
typedef struct {
  size_t n, cap;
  field *v;
} fbuf_t;

static void
fbuf_push(fbuf_t *b, pcamatrix A)
{
  size_t need = (size_t) A->rows * A->cols, j;
  if (b->n + need > b->cap) {
    b->cap = (b->n + need) * 2 + 1024;
    b->v = realloc(b->v, sizeof(field) * b->cap);
  }
  for (j = 0; j < A->cols; j++)
    memcpy(b->v + b->n + j * A->rows, A->a + j * A->ld, sizeof(field) * A->rows);
  b->n += need;
}

static void
collect_basis(pcclusterbasis cb, fbuf_t *V, fbuf_t *E, int is_root)
{
  uint i;
  if (!is_root)
    fbuf_push(E, &cb->E);
  if (cb->sons == 0)
    fbuf_push(V, &cb->V);
  for (i = 0; i < cb->sons; i++)
    collect_basis(cb->son[i], V, E, 0);
}

static void
dump_basis(const char *prefix, pcclusterbasis cb)
{
  fbuf_t V = { 0, 0, NULL }, E = { 0, 0, NULL };
  char name[256];
  collect_basis(cb, &V, &E, 1);
#ifdef USE_COMPLEX
  const char *dt = "c16";
#else
  const char *dt = "f8";
#endif
  snprintf(name, sizeof(name), "%s_V", prefix);
  dump(name, dt, sizeof(field), V.v, 1, V.n, 0);
  snprintf(name, sizeof(name), "%s_E", prefix);
  dump(name, dt, sizeof(field), E.v, 1, E.n, 0);
  free(V.v);
  free(E.v);
}

/* Coupling matrices of the first `limit` admissible leaves (block-tree pre-order). */
static void
collect_coupling(pch2matrix G, fbuf_t *S, uint *count, uint limit)
{
  uint i, j;
  if (*count >= limit)
    return;
  if (G->u) {
    fbuf_push(S, &G->u->S);
    (*count)++;
    return;
  }
  if (G->son)
    for (j = 0; j < G->csons; j++)
      for (i = 0; i < G->rsons; i++)
        collect_coupling(G->son[i + j * G->rsons], S, count, limit);
}

/* Nearfield matrices of the first `limit` inadmissible leaves (block-tree pre-order). */
static void
collect_near(pch2matrix G, fbuf_t *N, uint *count, uint limit)
{
  uint i, j;
  if (*count >= limit)
    return;
  if (G->f) {
    fbuf_push(N, G->f);
    (*count)++;
    return;
  }
  if (G->son)
    for (j = 0; j < G->csons; j++)
      for (i = 0; i < G->rsons; i++)
        collect_near(G->son[i + j * G->rsons], N, count, limit);
}

/* The nearfield leaves in block-tree pre-order (sons column-major), as a flat list. */
typedef struct {
  pch2matrix *b;
  uint n, cap;
} nearlist_t;

static void
list_near(pch2matrix G, nearlist_t *l)
{
  uint i, j;
  if (G->f) {
    if (l->n == l->cap) {
      l->cap = l->cap ? 2 * l->cap : 1024;
      l->b = realloc(l->b, sizeof(pch2matrix) * l->cap);
    }
    l->b[l->n++] = G;
    return;
  }
  if (G->son)
    for (j = 0; j < G->csons; j++)
      for (i = 0; i < G->rsons; i++)
        list_near(G->son[i + j * G->rsons], l);
}

/* Three whole nearfield blocks of V and K for entrywise comparison: the largest block, the most
 * ragged one (largest |rows - cols|) and the largest diagonal one (row cluster == column
 * cluster).  <prefix>_nblk_idx holds their positions in the list of nearfield blocks. */
static void
dump_selected_near(const char *prefix, pch2matrix V, pch2matrix K)
{
  nearlist_t lv = { NULL, 0, 0 }, lk = { NULL, 0, 0 };
  uint sel[3] = { 0, 0, 0 }, i, s;
  size_t best[3] = { 0, 0, 0 };
  char name[256];
  list_near(V, &lv);
  list_near(K, &lk);
  for (i = 0; i < lv.n; i++) {
    pamatrix f = lv.b[i]->f;
    size_t sz = (size_t) f->rows * f->cols;
    size_t rag = f->rows > f->cols ? f->rows - f->cols : f->cols - f->rows;
    if (sz > best[0]) best[0] = sz, sel[0] = i;
    if (rag > best[1]) best[1] = rag, sel[1] = i;
    if (lv.b[i]->rb->t == lv.b[i]->cb->t && sz > best[2]) best[2] = sz, sel[2] = i;
  }
  snprintf(name, sizeof(name), "%s_nblk_idx", prefix);
  dump_uint(name, sel, 1, 3, 0);
  for (s = 0; s < 3; s++) {
    snprintf(name, sizeof(name), "%s_nblkV_%u", prefix, s);
    dump_amatrix(name, lv.b[sel[s]]->f);
    snprintf(name, sizeof(name), "%s_nblkK_%u", prefix, s);
    dump_amatrix(name, lk.b[sel[s]]->f);
  }
  free(lv.b);
  free(lk.b);
}

/* solve_gmres_avector (Library/krylovsolvers.c:183) with the same calls in the same order, also
 * recording the residual estimate |rhat_k| of every iteration: trace[0] after init_gmres,
 * trace[i] after step i.  The caller's trace array holds maxiter entries. */
static uint
solve_gmres_traced(void *A, addeval_t addeval_A, pcavector b, pavector x, real eps,
                   uint maxiter, uint kmax, real *trace, real *threshold)
{
  pavector rhat, q, tau;
  pamatrix qr;
  real norm, error;
  uint n = x->dim, iter, k;

  rhat = new_avector(n);
  q = new_avector(n);
  qr = new_amatrix(n, kmax);
  tau = new_avector(kmax);
  norm = norm2_avector(b);
  init_gmres(addeval_A, A, b, x, rhat, q, &k, qr, tau);
  error = residualnorm_gmres(rhat, k);
  trace[0] = error;
  iter = 0;
  while (error > eps * norm && iter + 1 != maxiter) {
    if (k + 1 >= kmax)
      finish_gmres(addeval_A, A, b, x, rhat, q, &k, qr, tau);
    step_gmres(addeval_A, A, b, x, rhat, q, &k, qr, tau);
    error = residualnorm_gmres(rhat, k);
    iter++;
    trace[iter] = error;
  }
  finish_gmres(addeval_A, A, b, x, rhat, q, &k, qr, tau);
  *threshold = eps * norm;
  del_avector(tau);
  del_amatrix(qr);
  del_avector(q);
  del_avector(rhat);
  return iter;
}

static void
dump_h2parts(const char *prefix, pch2matrix G, uint limit)
{
  fbuf_t S = { 0, 0, NULL }, N = { 0, 0, NULL };
  uint cnt = 0;
  char name[256];
#ifdef USE_COMPLEX
  const char *dt = "c16";
#else
  const char *dt = "f8";
#endif
  collect_coupling(G, &S, &cnt, limit);
  snprintf(name, sizeof(name), "%s_S", prefix);
  dump(name, dt, sizeof(field), S.v, 1, S.n, 0);
  cnt = 0;
  collect_near(G, &N, &cnt, limit);
  snprintf(name, sizeof(name), "%s_N", prefix);
  dump(name, dt, sizeof(field), N.v, 1, N.n, 0);
  free(S.v);
  free(N.v);
}

/* Dense nearfield matrix of an operator on the whole mesh (all pairs), and for the linear-linear
 * case a ragged sub-block and its transposed write. */
static void
dense_op(const char *prefix, psurface3d gr, pbem3d op, basisfunctionbem3d rb,
         basisfunctionbem3d cb, int with_block)
{
  uint n = (rb == BASIS_LINEAR_BEM3D) ? gr->vertices : gr->triangles;
  uint m = (cb == BASIS_LINEAR_BEM3D) ? gr->vertices : gr->triangles;
  pamatrix A = new_amatrix(n, m);
  char name[256];

  op->nearfield(NULL, NULL, op, false, A);
  dump_amatrix(prefix, A);
  del_amatrix(A);
  if (with_block) {
    uint ridx[7] = { 5, 9, 20, 33, 2, 61, 40 };
    uint cidx[5] = { 1, 40, 2, 60, 65 };
    pamatrix B = new_amatrix(7, 5), Bt = new_amatrix(5, 7);
    op->nearfield(ridx, cidx, op, false, B);
    snprintf(name, sizeof(name), "%s_block", prefix);
    dump_amatrix(name, B);
    op->nearfield(ridx, cidx, op, true, Bt);
    snprintf(name, sizeof(name), "%s_block_trans", prefix);
    dump_amatrix(name, Bt);
    del_amatrix(B);
    del_amatrix(Bt);
  }
}

/* H2 matrix of one operator on the mesh: trees, row and column bases, the first coupling and
 * nearfield blocks, and a matvec with a seeded vector. */
static void
h2_op(const char *prefix, psurface3d gr, pbem3d op, basisfunctionbem3d basis, uint clf,
      real eta, uint m, uint parts_limit)
{
  pcluster root;
  pblock broot;
  pclusterbasis rb, cb;
  ph2matrix G;
  pavector x, y;
  char name[256];

  root = build_bem3d_cluster(op, clf, basis);
  broot = build_strict_block(root, root, &eta, admissible_max_cluster);
  dump_cluster(prefix, root);
  dump_block(prefix, broot, root, root);
  rb = build_from_cluster_clusterbasis(root);
  cb = build_from_cluster_clusterbasis(root);
  G = build_from_block_h2matrix(broot, rb, cb);
  setup_h2matrix_aprx_inter_bem3d(op, rb, cb, broot, m);
  assemble_bem3d_h2matrix_row_clusterbasis(op, rb);
  assemble_bem3d_h2matrix_col_clusterbasis(op, cb);
  assemble_bem3d_h2matrix(op, G);
  snprintf(name, sizeof(name), "%s_row", prefix);
  dump_basis(name, rb);
  snprintf(name, sizeof(name), "%s_col", prefix);
  dump_basis(name, cb);
  snprintf(name, sizeof(name), "%s_parts", prefix);
  dump_h2parts(name, G, parts_limit);
  x = new_avector(G->cb->t->size);
  y = new_avector(G->rb->t->size);
  seeded_avector(x, 5);
  snprintf(name, sizeof(name), "%s_x", prefix);
  dump_avector(name, x);
  clear_avector(y);
  addeval_h2matrix_avector(1.0, G, x, y);
  snprintf(name, sizeof(name), "%s_y", prefix);
  dump_avector(name, y);
  del_avector(x);
  del_avector(y);
  del_h2matrix(G);
  del_block(broot);
  freemem(root->idx);
  del_cluster(root);
}

/* Ranks of a cluster basis, pre-order. */
static void
collect_ranks(pcclusterbasis cb, uint **r, uint *n, uint *cap)
{
  uint i;
  if (*n == *cap) {
    *cap = *cap ? 2 * *cap : 256;
    *r = realloc(*r, sizeof(uint) * *cap);
  }
  (*r)[(*n)++] = cb->k;
  for (i = 0; i < cb->sons; i++)
    collect_ranks(cb->son[i], r, n, cap);
}

static void
dump_ranks(const char *prefix, pcclusterbasis cb)
{
  uint *r = NULL, n = 0, cap = 0;
  collect_ranks(cb, &r, &n, &cap);
  dump_uint(prefix, r, 1, n, 0);
  free(r);
}

/* H2 matrix with the greenhybrid farfield (setup_h2matrix_aprx_greenhybrid_bem3d, cube quadrature
 * points): ranks, bases, the first coupling matrices and a matvec with a seeded vector. */
static void
green_op(const char *prefix, psurface3d gr, pbem3d op, basisfunctionbem3d basis, uint clf,
         real eta, uint m, uint l, real delta, real accur, uint parts_limit)
{
  pcluster root;
  pblock broot;
  pclusterbasis rb, cb;
  ph2matrix G;
  pavector x, y;
  char name[256];

  root = build_bem3d_cluster(op, clf, basis);
  broot = build_strict_block(root, root, &eta, admissible_max_cluster);
  dump_cluster(prefix, root);
  dump_block(prefix, broot, root, root);
  rb = build_from_cluster_clusterbasis(root);
  cb = build_from_cluster_clusterbasis(root);
  G = build_from_block_h2matrix(broot, rb, cb);
  setup_h2matrix_aprx_greenhybrid_bem3d(op, rb, cb, broot, m, l, delta, accur,
                                        build_bem3d_cube_quadpoints);
  assemble_bem3d_h2matrix_row_clusterbasis(op, rb);
  assemble_bem3d_h2matrix_col_clusterbasis(op, cb);
  assemble_bem3d_h2matrix(op, G);
  snprintf(name, sizeof(name), "%s_row_k", prefix);
  dump_ranks(name, rb);
  snprintf(name, sizeof(name), "%s_col_k", prefix);
  dump_ranks(name, cb);
  snprintf(name, sizeof(name), "%s_row", prefix);
  dump_basis(name, rb);
  snprintf(name, sizeof(name), "%s_col", prefix);
  dump_basis(name, cb);
  snprintf(name, sizeof(name), "%s_parts", prefix);
  dump_h2parts(name, G, parts_limit);
  x = new_avector(G->cb->t->size);
  y = new_avector(G->rb->t->size);
  seeded_avector(x, 5);
  snprintf(name, sizeof(name), "%s_x", prefix);
  dump_avector(name, x);
  clear_avector(y);
  addeval_h2matrix_avector(1.0, G, x, y);
  snprintf(name, sizeof(name), "%s_y", prefix);
  dump_avector(name, y);
  del_avector(x);
  del_avector(y);
  del_h2matrix(G);
  del_block(broot);
  freemem(root->idx);
  del_cluster(root);
}

/* ---------- sections ---------- */

#ifndef USE_COMPLEX

static void
section_quad(void)
{
  uint qs[4] = { 2, 3, 4, 5 }, i, j;
  char name[64];
  psingquad2d sq;
  pmacrosurface3d mg;
  psurface3d gr;

  for (i = 0; i < 4; i++) {
    real x[8], w[8];
    assemble_gauss(qs[i], x, w);
    for (j = 0; j < qs[i]; j++) {
      x[j] = 0.5 + 0.5 * x[j];
      w[j] = 0.5 * w[j];
    }
    snprintf(name, sizeof(name), "gauss%u_x", qs[i]);
    dump_real(name, x, 1, qs[i], 0);
    snprintf(name, sizeof(name), "gauss%u_w", qs[i]);
    dump_real(name, w, 1, qs[i], 0);
  }

  mg = new_sphere_macrosurface3d();
  gr = build_from_macrosurface3d_surface3d(mg, 2);
  sq = build_singquad2d(gr, 2, 4);
  /* VREAL == 1 in the scalar build, so vnq == n for every rule. */
  dump_real("dist_x", sq->x_dist, 2, 2, sq->n_dist);
  dump_real("dist_y", sq->y_dist, 2, 2, sq->n_dist);
  dump_real("dist_w", sq->w_dist + 9 * sq->n_dist, 1, sq->n_dist, 0);
  dump_real("vert_x", sq->x_vert, 2, 2, sq->n_vert);
  dump_real("vert_y", sq->y_vert, 2, 2, sq->n_vert);
  dump_real("vert_w", sq->w_vert + 9 * sq->n_vert, 1, sq->n_vert, 0);
  dump_real("edge_x", sq->x_edge, 2, 2, sq->n_edge);
  dump_real("edge_y", sq->y_edge, 2, 2, sq->n_edge);
  dump_real("edge_w", sq->w_edge + 9 * sq->n_edge, 1, sq->n_edge, 0);
  dump_real("id_x", sq->x_id, 2, 2, sq->n_id);
  dump_real("id_y", sq->y_id, 2, 2, sq->n_id);
  dump_real("id_w", sq->w_id + 9 * sq->n_id, 1, sq->n_id, 0);
  dump_real("single_x", sq->x_single, 1, sq->n_single, 0);
  dump_real("single_y", sq->y_single, 1, sq->n_single, 0);
  dump_real("single_w", sq->w_single + 3 * sq->n_single, 1, sq->n_single, 0);
  /* basis-weighted (ll) edge rule: all ten weight rows */
  weight_basisfunc_ll_singquad2d(sq->x_edge, sq->y_edge, sq->w_edge, sq->n_edge);
  dump_real("edge_w_ll", sq->w_edge, 2, 10, sq->n_edge);
  weight_basisfunc_l_singquad2d(sq->x_single, sq->y_single, sq->w_single, sq->n_single);
  dump_real("single_w_l", sq->w_single, 2, 4, sq->n_single);
  del_singquad2d(sq);
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

static void
dense_pair(const char *prefix, psurface3d gr, basisfunctionbem3d rb, basisfunctionbem3d cb,
           int with_block)
{
  pbem3d slp, dlp;
  pamatrix A;
  uint n = (rb == BASIS_LINEAR_BEM3D) ? gr->vertices : gr->triangles;
  uint m = (cb == BASIS_LINEAR_BEM3D) ? gr->vertices : gr->triangles;
  char name[256];

  slp = new_slp_laplace_bem3d(gr, 2, 4, rb, cb);
  dlp = new_dlp_laplace_bem3d(gr, 2, 4, rb, cb, 0.5);

  A = new_amatrix(n, m);
  slp->nearfield(NULL, NULL, slp, false, A);
  snprintf(name, sizeof(name), "%s_slp", prefix);
  dump_amatrix(name, A);
  dlp->nearfield(NULL, NULL, dlp, false, A);
  snprintf(name, sizeof(name), "%s_dlp", prefix);
  dump_amatrix(name, A);
  del_amatrix(A);

  if (with_block) {
    /* a ragged sub-block with non-contiguous, unsorted index lists */
    uint ridx[7] = { 5, 9, 20, 33, 2, 61, 40 };
    uint cidx[5] = { 1, 40, 2, 60, 65 };
    pamatrix B = new_amatrix(7, 5);
    slp->nearfield(ridx, cidx, slp, false, B);
    snprintf(name, sizeof(name), "%s_slp_block", prefix);
    dump_amatrix(name, B);
    dlp->nearfield(ridx, cidx, dlp, false, B);
    snprintf(name, sizeof(name), "%s_dlp_block", prefix);
    dump_amatrix(name, B);
    /* transposed write */
    {
      pamatrix Bt = new_amatrix(5, 7);
      dlp->nearfield(ridx, cidx, dlp, true, Bt);
      snprintf(name, sizeof(name), "%s_dlp_block_trans", prefix);
      dump_amatrix(name, Bt);
      del_amatrix(Bt);
    }
    dump_uint("block_ridx", ridx, 1, 7, 0);
    dump_uint("block_cidx", cidx, 1, 5, 0);
    del_amatrix(B);
  }
  del_laplace_bem3d(slp);
  del_laplace_bem3d(dlp);
}

static void
section_sphere8(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 8);
  pbem3d slp, dlp;
  pamatrix G;

  dump_mesh("sphere8", gr);
  /* config 1: assemble_bem3d_amatrix, cc, q=2/4 */
  slp = new_slp_laplace_bem3d(gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D);
  dlp = new_dlp_laplace_bem3d(gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D, 0.5);
  G = new_amatrix(gr->triangles, gr->triangles);
  assemble_bem3d_amatrix(slp, G);
  dump_amatrix("c1_slp", G);
  assemble_bem3d_amatrix(dlp, G);
  dump_amatrix("c1_dlp", G);
  del_amatrix(G);
  del_laplace_bem3d(slp);
  del_laplace_bem3d(dlp);
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

static void
section_sphere4(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 4);

  dump_mesh("sphere4", gr);
  dense_pair("s4cc", gr, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D, 0);
  dense_pair("s4ll", gr, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D, 1);
  dense_pair("s4cl", gr, BASIS_CONSTANT_BEM3D, BASIS_LINEAR_BEM3D, 0);
  dense_pair("s4lc", gr, BASIS_LINEAR_BEM3D, BASIS_CONSTANT_BEM3D, 0);
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

/* Full H2 pipeline on one mesh: trees, bases, coupling, nearfield, matvec. */
static void
h2_case(const char *prefix, psurface3d gr, basisfunctionbem3d basis, uint clf, real eta,
        uint m, uint parts_limit, int with_solve)
{
  pbem3d slp, dlp;
  pcluster root;
  pblock broot;
  pclusterbasis Vrb, Vcb, Krb, Kcb;
  ph2matrix V, K;
  pavector x, y;
  char name[256];
  double t0;
  pstopwatch sw = new_stopwatch();

  slp = new_slp_laplace_bem3d(gr, 2, 4, basis, basis);
  dlp = new_dlp_laplace_bem3d(gr, 2, 4, basis, basis, 0.5);
  root = build_bem3d_cluster(slp, clf, basis);
  broot = build_strict_block(root, root, &eta, admissible_max_cluster);
  snprintf(name, sizeof(name), "%s", prefix);
  dump_cluster(name, root);
  dump_block(name, broot, root, root);

  Vrb = build_from_cluster_clusterbasis(root);
  Vcb = build_from_cluster_clusterbasis(root);
  Krb = build_from_cluster_clusterbasis(root);
  Kcb = build_from_cluster_clusterbasis(root);
  V = build_from_block_h2matrix(broot, Vrb, Vcb);
  K = build_from_block_h2matrix(broot, Krb, Kcb);
  setup_h2matrix_aprx_inter_bem3d(slp, Vrb, Vcb, broot, m);
  setup_h2matrix_aprx_inter_bem3d(dlp, Krb, Kcb, broot, m);

  start_stopwatch(sw);
  assemble_bem3d_h2matrix_row_clusterbasis(slp, Vrb);
  assemble_bem3d_h2matrix_col_clusterbasis(slp, Vcb);
  assemble_bem3d_h2matrix(slp, V);
  t0 = stop_stopwatch(sw);
  snprintf(name, sizeof(name), "%s_time_slp_assembly", prefix);
  dump_scalar(name, t0);
  start_stopwatch(sw);
  assemble_bem3d_h2matrix_row_clusterbasis(dlp, Krb);
  assemble_bem3d_h2matrix_col_clusterbasis(dlp, Kcb);
  assemble_bem3d_h2matrix(dlp, K);
  t0 = stop_stopwatch(sw);
  snprintf(name, sizeof(name), "%s_time_dlp_assembly", prefix);
  dump_scalar(name, t0);

  if (parts_limit > 0) {
    snprintf(name, sizeof(name), "%s_Vrow", prefix);
    dump_basis(name, Vrb);
    snprintf(name, sizeof(name), "%s_Kcol", prefix);
    dump_basis(name, Kcb);
    snprintf(name, sizeof(name), "%s_Vparts", prefix);
    dump_h2parts(name, V, parts_limit);
    snprintf(name, sizeof(name), "%s_Kparts", prefix);
    dump_h2parts(name, K, parts_limit);
  }
  if (!strcmp(prefix, "c2"))
    dump_selected_near(prefix, V, K);

  x = new_avector(V->cb->t->size);
  y = new_avector(V->rb->t->size);
  seeded_avector(x, 1);
  snprintf(name, sizeof(name), "%s_x", prefix);
  dump_avector(name, x);
  clear_avector(y);
  start_stopwatch(sw);
  addeval_h2matrix_avector(1.0, V, x, y);
  t0 = stop_stopwatch(sw);
  snprintf(name, sizeof(name), "%s_time_matvec", prefix);
  dump_scalar(name, t0);
  snprintf(name, sizeof(name), "%s_ySLP", prefix);
  dump_avector(name, y);
  clear_avector(y);
  addeval_h2matrix_avector(1.0, K, x, y);
  snprintf(name, sizeof(name), "%s_yDLP", prefix);
  dump_avector(name, y);

  if (with_solve) {
    /* Interior Dirichlet problem: V u = (K + 1/2 M) g_D, GMRES(50) to 1e-8, start from zero. */
    pavector f = new_avector(x->dim), b = new_avector(x->dim), u = new_avector(x->dim);
    uint iter;
    real err, nrm;
    projectL2_bem3d_l_avector(dlp, eval_dirichlet_fundamental_laplacebem3d, f, NULL);
    snprintf(name, sizeof(name), "%s_gD", prefix);
    dump_avector(name, f);
    clear_avector(b);
    addeval_h2matrix_avector(1.0, K, f, b);
    snprintf(name, sizeof(name), "%s_b", prefix);
    dump_avector(name, b);
    clear_avector(u);
    {
      /* solve_gmres_h2matrix_avector (Library/krylovsolvers.c:254), with its residual trace */
      real *trace = (real *) calloc(1000, sizeof(real)), thr = 0.0;
      start_stopwatch(sw);
      iter = solve_gmres_traced(V, (addeval_t) addeval_h2matrix_avector, b, u, 1.0e-8, 1000, 50,
                                trace, &thr);
      t0 = stop_stopwatch(sw);
      snprintf(name, sizeof(name), "%s_gmres_trace", prefix);
      dump_real(name, trace, 1, iter + 1, 0);
      snprintf(name, sizeof(name), "%s_gmres_threshold", prefix);
      dump_scalar(name, thr);
      free(trace);
    }
    snprintf(name, sizeof(name), "%s_time_gmres", prefix);
    dump_scalar(name, t0);
    snprintf(name, sizeof(name), "%s_gmres_iter", prefix);
    dump_scalar(name, (double) iter);
    snprintf(name, sizeof(name), "%s_u", prefix);
    dump_avector(name, u);
    err = normL2diff_l_bem3d(slp, u, eval_neumann_fundamental_laplacebem3d, NULL);
    nrm = normL2_bem3d(slp, eval_neumann_fundamental_laplacebem3d, NULL);
    snprintf(name, sizeof(name), "%s_l2err", prefix);
    dump_scalar(name, err);
    snprintf(name, sizeof(name), "%s_l2norm", prefix);
    dump_scalar(name, nrm);
    del_avector(f);
    del_avector(b);
    del_avector(u);
  }

  del_avector(x);
  del_avector(y);
  del_h2matrix(V);
  del_h2matrix(K);
  del_block(broot);
  freemem(root->idx);
  del_cluster(root);
  del_laplace_bem3d(slp);
  del_laplace_bem3d(dlp);
  del_stopwatch(sw);
}

static void
section_h2small(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 8);
  h2_case("h2ll", gr, BASIS_LINEAR_BEM3D, 16, 1.4, 3, 24, 1);
  h2_case("h2cc", gr, BASIS_CONSTANT_BEM3D, 16, 1.4, 3, 24, 0);
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

/* Greenhybrid H2 matrices (the reference's Laplace test parameters m 2, l 1, delta 1, accuracy
 * 5e-3) on the sphere refined 8 times, scaled to an ellipsoid and turned: single layer with
 * linear and constant bases, double layer with linear and constant bases. */
static void
section_green(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 8);
  pbem3d slp_l, slp_c, dlp_l;
  uint v;
  /* scaled and turned out of the axes: the cluster boxes and their quadrature points are then
   * aligned with no symmetry of the mesh, so no two candidates of a pivot search tie */
  const real ax[3] = { 1.0, 0.8, 0.65 }, ca = cos(0.37), sa = sin(0.37), cb = cos(0.61),
             sb = sin(0.61), cc = cos(0.23), sc = sin(0.23);
  for (v = 0; v < gr->vertices; v++) {
    real p0 = gr->x[v][0] * ax[0], p1 = gr->x[v][1] * ax[1], p2 = gr->x[v][2] * ax[2], q0, q1, q2;
    q1 = cc * p1 - sc * p2;            /* about x */
    q2 = sc * p1 + cc * p2;
    q0 = cb * p0 + sb * q2;            /* about y */
    q2 = -sb * p0 + cb * q2;
    p0 = ca * q0 - sa * q1;            /* about z */
    p1 = sa * q0 + ca * q1;
    gr->x[v][0] = p0;
    gr->x[v][1] = p1;
    gr->x[v][2] = q2;
  }
  prepare_surface3d(gr);
  dump_mesh("green", gr);
  slp_l = new_slp_laplace_bem3d(gr, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D);
  green_op("gsll", gr, slp_l, BASIS_LINEAR_BEM3D, 16, 1.4, 2, 1, 1.0, 5e-3, 24);
  del_bem3d(slp_l);
  slp_c = new_slp_laplace_bem3d(gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D);
  green_op("gscc", gr, slp_c, BASIS_CONSTANT_BEM3D, 16, 1.4, 2, 1, 1.0, 5e-3, 24);
  del_bem3d(slp_c);
  dlp_l = new_dlp_laplace_bem3d(gr, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D, 0.5);
  green_op("gdll", gr, dlp_l, BASIS_LINEAR_BEM3D, 16, 1.4, 2, 1, 1.0, 5e-3, 24);
  del_bem3d(dlp_l);
  dlp_l = new_dlp_laplace_bem3d(gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D, 0.5);
  green_op("gdcc", gr, dlp_l, BASIS_CONSTANT_BEM3D, 16, 1.4, 2, 1, 1.0, 5e-3, 24);
  del_bem3d(dlp_l);
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

static void
section_config2(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 64);
  dump_real("c2mesh_x", &gr->x[0][0], 2, gr->vertices, 3);
  dump_uint("c2mesh_t", &gr->t[0][0], 2, gr->triangles, 3);
  h2_case("c2", gr, BASIS_LINEAR_BEM3D, 64, 1.4, 4, 0, 1);
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

static void
section_cube(void)
{
  pmacrosurface3d mg = new_cube_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 4);
  dump_mesh("cube4", gr);
  del_surface3d(gr);
  gr = build_from_macrosurface3d_surface3d(mg, 64);
  dump_real("cube64_x", &gr->x[0][0], 2, gr->vertices, 3);
  dump_uint("cube64_t", &gr->t[0][0], 2, gr->triangles, 3);
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

/* Adjoint double layer K' + M/2 (new_adlp_laplace_bem3d, Library/laplacebem3d.c:1180): dense on
 * the sphere refined x4 for the four basis pairs, and H2 matrices on the sphere refined x8. */
static void
section_adlp(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d g4 = build_from_macrosurface3d_surface3d(mg, 4);
  psurface3d g8 = build_from_macrosurface3d_surface3d(mg, 8);
  basisfunctionbem3d C = BASIS_CONSTANT_BEM3D, L = BASIS_LINEAR_BEM3D;
  pbem3d op;

  op = new_adlp_laplace_bem3d(g4, 2, 4, C, C, 0.5);
  dense_op("ad4cc", g4, op, C, C, 0);
  del_laplace_bem3d(op);
  op = new_adlp_laplace_bem3d(g4, 2, 4, L, L, 0.5);
  dense_op("ad4ll", g4, op, L, L, 1);
  del_laplace_bem3d(op);
  op = new_adlp_laplace_bem3d(g4, 2, 4, C, L, 0.5);
  dense_op("ad4cl", g4, op, C, L, 0);
  del_laplace_bem3d(op);
  op = new_adlp_laplace_bem3d(g4, 2, 4, L, C, 0.5);
  dense_op("ad4lc", g4, op, L, C, 0);
  del_laplace_bem3d(op);
  op = new_adlp_laplace_bem3d(g8, 2, 4, L, L, 0.5);
  h2_op("adh2ll", g8, op, L, 16, 1.4, 3, 24);
  del_laplace_bem3d(op);
  op = new_adlp_laplace_bem3d(g8, 2, 4, C, C, 0.5);
  h2_op("adh2cc", g8, op, C, 16, 1.4, 3, 24);
  del_laplace_bem3d(op);
  del_surface3d(g4);
  del_surface3d(g8);
  del_macrosurface3d(mg);
}

#else /* USE_COMPLEX */

static void
section_helm_sphere4(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 4);
  field k = 2.0;
  pbem3d slp, dlp;
  pamatrix A = new_amatrix(gr->triangles, gr->triangles);

  slp = new_slp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D);
  dlp = new_dlp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D, 0.5);
  slp->nearfield(NULL, NULL, slp, false, A);
  dump_amatrix("hs4cc_slp", A);
  dlp->nearfield(NULL, NULL, dlp, false, A);
  dump_amatrix("hs4cc_dlp", A);
  del_helmholtz_bem3d(slp);
  del_helmholtz_bem3d(dlp);
  /* complex wavenumber (damped) */
  k = 2.0 + 0.5 * I;
  slp = new_slp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D);
  slp->nearfield(NULL, NULL, slp, false, A);
  dump_amatrix("hs4cc_slp_damped", A);
  del_helmholtz_bem3d(slp);
  del_amatrix(A);
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

static void
section_helm_h2small(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 8);
  field k = 2.0;
  real eta = 1.4;
  pbem3d slp, dlp;
  pcluster root;
  pblock broot;
  pclusterbasis Vrb, Vcb, Krb, Kcb;
  ph2matrix V, K;
  pavector x, y;

  slp = new_slp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D);
  dlp = new_dlp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D, 0.5);
  root = build_bem3d_cluster(slp, 16, BASIS_CONSTANT_BEM3D);
  broot = build_strict_block(root, root, &eta, admissible_max_cluster);
  dump_cluster("hh2", root);
  dump_block("hh2", broot, root, root);
  Vrb = build_from_cluster_clusterbasis(root);
  Vcb = build_from_cluster_clusterbasis(root);
  Krb = build_from_cluster_clusterbasis(root);
  Kcb = build_from_cluster_clusterbasis(root);
  V = build_from_block_h2matrix(broot, Vrb, Vcb);
  K = build_from_block_h2matrix(broot, Krb, Kcb);
  setup_h2matrix_aprx_inter_bem3d(slp, Vrb, Vcb, broot, 3);
  setup_h2matrix_aprx_inter_bem3d(dlp, Krb, Kcb, broot, 3);
  assemble_bem3d_h2matrix_row_clusterbasis(slp, Vrb);
  assemble_bem3d_h2matrix_col_clusterbasis(slp, Vcb);
  assemble_bem3d_h2matrix(slp, V);
  assemble_bem3d_h2matrix_row_clusterbasis(dlp, Krb);
  assemble_bem3d_h2matrix_col_clusterbasis(dlp, Kcb);
  assemble_bem3d_h2matrix(dlp, K);
  dump_basis("hh2_Vrow", Vrb);
  dump_basis("hh2_Kcol", Kcb);
  dump_h2parts("hh2_Vparts", V, 24);

  x = new_avector(gr->triangles);
  y = new_avector(gr->triangles);
  seeded_avector(x, 2);
  dump_avector("hh2_x", x);
  clear_avector(y);
  addeval_h2matrix_avector(1.0, V, x, y);
  dump_avector("hh2_ySLP", y);
  clear_avector(y);
  addeval_h2matrix_avector(1.0, K, x, y);
  dump_avector("hh2_yDLP", y);

  del_avector(x);
  del_avector(y);
  del_h2matrix(V);
  del_h2matrix(K);
  del_block(broot);
  freemem(root->idx);
  del_cluster(root);
  del_helmholtz_bem3d(slp);
  del_helmholtz_bem3d(dlp);
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

/* Brakhage-Werner operator (K + M/2) - i eta V of Tests/test_helmholtzbem3d.c:26-65 */
typedef struct {
  ph2matrix V, KM;
  field eta;
} bw_t;

static void
addeval_bw(field alpha, void *matrix, pcavector x, pavector y)
{
  bw_t *bw = (bw_t *) matrix;
  addeval_h2matrix_avector(alpha, bw->KM, x, y);
  addeval_h2matrix_avector(-I * alpha * bw->eta, bw->V, x, y);
}

/* Config 3: cube refined to 49152 triangles, constant basis, wavenumber k, m = 5, leaf 64,
 * eta 1.4; plane wave along (1,1,1)/sqrt(3); Dirichlet data -u_inc; GMRES(80) to 1e-8.  The
 * trees are dumped once (they do not depend on k); the solve records its residual trace. */
static void
config3_case(const char *p, field k, int with_trees)
{
  pmacrosurface3d mg = new_cube_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 64);
  real eta = 1.4;
  char name[256];
  pbem3d slp, dlp;
  pcluster root;
  pblock broot;
  pclusterbasis Vrb, Vcb, Krb, Kcb;
  ph2matrix V, K;
  pavector x, y, b, u;
  helmholtz_data hdata;
  real kvec[3], src[3] = {0.0, 0.0, 0.0};
  bw_t bw;
  uint iter, i;
  pstopwatch sw = new_stopwatch();

  slp = new_slp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D);
  dlp = new_dlp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D, 0.5);
  root = build_bem3d_cluster(slp, 64, BASIS_CONSTANT_BEM3D);
  broot = build_strict_block(root, root, &eta, admissible_max_cluster);
  if (with_trees) {
    dump_cluster(p, root);
    dump_block(p, broot, root, root);
  }
  Vrb = build_from_cluster_clusterbasis(root);
  Vcb = build_from_cluster_clusterbasis(root);
  Krb = build_from_cluster_clusterbasis(root);
  Kcb = build_from_cluster_clusterbasis(root);
  V = build_from_block_h2matrix(broot, Vrb, Vcb);
  K = build_from_block_h2matrix(broot, Krb, Kcb);
  setup_h2matrix_aprx_inter_bem3d(slp, Vrb, Vcb, broot, 5);
  setup_h2matrix_aprx_inter_bem3d(dlp, Krb, Kcb, broot, 5);
  start_stopwatch(sw);
  assemble_bem3d_h2matrix_row_clusterbasis(slp, Vrb);
  assemble_bem3d_h2matrix_col_clusterbasis(slp, Vcb);
  assemble_bem3d_h2matrix(slp, V);
  assemble_bem3d_h2matrix_row_clusterbasis(dlp, Krb);
  assemble_bem3d_h2matrix_col_clusterbasis(dlp, Kcb);
  assemble_bem3d_h2matrix(dlp, K);
  snprintf(name, sizeof(name), "%s_time_assembly", p);
  dump_scalar(name, stop_stopwatch(sw));

  x = new_avector(gr->triangles);
  y = new_avector(gr->triangles);
  seeded_avector(x, 3);
  snprintf(name, sizeof(name), "%s_x", p);
  dump_avector(name, x);
  clear_avector(y);
  addeval_h2matrix_avector(1.0, V, x, y);
  snprintf(name, sizeof(name), "%s_ySLP", p);
  dump_avector(name, y);
  clear_avector(y);
  addeval_h2matrix_avector(1.0, K, x, y);
  snprintf(name, sizeof(name), "%s_yDLP", p);
  dump_avector(name, y);

  for (i = 0; i < 3; i++)
    kvec[i] = REAL(k) / REAL_SQRT(3.0);
  hdata.kvec = kvec;
  hdata.source = src;
  hdata.eta = k;
  b = new_avector(gr->triangles);
  u = new_avector(gr->triangles);
  integrate_bem3d_c_avector(dlp, rhs_dirichlet_plane_helmholtzbem3d, b, (void *) &hdata);
  scale_avector(-1.0, b);
  snprintf(name, sizeof(name), "%s_b", p);
  dump_avector(name, b);
  bw.V = V;
  bw.KM = K;
  bw.eta = k;
  clear_avector(u);
  {
    real *trace = (real *) calloc(1000, sizeof(real)), thr = 0.0;
    start_stopwatch(sw);
    iter = solve_gmres_traced(&bw, addeval_bw, b, u, 1.0e-8, 1000, 80, trace, &thr);
    snprintf(name, sizeof(name), "%s_time_gmres", p);
    dump_scalar(name, stop_stopwatch(sw));
    snprintf(name, sizeof(name), "%s_gmres_trace", p);
    dump_real(name, trace, 1, iter + 1, 0);
    snprintf(name, sizeof(name), "%s_gmres_threshold", p);
    dump_scalar(name, thr);
    free(trace);
  }
  snprintf(name, sizeof(name), "%s_gmres_iter", p);
  dump_scalar(name, (double) iter);
  snprintf(name, sizeof(name), "%s_u", p);
  dump_avector(name, u);

  del_avector(x); del_avector(y); del_avector(b); del_avector(u);
  del_h2matrix(V);
  del_h2matrix(K);
  del_block(broot);
  freemem(root->idx);
  del_cluster(root);
  del_helmholtz_bem3d(slp);
  del_helmholtz_bem3d(dlp);
  del_surface3d(gr);
  del_macrosurface3d(mg);
  del_stopwatch(sw);
}

static void
section_config3(void)
{
  config3_case("c3", 2.0, 1);
}

static void
section_config3_k8(void)
{
  config3_case("c8", 8.0, 0);
}

/* Helmholtz adjoint double layer K' + M/2 (new_adlp_helmholtz_bem3d, Library/helmholtzbem3d.c:
 * 1346), constant basis: dense on the sphere refined x4 (k = 2 and the damped k = 2 + 0.5i) and
 * the H2 matrix on the sphere refined x8 (k = 2). */
static void
section_helm_adlp(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d g4 = build_from_macrosurface3d_surface3d(mg, 4);
  psurface3d g8 = build_from_macrosurface3d_surface3d(mg, 8);
  basisfunctionbem3d C = BASIS_CONSTANT_BEM3D;
  pbem3d op;

  op = new_adlp_helmholtz_bem3d(2.0, g4, 2, 4, C, C, 0.5);
  dense_op("had4cc", g4, op, C, C, 0);
  del_helmholtz_bem3d(op);
  op = new_adlp_helmholtz_bem3d(2.0 + 0.5 * I, g4, 2, 4, C, C, 0.5);
  dense_op("had4cc_damped", g4, op, C, C, 0);
  del_helmholtz_bem3d(op);
  op = new_adlp_helmholtz_bem3d(2.0, g8, 2, 4, C, C, 0.5);
  h2_op("hadh2cc", g8, op, C, 16, 1.4, 3, 24);
  del_helmholtz_bem3d(op);
  del_surface3d(g4);
  del_surface3d(g8);
  del_macrosurface3d(mg);
}

/* The reference's complex GMRES on a small Brakhage-Werner system: sphere refined x10 (800
 * triangles), constant basis, k = 5, leaf 32, eta 1.4, m = 4, seeded right-hand side, GMRES(80)
 * to 1e-8.  Records the iteration count, the solution and its true relative residual
 * |b - A u| / |b| (the reference stops on its residual estimate). */
static void
section_helm_gmres(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 10);
  field k = 5.0;
  real eta = 1.4;
  pbem3d slp, dlp;
  pcluster root;
  pblock broot;
  pclusterbasis Vrb, Vcb, Krb, Kcb;
  ph2matrix V, K;
  pavector b, u, r;
  bw_t bw;
  uint iter;

  slp = new_slp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D);
  dlp = new_dlp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D, 0.5);
  root = build_bem3d_cluster(slp, 32, BASIS_CONSTANT_BEM3D);
  broot = build_strict_block(root, root, &eta, admissible_max_cluster);
  dump_mesh("hg", gr);
  dump_cluster("hg", root);
  dump_block("hg", broot, root, root);
  Vrb = build_from_cluster_clusterbasis(root);
  Vcb = build_from_cluster_clusterbasis(root);
  Krb = build_from_cluster_clusterbasis(root);
  Kcb = build_from_cluster_clusterbasis(root);
  V = build_from_block_h2matrix(broot, Vrb, Vcb);
  K = build_from_block_h2matrix(broot, Krb, Kcb);
  setup_h2matrix_aprx_inter_bem3d(slp, Vrb, Vcb, broot, 4);
  setup_h2matrix_aprx_inter_bem3d(dlp, Krb, Kcb, broot, 4);
  assemble_bem3d_h2matrix_row_clusterbasis(slp, Vrb);
  assemble_bem3d_h2matrix_col_clusterbasis(slp, Vcb);
  assemble_bem3d_h2matrix(slp, V);
  assemble_bem3d_h2matrix_row_clusterbasis(dlp, Krb);
  assemble_bem3d_h2matrix_col_clusterbasis(dlp, Kcb);
  assemble_bem3d_h2matrix(dlp, K);

  b = new_avector(gr->triangles);
  u = new_avector(gr->triangles);
  r = new_avector(gr->triangles);
  seeded_avector(b, 4);
  dump_avector("hg_b", b);
  bw.V = V;
  bw.KM = K;
  bw.eta = k;
  clear_avector(u);
  iter = solve_gmres_avector(&bw, addeval_bw, b, u, 1.0e-8, 1000, 80);
  dump_scalar("hg_gmres_iter", (double) iter);
  dump_avector("hg_u", u);
  copy_avector(b, r);
  addeval_bw(-1.0, &bw, u, r);
  dump_scalar("hg_true_residual", norm2_avector(r) / norm2_avector(b));

  del_avector(b); del_avector(u); del_avector(r);
  del_h2matrix(V);
  del_h2matrix(K);
  del_block(broot);
  freemem(root->idx);
  del_cluster(root);
  del_helmholtz_bem3d(slp);
  del_helmholtz_bem3d(dlp);
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

/* The reference test's own evaluation of a Brakhage-Werner density at points outside the surface
 * and its error measure, compiled from Tests/test_helmholtzbem3d.c (main renamed there). */
field eval_brakhage_werner_c(pcbem3d bem, pcavector w, field eta, real *x);
field eval_brakhage_werner_l(pcbem3d bem, pcavector w, field eta, real *x);
real max_rel_outer_error(pcbem3d bem, helmholtz_data *hdata, pcavector x, boundary_func3d rhs,
                         basisfunctionbem3d basis);

/* The Brakhage-Werner operator on dense matrices */
typedef struct {
  pamatrix V, KM;
  field eta;
} bw_dense_t;

static void
addeval_bw_dense(field alpha, void *matrix, pcavector x, pavector y)
{
  bw_dense_t *bw = (bw_dense_t *) matrix;
  addeval_amatrix_avector(alpha, bw->KM, x, y);
  addeval_amatrix_avector(-I * alpha * bw->eta, bw->V, x, y);
}

/* The reference's exterior test problem (Tests/test_helmholtzbem3d.c:354-459 with main's
 * parameters, :694): unit sphere with 512 triangles, k = 2, quadrature orders 2 / 4, a point
 * source at (0, 0, 0.2) inside, kvec (k, 0, 0).  Per basis (constant "hpc", linear "hpl"): the
 * tested datum b (integrate_bem3d_c/l_avector with rhs_dirichlet_point_helmholtzbem3d), the
 * Brakhage-Werner system (K + M/2) - i k V assembled densely and solved by GMRES(50) to 1e-12,
 * the evaluation points of max_rel_outer_error, the potential of the solution there
 * (eval_brakhage_werner_c / _l with eta = k) and the maximal relative error against the source's
 * field. */
static void
section_helm_point(void)
{
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, 8);
  const field k = 2.0;
  real kvec[3] = {2.0, 0.0, 0.0}, source[3] = {0.0, 0.0, 0.2};
  helmholtz_data hdata;
  int lin;

  hdata.kvec = kvec;
  hdata.source = source;
  for (lin = 0; lin < 2; lin++) {
    basisfunctionbem3d basis = lin ? BASIS_LINEAR_BEM3D : BASIS_CONSTANT_BEM3D;
    const char *p = lin ? "hpl" : "hpc";
    uint n = lin ? gr->vertices : gr->triangles;
    pbem3d slp = new_slp_helmholtz_bem3d(k, gr, 2, 4, basis, basis);
    pbem3d dlp = new_dlp_helmholtz_bem3d(k, gr, 2, 4, basis, basis, 0.5);
    pamatrix V = new_amatrix(n, n), KM = new_amatrix(n, n);
    pavector b = new_avector(n), x = new_avector(n);
    bw_dense_t bw;
    uint iter, i, j, np = 0;
    real (*pts)[3] = (real (*)[3]) allocreal(3 * 400);
    field *y;
    char name[64];

    assemble_bem3d_amatrix(slp, V);
    assemble_bem3d_amatrix(dlp, KM);
    if (lin)
      integrate_bem3d_l_avector(dlp, rhs_dirichlet_point_helmholtzbem3d, b, &hdata);
    else
      integrate_bem3d_c_avector(dlp, rhs_dirichlet_point_helmholtzbem3d, b, &hdata);
    bw.V = V;
    bw.KM = KM;
    bw.eta = k;
    clear_avector(x);
    iter = solve_gmres_avector(&bw, addeval_bw_dense, b, x, 1.0e-12, 1000, 50);
    /* the points of max_rel_outer_error (Tests/test_helmholtzbem3d.c:224) */
    for (j = 0; j < 20; j++)
      for (i = 0; i < 20; i++) {
        pts[np][0] = -10.0 + (20.0 / 19) * i;
        pts[np][1] = 0.0;
        pts[np][2] = -10.0 + (20.0 / 19) * j;
        if (pts[np][0] * pts[np][0] + pts[np][2] * pts[np][2] > 1)
          np++;
      }
    y = (field *) malloc(sizeof(field) * np);
    for (j = 0; j < np; j++)
      y[j] = lin ? eval_brakhage_werner_l(slp, x, k, pts[j])
                 : eval_brakhage_werner_c(slp, x, k, pts[j]);
    snprintf(name, sizeof(name), "%s_b", p);
    dump_avector(name, b);
    snprintf(name, sizeof(name), "%s_x", p);
    dump_avector(name, x);
    snprintf(name, sizeof(name), "%s_iter", p);
    dump_scalar(name, (double) iter);
    snprintf(name, sizeof(name), "%s_points", p);
    dump_real(name, &pts[0][0], 2, np, 3);
    snprintf(name, sizeof(name), "%s_u", p);
    dump(name, "c16", sizeof(field), y, 1, np, 0);
    snprintf(name, sizeof(name), "%s_maxerr", p);
    dump_scalar(name, max_rel_outer_error(slp, &hdata, x, rhs_dirichlet_point_helmholtzbem3d,
                                          basis));
    free(y);
    freemem(pts);
    del_avector(b);
    del_avector(x);
    del_amatrix(V);
    del_amatrix(KM);
    del_helmholtz_bem3d(slp);
    del_helmholtz_bem3d(dlp);
  }
  del_surface3d(gr);
  del_macrosurface3d(mg);
}

#endif

int
main(int argc, char **argv)
{
  char path[4096];
  int i;

  init_h2lib(&argc, &argv);
  if (argc < 3) {
    fprintf(stderr, "usage: %s outdir section...\n", argv[0]);
    return 2;
  }
  outdir = argv[1];
  snprintf(path, sizeof(path), "%s/manifest.txt", outdir);
  manifest = fopen(path, "a");
  if (!manifest) {
    perror(path);
    return 1;
  }
  for (i = 2; i < argc; i++) {
#ifndef USE_COMPLEX
    if (!strcmp(argv[i], "quad"))
      section_quad();
    else if (!strcmp(argv[i], "sphere8"))
      section_sphere8();
    else if (!strcmp(argv[i], "sphere4"))
      section_sphere4();
    else if (!strcmp(argv[i], "h2small"))
      section_h2small();
    else if (!strcmp(argv[i], "config2"))
      section_config2();
    else if (!strcmp(argv[i], "cube"))
      section_cube();
    else if (!strcmp(argv[i], "adlp"))
      section_adlp();
    else if (!strcmp(argv[i], "green"))
      section_green();
#else
    if (!strcmp(argv[i], "helm_sphere4"))
      section_helm_sphere4();
    else if (!strcmp(argv[i], "helm_h2small"))
      section_helm_h2small();
    else if (!strcmp(argv[i], "config3"))
      section_config3();
    else if (!strcmp(argv[i], "config3_k8"))
      section_config3_k8();
    else if (!strcmp(argv[i], "helm_gmres"))
      section_helm_gmres();
    else if (!strcmp(argv[i], "helm_point"))
      section_helm_point();
    else if (!strcmp(argv[i], "helm_adlp"))
      section_helm_adlp();
#endif
    else {
      fprintf(stderr, "unknown section %s\n", argv[i]);
      return 2;
    }
  }
  fclose(manifest);
  uninit_h2lib();
  return 0;
}
