/* H2Lib drop-in layer over the B200 C ABI (see h2b_h2lib.h for what it replaces and why).
 *
 * Compiled against H2Lib's own headers (the Library directory) in the same configuration as the H2Lib it is
 * linked with: without USE_COMPLEX it handles the Laplace operators, with USE_COMPLEX the
 * Helmholtz operators (field = double complex, whose memory layout is the interleaved (re, im)
 * pairs of include/h2b200.h).
 *
 * Device objects are found from H2Lib objects through small registries (surface3d -> device
 * surface, bem3d -> device operator, h2matrix -> device tree + H2 matrix).  H2 structures are
 * handed to the library as flattened trees (h2b_tree_new_flat): clusters in pre-order with their
 * offsets into the root index array, and the leaf blocks in block-tree pre-order with sons
 * column-major, the order of H2Lib's own enumerate_h2matrix (Library/h2matrix.c:549).
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "basic.h"
#include "bem3d.h"
#include "block.h"
#include "cluster.h"
#include "clusterbasis.h"
#include "h2matrix.h"
#include "krylov.h"
#include "krylovsolvers.h"
#include "surface3d.h"
#include "uniform.h"
#ifdef USE_COMPLEX
#include "helmholtzbem3d.h"
#else
#include "laplacebem3d.h"
#endif

#include "h2b200.h"
#include "h2b_h2lib.h"

/* ------------------------------------------------------------------------------------------
 * plumbing
 * ------------------------------------------------------------------------------------------ */

static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;
static int g_bypass = 0;
static unsigned long long g_counts[6];
static int g_device_ready = 0;

void h2b_shim_set_bypass(int on) { g_bypass = on; }

void h2b_shim_counts(unsigned long long out[6]) {
  memcpy(out, g_counts, sizeof(g_counts));
}

static void die(const char *what) {
  fprintf(stderr, "h2b_h2lib: %s failed: %s\n", what, h2b_last_error());
  abort();
}

static void check(int rc, const char *what) {
  if (rc < 0) die(what);
}

static void *original(const char *name) {
  void *p = dlsym(RTLD_NEXT, name);
  if (!p) {
    fprintf(stderr, "h2b_h2lib: H2Lib's %s not found behind the shim\n", name);
    abort();
  }
  return p;
}

/* H2Lib's own definition of `name`, looked up once. */
#define ORIGINAL(name) \
  static __typeof__(&name) o_; \
  if (!o_) o_ = (__typeof__(&name)) original(#name)

static void device_ready(void) {
  if (g_device_ready) return;
  const char *e = getenv("H2B_DEVICE");
  check(h2b_device_init(e ? atoi(e) : 0), "h2b_device_init");
  g_device_ready = 1;
}

#ifdef USE_COMPLEX
#define SHIM_PDE H2B_HELMHOLTZ
#define FIELD_DOUBLES 2
static double re_of(field f) { return creal(f); }
static double im_of(field f) { return cimag(f); }
#else
#define SHIM_PDE H2B_LAPLACE
#define FIELD_DOUBLES 1
static double re_of(field f) { return f; }
static double im_of(field f) { (void) f; return 0.0; }
#endif

/* ------------------------------------------------------------------------------------------
 * registries
 * ------------------------------------------------------------------------------------------ */

typedef struct {
  pcsurface3d gr;
  h2b_surface *s;
} surf_rec;

typedef struct {
  pcbem3d bem;
  h2b_bem *g;
  pcsurface3d gr;
  uint m;  /* interpolation order (setup_h2matrix_aprx_inter_bem3d), 0 until set */
  /* greenhybrid farfield (setup_h2matrix_aprx_greenhybrid_bem3d with the cube points): m is then
   * its Gauss order, and l, delta and the ACA accuracy are kept here */
  int layer;  /* H2B_SLP / H2B_DLP / H2B_ADLP */
  int green;
  uint gl;
  double gdelta, gaccur;
} bem_rec;

typedef struct {
  pch2matrix G;
  pcbem3d bem;
  h2b_tree *tree;
  h2b_h2matrix *h;
} h2_rec;

#define REG(T, name)                                                           \
  static T *name;                                                              \
  static size_t name##_n, name##_cap;                                          \
  static T *name##_push(void) {                                                \
    if (name##_n == name##_cap) {                                              \
      name##_cap = name##_cap ? 2 * name##_cap : 16;                           \
      name = (T *) realloc(name, sizeof(T) * name##_cap);                      \
      if (!name) {                                                             \
        fprintf(stderr, "h2b_h2lib: out of host memory\n");                    \
        abort();                                                               \
      }                                                                        \
    }                                                                          \
    return &name[name##_n++];                                                  \
  }
REG(surf_rec, g_surf)
REG(bem_rec, g_bem)
REG(h2_rec, g_h2)

static bem_rec *find_bem(pcbem3d bem) {
  for (size_t i = 0; i < g_bem_n; i++)
    if (g_bem[i].bem == bem) return &g_bem[i];
  return NULL;
}

static h2_rec *find_h2(pch2matrix G) {
  for (size_t i = 0; i < g_h2_n; i++)
    if (g_h2[i].G == G) return &g_h2[i];
  return NULL;
}

static void drop_h2_at(size_t i) {
  h2b_h2matrix_del(g_h2[i].h);
  h2b_tree_del(g_h2[i].tree);
  g_h2[i] = g_h2[--g_h2_n];
}

static h2b_surface *surface_for(pcsurface3d gr) {
  for (size_t i = 0; i < g_surf_n; i++)
    if (g_surf[i].gr == gr) return g_surf[i].s;
  h2b_surface *s = h2b_surface_new(gr->vertices, &gr->x[0][0], gr->triangles, &gr->t[0][0],
                                   &gr->n[0][0], gr->g);
  if (!s) die("h2b_surface_new");
  surf_rec *r = g_surf_push();
  r->gr = gr;
  r->s = s;
  return s;
}

/* ------------------------------------------------------------------------------------------
 * operators
 * ------------------------------------------------------------------------------------------ */

/* The GPU block fill installed as bem->nearfield (Library/bem3d.h:380): N (rows x cols, or its
 * transpose when ntrans) is H2Lib's host matrix with its own leading dimension. */
static void shim_nearfield(const uint *ridx, const uint *cidx, pcbem3d bem, bool ntrans,
                           pamatrix N) {
  pthread_mutex_lock(&g_lock);
  bem_rec *r = find_bem(bem);
  h2b_bem *g = r ? r->g : NULL;
  pthread_mutex_unlock(&g_lock);
  if (!g) {
    fprintf(stderr, "h2b_h2lib: nearfield callback of an operator the shim does not know\n");
    abort();
  }
  const uint rows = ntrans ? N->cols : N->rows, cols = ntrans ? N->rows : N->cols;
  check(h2b_bem_nearfield(g, ridx, rows, cidx, cols, ntrans ? 1 : 0, (double *) N->a, N->ld),
        "h2b_bem_nearfield");
  __atomic_add_fetch(&g_counts[0], 1, __ATOMIC_RELAXED);
}

static void attach(pbem3d bem, pcsurface3d gr, int layer, uint q, uint q2, field k, field alpha) {
  if (!bem) return;
  device_ready();
  pthread_mutex_lock(&g_lock);
  h2b_bem *g = h2b_bem_new(surface_for(gr), SHIM_PDE, layer, bem->row_basis, bem->col_basis, q,
                           q2, re_of(k), im_of(k), re_of(alpha), im_of(alpha));
  if (!g) {
    pthread_mutex_unlock(&g_lock);
    die("h2b_bem_new");
  }
  bem_rec *r = g_bem_push();
  r->bem = bem;
  r->g = g;
  r->gr = gr;
  r->m = 0;
  r->layer = layer;
  r->green = 0;
  pthread_mutex_unlock(&g_lock);
  bem->nearfield = shim_nearfield;
}

static void detach_bem(pcbem3d bem) {
  pthread_mutex_lock(&g_lock);
  for (size_t i = 0; i < g_h2_n;)
    if (g_h2[i].bem == bem) drop_h2_at(i);
    else i++;
  for (size_t i = 0; i < g_bem_n; i++)
    if (g_bem[i].bem == bem) {
      h2b_bem_del(g_bem[i].g);
      g_bem[i] = g_bem[--g_bem_n];
      break;
    }
  pthread_mutex_unlock(&g_lock);
}

#ifndef USE_COMPLEX
pbem3d new_slp_laplace_bem3d(pcsurface3d gr, uint q_regular, uint q_singular,
                             basisfunctionbem3d row_basis, basisfunctionbem3d col_basis) {
  ORIGINAL(new_slp_laplace_bem3d);
  pbem3d bem = o_(gr, q_regular, q_singular, row_basis, col_basis);
  if (!g_bypass) attach(bem, gr, H2B_SLP, q_regular, q_singular, 0.0, 0.0);
  return bem;
}

pbem3d new_dlp_laplace_bem3d(pcsurface3d gr, uint q_regular, uint q_singular,
                             basisfunctionbem3d row_basis, basisfunctionbem3d col_basis,
                             field alpha) {
  ORIGINAL(new_dlp_laplace_bem3d);
  pbem3d bem = o_(gr, q_regular, q_singular, row_basis, col_basis, alpha);
  if (!g_bypass) attach(bem, gr, H2B_DLP, q_regular, q_singular, 0.0, alpha);
  return bem;
}

pbem3d new_adlp_laplace_bem3d(pcsurface3d gr, uint q_regular, uint q_singular,
                              basisfunctionbem3d row_basis, basisfunctionbem3d col_basis,
                              field alpha) {
  ORIGINAL(new_adlp_laplace_bem3d);
  pbem3d bem = o_(gr, q_regular, q_singular, row_basis, col_basis, alpha);
  if (!g_bypass) attach(bem, gr, H2B_ADLP, q_regular, q_singular, 0.0, alpha);
  return bem;
}

void del_laplace_bem3d(pbem3d bem) {
  ORIGINAL(del_laplace_bem3d);
  detach_bem(bem);
  o_(bem);
}
#else
pbem3d new_slp_helmholtz_bem3d(field k, pcsurface3d gr, uint q_regular, uint q_singular,
                               basisfunctionbem3d row_basis, basisfunctionbem3d col_basis) {
  ORIGINAL(new_slp_helmholtz_bem3d);
  pbem3d bem = o_(k, gr, q_regular, q_singular, row_basis, col_basis);
  if (!g_bypass) attach(bem, gr, H2B_SLP, q_regular, q_singular, k, 0.0);
  return bem;
}

pbem3d new_dlp_helmholtz_bem3d(field k, pcsurface3d gr, uint q_regular, uint q_singular,
                               basisfunctionbem3d row_basis, basisfunctionbem3d col_basis,
                               field alpha) {
  ORIGINAL(new_dlp_helmholtz_bem3d);
  pbem3d bem = o_(k, gr, q_regular, q_singular, row_basis, col_basis, alpha);
  if (!g_bypass) attach(bem, gr, H2B_DLP, q_regular, q_singular, k, alpha);
  return bem;
}

pbem3d new_adlp_helmholtz_bem3d(field k, pcsurface3d gr, uint q_regular, uint q_singular,
                                basisfunctionbem3d row_basis, basisfunctionbem3d col_basis,
                                field alpha) {
  ORIGINAL(new_adlp_helmholtz_bem3d);
  pbem3d bem = o_(k, gr, q_regular, q_singular, row_basis, col_basis, alpha);
  if (!g_bypass) attach(bem, gr, H2B_ADLP, q_regular, q_singular, k, alpha);
  return bem;
}

void del_helmholtz_bem3d(pbem3d bem) {
  ORIGINAL(del_helmholtz_bem3d);
  detach_bem(bem);
  o_(bem);
}
#endif

void del_surface3d(psurface3d gr) {
  ORIGINAL(del_surface3d);
  pthread_mutex_lock(&g_lock);
  for (size_t i = 0; i < g_surf_n; i++)
    if (g_surf[i].gr == gr) {
      h2b_surface_del(g_surf[i].s);
      g_surf[i] = g_surf[--g_surf_n];
      break;
    }
  pthread_mutex_unlock(&g_lock);
  o_(gr);
}

void setup_h2matrix_aprx_inter_bem3d(pbem3d bem, pcclusterbasis rb, pcclusterbasis cb,
                                     pcblock tree, uint m) {
  ORIGINAL(setup_h2matrix_aprx_inter_bem3d);
  o_(bem, rb, cb, tree, m);
  pthread_mutex_lock(&g_lock);
  bem_rec *r = find_bem(bem);
  if (r) {
    r->m = m;
    r->green = 0;
  }
  pthread_mutex_unlock(&g_lock);
}

void setup_h2matrix_aprx_greenhybrid_bem3d(pbem3d bem, pcclusterbasis rb, pcclusterbasis cb,
                                           pcblock tree, uint m, uint l, real delta, real accur,
                                           quadpoints3d quadpoints) {
  ORIGINAL(setup_h2matrix_aprx_greenhybrid_bem3d);
  o_(bem, rb, cb, tree, m, l, delta, accur, quadpoints);
  pthread_mutex_lock(&g_lock);
  bem_rec *r = find_bem(bem);
  if (r) {
    /* the device builds the Laplace single and double layer with the cube points */
#ifdef USE_COMPLEX
    const int device = 0;
#else
    const int device = quadpoints == build_bem3d_cube_quadpoints && r->layer != H2B_ADLP;
#endif
    if (device) {
      r->m = m;
      r->green = 1;
      r->gl = l;
      r->gdelta = delta;
      r->gaccur = accur;
    } else {
      r->green = -1;  /* other point sets: the H2 matrices stay on H2Lib's CPU path */
    }
  }
  pthread_mutex_unlock(&g_lock);
}

void assemble_bem3d_amatrix(pbem3d bem, pamatrix G) {
  ORIGINAL(assemble_bem3d_amatrix);
  pthread_mutex_lock(&g_lock);
  bem_rec *r = g_bypass ? NULL : find_bem(bem);
  h2b_bem *g = r ? r->g : NULL;
  pthread_mutex_unlock(&g_lock);
  if (!g) {
    o_(bem, G);
    return;
  }
  check(h2b_bem_assemble_amatrix(g, (double *) G->a, G->ld), "h2b_bem_assemble_amatrix");
  __atomic_add_fetch(&g_counts[1], 1, __ATOMIC_RELAXED);
}

/* ------------------------------------------------------------------------------------------
 * flattened trees
 * ------------------------------------------------------------------------------------------ */

typedef struct {
  uint n, cap;
  uint *off, *size, *sons;
  double *box;
  pccluster *ptr;  /* pre-order id -> cluster */
} flat_tree;

static void flat_push(flat_tree *f, pccluster t, const uint *root_idx) {
  if (f->n == f->cap) {
    f->cap = f->cap ? 2 * f->cap : 256;
    f->off = (uint *) realloc(f->off, sizeof(uint) * f->cap);
    f->size = (uint *) realloc(f->size, sizeof(uint) * f->cap);
    f->sons = (uint *) realloc(f->sons, sizeof(uint) * f->cap);
    f->box = (double *) realloc(f->box, sizeof(double) * 6 * f->cap);
    f->ptr = (pccluster *) realloc(f->ptr, sizeof(pccluster) * f->cap);
    if (!f->off || !f->size || !f->sons || !f->box || !f->ptr) {
      fprintf(stderr, "h2b_h2lib: out of host memory\n");
      abort();
    }
  }
  const uint i = f->n++;
  f->off[i] = (uint) (t->idx - root_idx);
  f->size[i] = t->size;
  f->sons[i] = t->sons;
  for (int d = 0; d < 3; d++) {
    f->box[6 * i + d] = t->bmin[d];
    f->box[6 * i + 3 + d] = t->bmax[d];
  }
  f->ptr[i] = t;
  for (uint s = 0; s < t->sons; s++) flat_push(f, t->son[s], root_idx);
}

static void flat_free(flat_tree *f) {
  free(f->off);
  free(f->size);
  free(f->sons);
  free(f->box);
  free(f->ptr);
}

/* pre-order id of cluster t (clusters of one tree are few enough for a sorted lookup) */
typedef struct {
  pccluster t;
  uint id;
} ptr_id;

static int cmp_ptr(const void *a, const void *b) {
  const uintptr_t x = (uintptr_t) ((const ptr_id *) a)->t, y = (uintptr_t) ((const ptr_id *) b)->t;
  return x < y ? -1 : x > y;
}

static ptr_id *ptr_index(const flat_tree *f) {
  ptr_id *p = (ptr_id *) malloc(sizeof(ptr_id) * (f->n ? f->n : 1));
  for (uint i = 0; i < f->n; i++) p[i].t = f->ptr[i], p[i].id = i;
  qsort(p, f->n, sizeof(ptr_id), cmp_ptr);
  return p;
}

static uint lookup_id(const ptr_id *p, uint n, pccluster t) {
  ptr_id key = {t, 0};
  const ptr_id *hit = (const ptr_id *) bsearch(&key, p, n, sizeof(ptr_id), cmp_ptr);
  if (!hit) {
    fprintf(stderr, "h2b_h2lib: block refers to a cluster outside the basis trees\n");
    abort();
  }
  return hit->id;
}

typedef struct {
  uint n, cap;
  uint *rc, *cc;
  uint8_t *adm;
  ph2matrix *leaf;
} leaf_list;

static void leaves_of(ph2matrix G, leaf_list *l, const ptr_id *ri, uint rn, const ptr_id *ci,
                      uint cn) {
  if (G->son) {
    for (uint j = 0; j < G->csons; j++)
      for (uint i = 0; i < G->rsons; i++)
        leaves_of(G->son[i + j * G->rsons], l, ri, rn, ci, cn);
    return;
  }
  if (l->n == l->cap) {
    l->cap = l->cap ? 2 * l->cap : 1024;
    l->rc = (uint *) realloc(l->rc, sizeof(uint) * l->cap);
    l->cc = (uint *) realloc(l->cc, sizeof(uint) * l->cap);
    l->adm = (uint8_t *) realloc(l->adm, l->cap);
    l->leaf = (ph2matrix *) realloc(l->leaf, sizeof(ph2matrix) * l->cap);
    if (!l->rc || !l->cc || !l->adm || !l->leaf) {
      fprintf(stderr, "h2b_h2lib: out of host memory\n");
      abort();
    }
  }
  l->rc[l->n] = lookup_id(ri, rn, G->rb->t);
  l->cc[l->n] = lookup_id(ci, cn, G->cb->t);
  l->adm[l->n] = G->u ? 1 : 0;
  l->leaf[l->n] = G;
  l->n++;
}

static void leaves_free(leaf_list *l) {
  free(l->rc);
  free(l->cc);
  free(l->adm);
  free(l->leaf);
}

/* Device tree of H2 matrix G (all leaves), or of one cluster basis (rb != NULL: its tree as both
 * row and column tree, with a single admissible root block, which is all a basis needs). */
static h2b_tree *device_tree(pch2matrix G, pcclusterbasis rb, leaf_list *leaves) {
  pccluster rt = G ? G->rb->t : rb->t, ct = G ? G->cb->t : rb->t;
  flat_tree fr = {0}, fc = {0};
  flat_push(&fr, rt, rt->idx);
  flat_push(&fc, ct, ct->idx);
  ptr_id *ri = ptr_index(&fr), *ci = ptr_index(&fc);
  leaf_list l = {0};
  if (G) {
    leaves_of((ph2matrix) G, &l, ri, fr.n, ci, fc.n);
  } else {
    l.n = l.cap = 1;
    l.rc = (uint *) calloc(1, sizeof(uint));
    l.cc = (uint *) calloc(1, sizeof(uint));
    l.adm = (uint8_t *) calloc(1, 1);
    l.leaf = (ph2matrix *) calloc(1, sizeof(ph2matrix));
    l.adm[0] = 1;
  }
  h2b_tree *tree = h2b_tree_new_flat(fr.n, fr.off, fr.size, fr.sons, fr.box, rt->size, rt->idx,
                                     fc.n, fc.off, fc.size, fc.sons, fc.box, ct->size, ct->idx,
                                     l.n, l.rc, l.cc, l.adm);
  free(ri);
  free(ci);
  flat_free(&fr);
  flat_free(&fc);
  if (leaves) *leaves = l;
  else leaves_free(&l);
  if (!tree) die("h2b_tree_new_flat");
  return tree;
}

/* ------------------------------------------------------------------------------------------
 * copies into H2Lib's host structures
 * ------------------------------------------------------------------------------------------ */

static double *export_part(const h2b_h2matrix *h, int part, uint64_t *n) {
  check(h2b_h2matrix_export(h, part, UINT32_MAX, NULL, n), "h2b_h2matrix_export");
  double *buf = (double *) malloc(sizeof(double) * (*n ? *n : 1));
  if (!buf) {
    fprintf(stderr, "h2b_h2lib: out of host memory\n");
    abort();
  }
  uint64_t got = 0;
  check(h2b_h2matrix_export(h, part, UINT32_MAX, buf, &got), "h2b_h2matrix_export");
  if (got != *n) {
    fprintf(stderr, "h2b_h2lib: export of part %d returned %llu of %llu values\n", part,
            (unsigned long long) got, (unsigned long long) *n);
    abort();
  }
  return buf;
}

/* rows x cols real (bases, transfers) or field (coupling, nearfield) column-major values into A */
static const double *copy_into(pamatrix A, const double *src, int is_field) {
  const size_t w = is_field ? FIELD_DOUBLES : 1;
  for (uint j = 0; j < A->cols; j++)
    for (uint i = 0; i < A->rows; i++) {
      const double *v = src + w * ((size_t) i + (size_t) j * A->rows);
#ifdef USE_COMPLEX
      A->a[i + (size_t) j * A->ld] = is_field ? v[0] + v[1] * I : v[0];
#else
      A->a[i + (size_t) j * A->ld] = v[0];
#endif
    }
  return src + w * (size_t) A->rows * A->cols;
}

typedef struct {
  const double *V, *E;
} basis_cursor;

/* Leaf bases V (size x k) and transfer matrices E (k x k) in pre-order, as H2Lib's leaf_row /
 * transfer_row callbacks leave them (Library/bem3d.c:5937-6075), then ranks and tree sizes. */
static void fill_basis(pclusterbasis cb, uint k, basis_cursor *c, int is_root) {
  cb->k = k;
  if (!is_root) {
    resize_amatrix(&cb->E, k, k);
    c->E = copy_into(&cb->E, c->E, 0);
  }
  if (cb->sons == 0) {
    resize_amatrix(&cb->V, cb->t->size, k);
    c->V = copy_into(&cb->V, c->V, 0);
  }
  for (uint s = 0; s < cb->sons; s++) fill_basis(cb->son[s], k, c, 0);
}

/* Greenhybrid bases: per-cluster ranks (pre-order ids), V_t (|t| x k_t) and E_s (k_s x k_father),
 * as assemble_bem3d_greenhybrid_leaf_row_clusterbasis / _transfer_row_ leave them
 * (Library/bem3d.c:6194/6262). */
static void fill_green_basis(pclusterbasis cb, const uint32_t *rank, uint *id, basis_cursor *c,
                             uint kf, int is_root) {
  const uint k = rank[(*id)++];
  cb->k = k;
  if (!is_root) {
    resize_amatrix(&cb->E, k, kf);
    c->E = copy_into(&cb->E, c->E, 0);
  }
  if (cb->sons == 0) {
    resize_amatrix(&cb->V, cb->t->size, k);
    c->V = copy_into(&cb->V, c->V, 0);
  } else {
    resize_amatrix(&cb->V, 0, k);
  }
  for (uint s = 0; s < cb->sons; s++) fill_green_basis(cb->son[s], rank, id, c, k, 0);
}

static double *export_green(const h2b_h2matrix *h, int part) {
  uint64_t n = 0;
  check(h2b_h2matrix_export_green(h, part, NULL, &n), "h2b_h2matrix_export_green");
  double *buf = (double *) malloc(sizeof(double) * (n ? n : 1));
  if (!buf) die("out of host memory");
  check(h2b_h2matrix_export_green(h, part, buf, &n), "h2b_h2matrix_export_green");
  return buf;
}

static void fill_bases(const h2b_h2matrix *h, pclusterbasis rb, pclusterbasis cb, uint k,
                       int green) {
  for (int side = 0; side < 2 && green; side++) {
    pclusterbasis b = side ? cb : rb;
    if (!b) continue;
    uint32_t *rank = (uint32_t *) malloc(sizeof(uint32_t) * b->t->desc);
    if (!rank) die("out of host memory");
    check(h2b_h2matrix_green_ranks(h, side, rank), "h2b_h2matrix_green_ranks");
    double *V = export_green(h, side ? 2 : 0), *E = export_green(h, side ? 3 : 1);
    basis_cursor c = {V, E};
    uint id = 0;
    fill_green_basis(b, rank, &id, &c, 0, 1);
    update_tree_clusterbasis(b);
    free(V);
    free(E);
    free(rank);
  }
  if (green) return;
  for (int side = 0; side < 2; side++) {
    pclusterbasis b = side ? cb : rb;
    if (!b) continue;
    uint64_t nv, ne;
    double *V = export_part(h, side ? 2 : 0, &nv), *E = export_part(h, side ? 3 : 1, &ne);
    basis_cursor c = {V, E};
    fill_basis(b, k, &c, 1);
    update_tree_clusterbasis(b);
    free(V);
    free(E);
  }
}

static void fill_blocks(const h2b_h2matrix *h, const leaf_list *l, int near, int far, uint k,
                        int green) {
  uint64_t n;
  if (far) {
    /* greenhybrid couplings are k_row x k_col with the ranks of the host bases, which the
     * basis assembly has filled (assemble_bem3d_greenhybrid_uniform, Library/bem3d.c:6493) */
    double *S = green ? export_green(h, 4) : export_part(h, 4, &n);
    const double *p = S;
    for (uint i = 0; i < l->n; i++)
      if (l->adm[i]) {
        puniform U = l->leaf[i]->u;
        if (green) resize_amatrix(&U->S, U->rb->k, U->cb->k);
        else resize_amatrix(&U->S, k, k);
        p = copy_into(&U->S, p, 1);
      }
    free(S);
  }
  if (near) {
    double *N = export_part(h, 5, &n);
    const double *p = N;
    for (uint i = 0; i < l->n; i++)
      if (!l->adm[i]) p = copy_into(l->leaf[i]->f, p, 1);
    free(N);
  }
}

/* ------------------------------------------------------------------------------------------
 * H2 assembly
 * ------------------------------------------------------------------------------------------ */

static bem_rec *h2_bem(pcbem3d bem, const char *who) {
  bem_rec *r = g_bypass ? NULL : find_bem(bem);
  if (r && r->green < 0) return NULL;
  if (r && r->m == 0) {
    fprintf(stderr, "h2b_h2lib: %s before setup_h2matrix_aprx_inter_bem3d\n", who);
    abort();
  }
  return r;
}

static h2b_h2matrix *new_matrix(const bem_rec *r, h2b_tree *tree) {
  h2b_h2matrix *h = r->green > 0 ? h2b_h2matrix_new_greenhybrid(r->g, tree, r->m, r->gl,
                                                                r->gdelta, r->gaccur)
                                 : h2b_h2matrix_new(r->g, tree, r->m);
  if (!h) die(r->green > 0 ? "h2b_h2matrix_new_greenhybrid" : "h2b_h2matrix_new");
  return h;
}

static void basis_assembly(pcbem3d bem, pclusterbasis b, int column) {
  pthread_mutex_lock(&g_lock);
  bem_rec *r = h2_bem(bem, "cluster basis assembly");
  if (!r) {
    pthread_mutex_unlock(&g_lock);
    if (column) {
      ORIGINAL(assemble_bem3d_h2matrix_col_clusterbasis);
      o_(bem, b);
    } else {
      ORIGINAL(assemble_bem3d_h2matrix_row_clusterbasis);
      o_(bem, b);
    }
    return;
  }
  h2b_tree *tree = device_tree(NULL, b, NULL);
  h2b_h2matrix *h = new_matrix(r, tree);
  check(column ? h2b_h2matrix_assemble_col_clusterbasis(h)
               : h2b_h2matrix_assemble_row_clusterbasis(h), "cluster basis assembly");
  uint64_t info[8];
  check(h2b_h2matrix_info(h, info), "h2b_h2matrix_info");
  fill_bases(h, column ? NULL : b, column ? b : NULL, (uint) info[7], r->green > 0);
  h2b_h2matrix_del(h);
  h2b_tree_del(tree);
  pthread_mutex_unlock(&g_lock);
  __atomic_add_fetch(&g_counts[2], 1, __ATOMIC_RELAXED);
}

void assemble_bem3d_h2matrix_row_clusterbasis(pcbem3d bem, pclusterbasis rb) {
  basis_assembly(bem, rb, 0);
}

void assemble_bem3d_h2matrix_col_clusterbasis(pcbem3d bem, pclusterbasis cb) {
  basis_assembly(bem, cb, 1);
}

/* what: 0 nearfield and farfield (assemble_bem3d_h2matrix), 1 nearfield, 2 farfield */
static int h2_assembly(pbem3d bem, ph2matrix G, int what) {
  pthread_mutex_lock(&g_lock);
  bem_rec *r = h2_bem(bem, "H2 matrix assembly");
  if (!r) {
    pthread_mutex_unlock(&g_lock);
    return 0;
  }
  for (size_t i = 0; i < g_h2_n; i++)
    if (g_h2[i].G == G) {
      drop_h2_at(i);
      break;
    }
  leaf_list l;
  h2b_tree *tree = device_tree(G, NULL, &l);
  h2b_h2matrix *h = new_matrix(r, tree);
  uint64_t info[8];
  check(h2b_h2matrix_info(h, info), "h2b_h2matrix_info");
  const uint k = (uint) info[7];
  if (what == 0) {
    // the bases as well: the device matrix serves later products and solves; H2Lib's host bases
    // receive the same values its own basis assembly would give
    check(h2b_h2matrix_assemble_all(h), "h2b_h2matrix_assemble_all");
    fill_bases(h, G->rb, G->cb, k, r->green > 0);
    fill_blocks(h, &l, 1, 1, k, r->green > 0);
  } else if (what == 1) {
    check(h2b_h2matrix_assemble_nearfield(h), "h2b_h2matrix_assemble_nearfield");
    fill_blocks(h, &l, 1, 0, k, r->green > 0);
  } else {
    check(h2b_h2matrix_assemble_farfield(h), "h2b_h2matrix_assemble_farfield");
    fill_blocks(h, &l, 0, 1, k, r->green > 0);
  }
  leaves_free(&l);
  if (what == 0) {
    h2_rec *rec = g_h2_push();
    rec->G = G;
    rec->bem = bem;
    rec->tree = tree;
    rec->h = h;
  } else {
    h2b_h2matrix_del(h);
    h2b_tree_del(tree);
  }
  pthread_mutex_unlock(&g_lock);
  __atomic_add_fetch(&g_counts[3], 1, __ATOMIC_RELAXED);
  return 1;
}

void assemble_bem3d_h2matrix(pbem3d bem, ph2matrix G) {
  ORIGINAL(assemble_bem3d_h2matrix);
  if (!h2_assembly(bem, G, 0)) o_(bem, G);
}

void assemble_bem3d_nearfield_h2matrix(pbem3d bem, ph2matrix G) {
  ORIGINAL(assemble_bem3d_nearfield_h2matrix);
  if (!h2_assembly(bem, G, 1)) o_(bem, G);
}

void assemble_bem3d_farfield_h2matrix(pbem3d bem, ph2matrix G) {
  ORIGINAL(assemble_bem3d_farfield_h2matrix);
  if (!h2_assembly(bem, G, 2)) o_(bem, G);
}

void del_h2matrix(ph2matrix h2) {
  ORIGINAL(del_h2matrix);
  pthread_mutex_lock(&g_lock);
  for (size_t i = 0; i < g_h2_n; i++)
    if (g_h2[i].G == h2) {
      drop_h2_at(i);
      break;
    }
  pthread_mutex_unlock(&g_lock);
  o_(h2);
}

/* ------------------------------------------------------------------------------------------
 * products and solves
 * ------------------------------------------------------------------------------------------ */

static h2b_h2matrix *resident(pch2matrix G) {
  if (g_bypass) return NULL;
  pthread_mutex_lock(&g_lock);
  h2_rec *r = find_h2(G);
  h2b_h2matrix *h = r ? r->h : NULL;
  pthread_mutex_unlock(&g_lock);
  return h;
}

void addeval_h2matrix_avector(field alpha, pch2matrix h2, pcavector x, pavector y) {
  ORIGINAL(addeval_h2matrix_avector);
  h2b_h2matrix *h = resident(h2);
  if (!h) {
    o_(alpha, h2, x, y);
    return;
  }
  check(h2b_h2matrix_addeval(re_of(alpha), im_of(alpha), h, (const double *) x->v,
                             (double *) y->v), "h2b_h2matrix_addeval");
  __atomic_add_fetch(&g_counts[4], 1, __ATOMIC_RELAXED);
}

static uint device_gmres(h2b_h2matrix *h, pcavector b, pavector x, real eps, uint maxiter,
                         uint kmax) {
  const h2b_h2matrix *ops[1] = {h};
  const double coef[2] = {1.0, 0.0};
  const int it = h2b_solve_gmres(1, ops, coef, (const double *) b->v, (double *) x->v, eps,
                                 maxiter, kmax);
  check(it, "h2b_solve_gmres");
  __atomic_add_fetch(&g_counts[5], 1, __ATOMIC_RELAXED);
  return (uint) it;
}

uint solve_gmres_h2matrix_avector(pch2matrix A, pcavector b, pavector x, real eps, uint maxiter,
                                  uint kmax) {
  ORIGINAL(solve_gmres_h2matrix_avector);
  h2b_h2matrix *h = resident(A);
  if (!h) return o_(A, b, x, eps, maxiter, kmax);
  return device_gmres(h, b, x, eps, maxiter, kmax);
}

uint solve_gmres_avector(void *A, addeval_t addeval_A, pcavector b, pavector x, real eps,
                         uint maxiter, uint kmax) {
  ORIGINAL(solve_gmres_avector);
  h2b_h2matrix *h = addeval_A == (addeval_t) addeval_h2matrix_avector
                        ? resident((pch2matrix) A) : NULL;
  if (!h) return o_(A, addeval_A, b, x, eps, maxiter, kmax);
  return device_gmres(h, b, x, eps, maxiter, kmax);
}
