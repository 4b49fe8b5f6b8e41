/* Timed CPU baseline: the unmodified H2Lib reference, built from its own sources by
 * oracle/Makefile (libh2ref_omp.so / libh2ref_complex_omp.so: OpenMP + AVX), driven through its
 * public API on all host cores.  Benchmark infrastructure only; nothing of the B200 library is
 * involved.  Every phase is H2Lib's own driver with its own OpenMP parallelism
 * (assemble_bem3d_h2matrix_{row,col}_clusterbasis, Library/bem3d.c:10407/10436;
 * assemble_bem3d_nearfield_h2matrix / _farfield_, :10325/:10337; solve_gmres_avector,
 * Library/krylovsolvers.c:183), over every block.
 *
 *   ref_bench assembly split clf eta m steps warmup [--solve]          (real build)
 *       Laplace single + double layer H2 matrices on the sphere refined x split (linear basis,
 *       q 2/4): per step both operators' bases, nearfield and farfield; --solve then times the
 *       interior Dirichlet GMRES(50) solve to 1e-8 and one matrix-vector product.
 *   ref_bench green split clf eta m l delta accur                      (real build)
 *       Laplace single layer with the greenhybrid farfield (setup_h2matrix_aprx_greenhybrid_bem3d,
 *       Library/bem3d.c:9689, cube quadrature points) on the sphere refined x split (linear
 *       basis, q 2/4): one assembly timed by phase (bases, nearfield, farfield) and one
 *       matrix-vector product.
 *   ref_bench helmholtz split k clf eta m applications [--solve]       (complex build)
 *       Brakhage-Werner operator (K + M/2) - i k V on the cube refined x split (constant basis):
 *       one assembly of both operators, `applications` timed operator applications, and with
 *       --solve the GMRES(80) solve of the plane-wave problem to 1e-8.
 *   ref_bench requests file [budget_seconds]                          (either build)
 *       Dirichlet problems of the requests in `file` (written by bench.py) that match the build's
 *       field type (real: Laplace, complex: Helmholtz), one after the other: per request one
 *       set-up and assembly and a solve per source; prints each one's set-up, assembly,
 *       right-hand side and solve seconds.  No request starts after budget_seconds.
 *
 * Prints one JSON object.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef USE_OPENMP
#include <omp.h>
#endif

#include "basic.h"
#include "bem3d.h"
#include "block.h"
#include "cluster.h"
#include "clusterbasis.h"
#include "h2matrix.h"
#include "krylovsolvers.h"
#include "macrosurface3d.h"
#include "surface3d.h"
#ifdef USE_COMPLEX
#include "helmholtzbem3d.h"
#else
#include "laplacebem3d.h"
#endif

static pstopwatch sw;

static void tic(void) { start_stopwatch(sw); }
static double toc(void) { return stop_stopwatch(sw); }

static double near_entries(pch2matrix G) {
  double n = 0.0;
  if (G->f) return (double) G->f->rows * G->f->cols;
  if (G->son)
    for (uint j = 0; j < G->csons; j++)
      for (uint i = 0; i < G->rsons; i++) n += near_entries(G->son[i + j * G->rsons]);
  return n;
}

typedef struct {
  pcluster root;
  pblock broot;
  ph2matrix G[2];
} h2pair;

/* trees and two H2 matrices (one per operator) on the same block tree */
static void h2pair_new(h2pair *p, pbem3d op0, pbem3d op1, basisfunctionbem3d basis, uint clf,
                       real eta, uint m) {
  pbem3d ops[2] = {op0, op1};
  p->root = build_bem3d_cluster(op0, clf, basis);
  p->broot = build_strict_block(p->root, p->root, &eta, admissible_max_cluster);
  for (int i = 0; i < 2; i++) {
    pclusterbasis rb = build_from_cluster_clusterbasis(p->root);
    pclusterbasis cb = build_from_cluster_clusterbasis(p->root);
    p->G[i] = build_from_block_h2matrix(p->broot, rb, cb);
    setup_h2matrix_aprx_inter_bem3d(ops[i], rb, cb, p->broot, m);
  }
}

static void h2pair_del(h2pair *p) {
  del_h2matrix(p->G[0]);
  del_h2matrix(p->G[1]);
  del_block(p->broot);
  freemem(p->root->idx);
  del_cluster(p->root);
}

/* bases, nearfield and farfield of G with H2Lib's drivers; t[0] bases, t[1] near, t[2] far */
static void assemble(pbem3d op, ph2matrix G, double t[3]) {
  tic();
  assemble_bem3d_h2matrix_row_clusterbasis(op, G->rb);
  assemble_bem3d_h2matrix_col_clusterbasis(op, G->cb);
  t[0] += toc();
  tic();
  assemble_bem3d_nearfield_h2matrix(op, G);
  t[1] += toc();
  tic();
  assemble_bem3d_farfield_h2matrix(op, G);
  t[2] += toc();
}

static int threads(void) {
#ifdef USE_OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ---------------------------------------------------------------------------------------- */

#ifndef USE_COMPLEX
/* 1/|x - src|, the harmonic Dirichlet datum of a point source (as
 * eval_dirichlet_fundamental_laplacebem3d, Library/laplacebem3d.c:1391, with the source passed
 * as data) */
static field harmonic(const real *x, const real *n, void *data) {
  const real *z = (const real *) data;
  (void) n;
  return REAL_RSQRT(REAL_SQR(x[0] - z[0]) + REAL_SQR(x[1] - z[1]) + REAL_SQR(x[2] - z[2]));
}

static int mode_assembly(int argc, char **argv) {
  if (argc < 8) return 2;
  const uint split = atoi(argv[2]), clf = atoi(argv[3]), m = atoi(argv[5]);
  const uint steps = atoi(argv[6]), warmup = atoi(argv[7]);
  const real eta = atof(argv[4]);
  const int solve = argc > 8 && !strcmp(argv[8], "--solve");
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, split);
  pbem3d slp = new_slp_laplace_bem3d(gr, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D);
  pbem3d dlp = new_dlp_laplace_bem3d(gr, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D, 0.5);
  h2pair p;
  h2pair_new(&p, slp, dlp, BASIS_LINEAR_BEM3D, clf, eta, m);
  const double entries = near_entries(p.G[0]) + near_entries(p.G[1]);
  printf("{\"threads\": %d, \"triangles\": %u, \"vertices\": %u, \"entries_per_step\": %.0f, "
         "\"steps\": [", threads(), gr->triangles, gr->vertices, entries);
  for (uint s = 0; s < warmup + steps; s++) {
    double t[3] = {0, 0, 0};
    assemble(slp, p.G[0], t);
    assemble(dlp, p.G[1], t);
    if (s >= warmup)
      printf("%s{\"seconds\": %.6f, \"bases\": %.6f, \"nearfield\": %.6f, \"farfield\": %.6f}",
             s > warmup ? ", " : "", t[0] + t[1] + t[2], t[0], t[1], t[2]);
    fflush(stdout);
  }
  printf("]");
  if (solve) {
    pavector f = new_avector(gr->vertices), b = new_avector(gr->vertices),
             u = new_avector(gr->vertices);
    real z[3] = {1.2, 1.2, 1.2};
    uint iter;
    double ts, tm;
    projectL2_bem3d_l_avector(dlp, harmonic, f, z);
    clear_avector(b);
    addeval_h2matrix_avector(1.0, p.G[1], f, b);
    clear_avector(u);
    tic();
    addeval_h2matrix_avector(1.0, p.G[0], b, u);
    tm = toc();
    clear_avector(u);
    tic();
    iter = solve_gmres_h2matrix_avector(p.G[0], b, u, 1.0e-8, 1000, 50);
    ts = toc();
    printf(", \"solve\": {\"seconds\": %.6f, \"iterations\": %u, \"matvec_seconds\": %.6f}", ts,
           iter, tm);
    del_avector(f);
    del_avector(b);
    del_avector(u);
  }
  printf("}\n");
  h2pair_del(&p);
  del_laplace_bem3d(slp);
  del_laplace_bem3d(dlp);
  del_surface3d(gr);
  del_macrosurface3d(mg);
  return 0;
}
#else
typedef struct {
  ph2matrix V, KM;
  field eta;
} bw_t;

/* (K + M/2) - i eta V, the Brakhage-Werner operator of Tests/test_helmholtzbem3d.c */
static void addeval_bw(field alpha, void *matrix, pcavector x, pavector y) {
  bw_t *bw = (bw_t *) matrix;
  addeval_h2matrix_avector(alpha, bw->KM, x, y);
  addeval_h2matrix_avector(-I * alpha * bw->eta, bw->V, x, y);
}

static void plane_wave_rhs(pbem3d dlp, field k, const real dir[3], pavector b) {
  real kvec[3], src[3] = {0.0, 0.0, 0.0};
  helmholtz_data hd;
  for (int i = 0; i < 3; i++) kvec[i] = creal(k) * dir[i];
  hd.kvec = kvec;
  hd.source = src;
  hd.eta = creal(k);
  integrate_bem3d_c_avector(dlp, rhs_dirichlet_plane_helmholtzbem3d, b, (void *) &hd);
  scale_avector(-1.0, b);
}

static int mode_helmholtz(int argc, char **argv) {
  if (argc < 8) return 2;
  const uint split = atoi(argv[2]), clf = atoi(argv[4]), m = atoi(argv[6]);
  const field k = atof(argv[3]);
  const real eta = atof(argv[5]);
  const uint apps = atoi(argv[7]);
  const int solve = argc > 8 && !strcmp(argv[8], "--solve");
  pmacrosurface3d mg = new_cube_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, split);
  pbem3d slp = new_slp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D);
  pbem3d dlp =
      new_dlp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D, 0.5);
  h2pair p;
  h2pair_new(&p, slp, dlp, BASIS_CONSTANT_BEM3D, clf, eta, m);
  double t[3] = {0, 0, 0};
  assemble(slp, p.G[0], t);
  assemble(dlp, p.G[1], t);
  const double entries = near_entries(p.G[0]) + near_entries(p.G[1]);
  printf("{\"threads\": %d, \"triangles\": %u, \"k\": %g, \"entries\": %.0f, "
         "\"assembly\": {\"seconds\": %.6f, \"bases\": %.6f, \"nearfield\": %.6f, "
         "\"farfield\": %.6f}", threads(), gr->triangles, creal(k), entries, t[0] + t[1] + t[2],
         t[0], t[1], t[2]);
  bw_t bw = {p.G[0], p.G[1], creal(k)};
  pavector b = new_avector(gr->triangles), u = new_avector(gr->triangles);
  const real dir[3] = {1.0 / sqrt(3.0), 1.0 / sqrt(3.0), 1.0 / sqrt(3.0)};
  plane_wave_rhs(dlp, k, dir, b);
  double ta = 0.0;
  for (uint a = 0; a < apps; a++) {
    clear_avector(u);
    tic();
    addeval_bw(1.0, &bw, b, u);
    ta += toc();
  }
  printf(", \"application_seconds\": %.6f", apps ? ta / apps : 0.0);
  if (solve) {
    clear_avector(u);
    tic();
    const uint iter = solve_gmres_avector(&bw, addeval_bw, b, u, 1.0e-8, 1000, 80);
    printf(", \"solve\": {\"seconds\": %.6f, \"iterations\": %u}", toc(), iter);
  }
  printf("}\n");
  del_avector(b);
  del_avector(u);
  h2pair_del(&p);
  del_helmholtz_bem3d(slp);
  del_helmholtz_bem3d(dlp);
  del_surface3d(gr);
  del_macrosurface3d(mg);
  return 0;
}
#endif

/* ---------------------------------------------------------------------------------------- */
/* requests: uint32 count; per request: uint32 pde (0 Laplace, 1 Helmholtz), uint32 kmax,
 * uint32 maxiter, double k, double eps, uint32 nsrc, double src[3 nsrc] (Laplace: point sources;
 * Helmholtz: plane-wave directions), uint32 vertices, uint32 triangles, double x[3 vertices],
 * uint32 t[3 triangles]. */

static int rd(void *p, size_t sz, size_t n, FILE *f) { return fread(p, sz, n, f) == n; }

static int mode_requests(int argc, char **argv) {
  if (argc < 3) return 2;
  FILE *f = fopen(argv[2], "rb");
  const double budget = argc > 3 ? atof(argv[3]) : 1e30;
  pstopwatch total = new_stopwatch();
  uint32_t count;
  if (!f || !rd(&count, 4, 1, f)) return 2;
  printf("{\"threads\": %d, \"requests\": [", threads());
  int first = 1;
  start_stopwatch(total);
  for (uint32_t r = 0; r < count; r++) {
    uint32_t pde, kmax, maxiter, nv, nt, nsrc;
    double k, eps, src[3 * 16];
    if (!rd(&pde, 4, 1, f) || !rd(&kmax, 4, 1, f) || !rd(&maxiter, 4, 1, f) || !rd(&k, 8, 1, f) ||
        !rd(&eps, 8, 1, f) || !rd(&nsrc, 4, 1, f) || nsrc < 1 || nsrc > 16 ||
        !rd(src, 8, 3 * (size_t) nsrc, f) || !rd(&nv, 4, 1, f) || !rd(&nt, 4, 1, f))
      return 3;
    double *x = malloc(sizeof(double) * 3 * nv);
    uint32_t *t = malloc(sizeof(uint32_t) * 3 * nt);
    if (!rd(x, 8, 3 * (size_t) nv, f) || !rd(t, 4, 3 * (size_t) nt, f)) return 3;
#ifdef USE_COMPLEX
    const uint32_t mine = 1;
#else
    const uint32_t mine = 0;
#endif
    if (pde != mine || stop_stopwatch(total) > budget) {
      free(x);
      free(t);
      continue;
    }
    double ph[4] = {0, 0, 0, 0};
    uint iter = 0;
    tic();
    psurface3d gr = new_surface3d(nv, 1, nt);
    memcpy(gr->x, x, sizeof(double) * 3 * nv);
    memcpy(gr->t, t, sizeof(uint32_t) * 3 * nt);
    gr->e[0][0] = gr->e[0][1] = 0;
    prepare_surface3d(gr);
#ifndef USE_COMPLEX
    const basisfunctionbem3d basis = BASIS_LINEAR_BEM3D;
    const uint n = nv, m = 4;
    pbem3d op0 = new_slp_laplace_bem3d(gr, 2, 4, basis, basis);
    pbem3d op1 = new_dlp_laplace_bem3d(gr, 2, 4, basis, basis, 0.5);
#else
    const basisfunctionbem3d basis = BASIS_CONSTANT_BEM3D;
    const uint n = nt, m = 5;
    pbem3d op0 = new_slp_helmholtz_bem3d(k, gr, 2, 4, basis, basis);
    pbem3d op1 = new_dlp_helmholtz_bem3d(k, gr, 2, 4, basis, basis, 0.5);
#endif
    h2pair p;
    h2pair_new(&p, op0, op1, basis, 64, 1.4, m);
    ph[0] = toc();
    double ta[3] = {0, 0, 0};
    assemble(op0, p.G[0], ta);
    assemble(op1, p.G[1], ta);
    ph[1] = ta[0] + ta[1] + ta[2];
    pavector b = new_avector(n), u = new_avector(n);
    for (uint32_t q = 0; q < nsrc; q++) {
      tic();
#ifndef USE_COMPLEX
      pavector gd = new_avector(n);
      projectL2_bem3d_l_avector(op1, harmonic, gd, src + 3 * q);
      clear_avector(b);
      addeval_h2matrix_avector(1.0, p.G[1], gd, b);
      del_avector(gd);
#else
      plane_wave_rhs(op1, k, src + 3 * q, b);
#endif
      ph[2] += toc();
      clear_avector(u);
      tic();
#ifndef USE_COMPLEX
      iter += solve_gmres_h2matrix_avector(p.G[0], b, u, eps, maxiter, kmax);
#else
      bw_t bw = {p.G[0], p.G[1], k};
      iter += solve_gmres_avector(&bw, addeval_bw, b, u, eps, maxiter, kmax);
#endif
      ph[3] += toc();
    }
    printf("%s{\"index\": %u, \"unknowns\": %u, \"solves\": %u, \"setup\": %.6f, "
           "\"assembly\": %.6f, \"rhs\": %.6f, \"solve\": %.6f, \"iterations\": %u}",
           first ? "" : ", ", r, n, nsrc, ph[0], ph[1], ph[2], ph[3], iter);
    first = 0;
    fflush(stdout);
    del_avector(b);
    del_avector(u);
    h2pair_del(&p);
#ifndef USE_COMPLEX
    del_laplace_bem3d(op0);
    del_laplace_bem3d(op1);
#else
    del_helmholtz_bem3d(op0);
    del_helmholtz_bem3d(op1);
#endif
    del_surface3d(gr);
    free(x);
    free(t);
  }
  printf("]}\n");
  fclose(f);
  del_stopwatch(total);
  return 0;
}

#ifndef USE_COMPLEX
static int mode_green(int argc, char **argv) {
  if (argc < 9) return 2;
  const uint split = atoi(argv[2]), clf = atoi(argv[3]), m = atoi(argv[5]), l = atoi(argv[6]);
  real eta = atof(argv[4]);
  const real delta = atof(argv[7]), accur = atof(argv[8]);
  pmacrosurface3d mg = new_sphere_macrosurface3d();
  psurface3d gr = build_from_macrosurface3d_surface3d(mg, split);
  prepare_surface3d(gr);
  pbem3d slp = new_slp_laplace_bem3d(gr, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D);
  pcluster root = build_bem3d_cluster(slp, clf, BASIS_LINEAR_BEM3D);
  pblock broot = build_strict_block(root, root, &eta, admissible_max_cluster);
  pclusterbasis rb = build_from_cluster_clusterbasis(root);
  pclusterbasis cb = build_from_cluster_clusterbasis(root);
  ph2matrix G = build_from_block_h2matrix(broot, rb, cb);
  double t[3] = {0.0, 0.0, 0.0}, tm;
  pavector x, y;
  setup_h2matrix_aprx_greenhybrid_bem3d(slp, rb, cb, broot, m, l, delta, accur,
                                        build_bem3d_cube_quadpoints);
  assemble(slp, G, t);
  x = new_avector(gr->vertices);
  y = new_avector(gr->vertices);
  random_avector(x);
  clear_avector(y);
  tic();
  addeval_h2matrix_avector(1.0, G, x, y);
  tm = toc();
  printf("{\"threads\": %d, \"triangles\": %u, \"vertices\": %u, \"seconds\": %.6f, "
         "\"bases\": %.6f, \"nearfield\": %.6f, \"farfield\": %.6f, \"matvec_seconds\": %.6f, "
         "\"root_rank\": %u}\n",
         threads(), gr->triangles, gr->vertices, t[0] + t[1] + t[2], t[0], t[1], t[2], tm,
         rb->k);
  del_avector(x);
  del_avector(y);
  del_h2matrix(G);
  del_block(broot);
  freemem(root->idx);
  del_cluster(root);
  del_bem3d(slp);
  del_surface3d(gr);
  del_macrosurface3d(mg);
  return 0;
}
#endif

int main(int argc, char **argv) {
  int rc = 2;
  init_h2lib(&argc, &argv);
  sw = new_stopwatch();
  if (argc >= 2 && !strcmp(argv[1], "requests")) rc = mode_requests(argc, argv);
#ifndef USE_COMPLEX
  else if (argc >= 2 && !strcmp(argv[1], "assembly")) rc = mode_assembly(argc, argv);
  else if (argc >= 2 && !strcmp(argv[1], "green")) rc = mode_green(argc, argv);
#else
  else if (argc >= 2 && !strcmp(argv[1], "helmholtz")) rc = mode_helmholtz(argc, argv);
#endif
  if (rc == 2)
    fprintf(stderr,
            "usage: %s assembly split clf eta m steps warmup [--solve]   (real build)\n"
            "       %s green split clf eta m l delta accur               (real build)\n"
            "       %s helmholtz split k clf eta m applications [--solve] (complex build)\n"
            "       %s requests file\n", argv[0], argv[0], argv[0], argv[0]);
  del_stopwatch(sw);
  uninit_h2lib();
  return rc;
}
