/* Timed CPU baseline: the unmodified H2Lib reference (libh2ref_omp.so: OpenMP + AVX SIMD, built
 * from the reference's own sources by oracle/Makefile) assembling the Laplace single and double
 * layer H2 matrices of the Dirichlet benchmark through its public API.  Test / benchmark
 * infrastructure only.
 *
 * One "step" = row/column cluster bases, coupling matrices and the nearfield blocks of both
 * operators; with stride s > 1 only every s-th nearfield block is assembled (a bounded sample;
 * entries are counted for what was actually assembled).  Optionally (--solve) one GMRES(kmax)
 * solve of V u = (K + M/2) g_D to 1e-8 is timed after the steps.
 *
 * usage: ref_bench split clf eta m steps warmup stride [--solve]
 * prints one JSON object.
 */
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
#include "laplacebem3d.h"
#include "macrosurface3d.h"
#include "surface3d.h"

typedef struct {
  ph2matrix *near;
  uint n, cap;
} nlist_t;

static void
collect(ph2matrix G, nlist_t *l)
{
  uint i, j;
  if (G->f) {
    if (l->n == l->cap) {
      l->cap = l->cap ? 2 * l->cap : 1024;
      l->near = realloc(l->near, sizeof(ph2matrix) * l->cap);
    }
    l->near[l->n++] = G;
    return;
  }
  if (G->son)
    for (j = 0; j < G->csons; j++)
      for (i = 0; i < G->rsons; i++)
        collect(G->son[i + j * G->rsons], l);
}

static double
assemble_step(pbem3d bem, ph2matrix G, nlist_t *nl, uint stride, double *entries)
{
  pstopwatch sw = new_stopwatch();
  double t;
  long long cnt = 0;
  int b;
  start_stopwatch(sw);
  assemble_bem3d_h2matrix_row_clusterbasis(bem, G->rb);
  assemble_bem3d_h2matrix_col_clusterbasis(bem, G->cb);
  assemble_bem3d_farfield_h2matrix(bem, G);
#ifdef USE_OPENMP
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : cnt)
#endif
  for (b = 0; b < (int) nl->n; b += (int) stride) {
    ph2matrix Gb = nl->near[b];
    bem->nearfield(Gb->rb->t->idx, Gb->cb->t->idx, bem, false, Gb->f);
    cnt += (long long) Gb->f->rows * Gb->f->cols;
  }
  t = stop_stopwatch(sw);
  del_stopwatch(sw);
  *entries = (double) cnt;
  return t;
}

int
main(int argc, char **argv)
{
  uint split, clf, m, steps, warmup, stride, s;
  real eta;
  int solve = 0, threads = 1;
  pmacrosurface3d mg;
  psurface3d gr;
  pbem3d slp, dlp;
  pcluster root;
  pblock broot;
  pclusterbasis Vrb, Vcb, Krb, Kcb;
  ph2matrix V, K;
  nlist_t nv = {NULL, 0, 0}, nk = {NULL, 0, 0};
  double ev, ek;

  init_h2lib(&argc, &argv);
  if (argc < 8) {
    fprintf(stderr, "usage: %s split clf eta m steps warmup stride [--solve]\n", argv[0]);
    return 2;
  }
  split = atoi(argv[1]);
  clf = atoi(argv[2]);
  eta = atof(argv[3]);
  m = atoi(argv[4]);
  steps = atoi(argv[5]);
  warmup = atoi(argv[6]);
  stride = atoi(argv[7]);
  if (stride < 1) stride = 1;
  solve = argc > 8 && !strcmp(argv[8], "--solve");
#ifdef USE_OPENMP
  threads = omp_get_max_threads();
#endif

  mg = new_sphere_macrosurface3d();
  gr = build_from_macrosurface3d_surface3d(mg, split);
  slp = new_slp_laplace_bem3d(gr, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D);
  dlp = new_dlp_laplace_bem3d(gr, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D, 0.5);
  root = build_bem3d_cluster(slp, clf, BASIS_LINEAR_BEM3D);
  broot = build_strict_block(root, root, &eta, admissible_max_cluster);
  Vrb = build_from_cluster_clusterbasis(root);
  Vcb = build_from_cluster_clusterbasis(root);
  Krb = build_from_cluster_clusterbasis(root);
  Kcb = build_from_cluster_clusterbasis(root);
  V = build_from_block_h2matrix(broot, Vrb, Vcb);
  K = build_from_block_h2matrix(broot, Krb, Kcb);
  setup_h2matrix_aprx_inter_bem3d(slp, Vrb, Vcb, broot, m);
  setup_h2matrix_aprx_inter_bem3d(dlp, Krb, Kcb, broot, m);
  collect(V, &nv);
  collect(K, &nk);

  printf("{\"threads\": %d, \"triangles\": %u, \"vertices\": %u, \"near_blocks\": %u, "
         "\"stride\": %u, \"steps\": [", threads, gr->triangles, gr->vertices, nv.n, stride);
  for (s = 0; s < warmup + steps; s++) {
    double tv = assemble_step(slp, V, &nv, stride, &ev);
    double tk = assemble_step(dlp, K, &nk, stride, &ek);
    if (s >= warmup)
      printf("%s{\"seconds\": %.6f, \"entries\": %.0f}", s > warmup ? ", " : "", tv + tk,
             ev + ek);
    fflush(stdout);
  }
  printf("]");
  if (solve) {
    pavector f = new_avector(gr->vertices), b = new_avector(gr->vertices),
             u = new_avector(gr->vertices);
    pstopwatch sw = new_stopwatch();
    uint iter;
    double t;
    if (stride != 1) {
      /* the solve needs the complete nearfield */
      assemble_step(slp, V, &nv, 1, &ev);
      assemble_step(dlp, K, &nk, 1, &ek);
    }
    projectL2_bem3d_l_avector(dlp, eval_dirichlet_fundamental_laplacebem3d, f, NULL);
    clear_avector(b);
    addeval_h2matrix_avector(1.0, K, f, b);
    clear_avector(u);
    start_stopwatch(sw);
    iter = solve_gmres_h2matrix_avector(V, b, u, 1.0e-8, 1000, 50);
    t = stop_stopwatch(sw);
    printf(", \"solve\": {\"seconds\": %.6f, \"iterations\": %u, \"l2err\": %.6e}", t, iter,
           normL2diff_l_bem3d(slp, u, eval_neumann_fundamental_laplacebem3d, NULL)
           / normL2_bem3d(slp, eval_neumann_fundamental_laplacebem3d, NULL));
    del_stopwatch(sw);
    del_avector(f);
    del_avector(b);
    del_avector(u);
  }
  printf("}\n");
  return 0;
}
