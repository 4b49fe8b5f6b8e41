/* An H2Lib application for the drop-in test: it calls only H2Lib's own API, in the order the
 * reference's tests and examples do (Tests/test_laplacebem3d.c, Tests/test_helmholtzbem3d.c), and
 * writes what it computes to an output directory (raw arrays plus a manifest, as gen_golden.c).
 *
 * Built twice from this file: linked to H2Lib alone (the reference run on the CPU) and with the
 * h2b_h2lib shim in front of H2Lib (the same program on the B200).  tests/test_gpu_shim.py runs
 * both and compares.  With -DWITH_SHIM the program also re-runs the matrix-vector products with
 * the shim bypassed, i.e. H2Lib's own CPU code on the host structures the shim filled.
 *
 * Real build (Laplace): sphere refined x8, dense cc single layer; linear-basis single and double
 * layer H2 matrices (leaf 16, eta 1.4, m 3), products, and the interior Dirichlet GMRES(50) solve;
 * greenhybrid single and double layer H2 matrices on the sphere scaled and turned, products.
 * Complex build (Helmholtz, k = 2): the same sphere, constant basis: a single-layer block through
 * the nearfield callback, the dense double layer, single and double layer H2 matrices (leaf 16,
 * eta 1.4, m 3), products and a GMRES solve of V.
 *
 * usage: h2lib_app <outdir>
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
#include "h2matrix.h"
#include "krylovsolvers.h"
#include "macrosurface3d.h"
#include "surface3d.h"
#ifdef USE_COMPLEX
#include "helmholtzbem3d.h"
#else
#include "laplacebem3d.h"
#endif
#ifdef WITH_SHIM
#include "h2b_h2lib.h"
#endif

static const char *outdir;
static FILE *manifest;

static void dump(const char *name, const void *data, size_t n, size_t esize, const char *dt) {
  char path[4096];
  FILE *f;
  snprintf(path, sizeof(path), "%s/%s.bin", outdir, name);
  f = fopen(path, "wb");
  if (!f || (n > 0 && fwrite(data, esize, n, f) != n)) {
    perror(path);
    exit(1);
  }
  fclose(f);
  fprintf(manifest, "%s %s %zu\n", name, dt, n);
  fflush(manifest);
}

#ifdef USE_COMPLEX
#define FDT "c16"
#else
#define FDT "f8"
#endif

static void dump_vec(const char *name, pcavector v) { dump(name, v->v, v->dim, sizeof(field), FDT); }

static void dump_mat(const char *name, pcamatrix A) {
  field *buf = (field *) malloc(sizeof(field) * ((size_t) A->rows * A->cols + 1));
  for (uint j = 0; j < A->cols; j++)
    memcpy(buf + (size_t) j * A->rows, A->a + (size_t) j * A->ld, sizeof(field) * A->rows);
  dump(name, buf, (size_t) A->rows * A->cols, sizeof(field), FDT);
  free(buf);
}

static void dump_num(const char *name, double v) { dump(name, &v, 1, sizeof(double), "f8"); }

static void seeded(pavector x) {
  for (uint i = 0; i < x->dim; i++) {
#ifdef USE_COMPLEX
    x->v[i] = sin(0.37 * i) + 0.5 * cos(1.3 * i) + (cos(0.21 * i) - 0.25 * sin(2.1 * i)) * I;
#else
    x->v[i] = sin(0.37 * i) + 0.5 * cos(1.3 * i);
#endif
  }
}

/* Greenhybrid H2 matrix of `op` (m 2, l 1, delta 1, accuracy 5e-3, cube points: the reference
 * test's parameters), assembled the way Tests/test_laplacebem3d.c does it. */
#ifndef USE_COMPLEX
static ph2matrix green_of(pbem3d op, pcluster root, pblock broot) {
  pclusterbasis rb = build_from_cluster_clusterbasis(root);
  pclusterbasis cb = build_from_cluster_clusterbasis(root);
  ph2matrix G = build_from_block_h2matrix(broot, rb, cb);
  setup_h2matrix_aprx_greenhybrid_bem3d(op, rb, cb, broot, 2, 1, 1.0, 5e-3,
                                        build_bem3d_cube_quadpoints);
  assemble_bem3d_h2matrix_row_clusterbasis(op, rb);
  assemble_bem3d_h2matrix_col_clusterbasis(op, cb);
  assemble_bem3d_h2matrix(op, G);
  return G;
}

/* the sphere scaled to an ellipsoid and turned out of the axes (no pivot ties in the cross
 * approximations, whose winners would otherwise depend on the last bit of a quadrature sum) */
static void turn(psurface3d gr) {
  const real ax[3] = { 1.0, 0.8, 0.65 }, ca = cos(0.37), sa = sin(0.37), cb = cos(0.61),
             sb = sin(0.61), cc = cos(0.23), sc = sin(0.23);
  for (uint v = 0; v < gr->vertices; v++) {
    real p0 = gr->x[v][0] * ax[0], p1 = gr->x[v][1] * ax[1], p2 = gr->x[v][2] * ax[2], q0, q1, q2;
    q1 = cc * p1 - sc * p2;
    q2 = sc * p1 + cc * p2;
    q0 = cb * p0 + sb * q2;
    q2 = -sb * p0 + cb * q2;
    gr->x[v][0] = ca * q0 - sa * q1;
    gr->x[v][1] = sa * q0 + ca * q1;
    gr->x[v][2] = q2;
  }
  prepare_surface3d(gr);
}
#endif

/* H2 matrix of `op` on the tree of `root`, assembled the way H2Lib's tests do it. */
static ph2matrix h2_of(pbem3d op, pcluster root, pblock broot, uint m) {
  pclusterbasis rb = build_from_cluster_clusterbasis(root);
  pclusterbasis cb = build_from_cluster_clusterbasis(root);
  ph2matrix G = build_from_block_h2matrix(broot, rb, cb);
  setup_h2matrix_aprx_inter_bem3d(op, rb, cb, broot, m);
  assemble_bem3d_h2matrix_row_clusterbasis(op, rb);
  assemble_bem3d_h2matrix_col_clusterbasis(op, cb);
  assemble_bem3d_h2matrix(op, G);
  return G;
}

static void products(const char *tag, ph2matrix G, pcavector x) {
  char name[64];
  pavector y = new_avector(G->rb->t->size);
  clear_avector(y);
  addeval_h2matrix_avector(1.0, G, x, y);
  snprintf(name, sizeof(name), "y%s", tag);
  dump_vec(name, y);
  /* y += alpha A x accumulates into y */
  addeval_h2matrix_avector(-2.0, G, x, y);
  snprintf(name, sizeof(name), "y%s_acc", tag);
  dump_vec(name, y);
#ifdef WITH_SHIM
  /* H2Lib's own product on the host matrix the shim filled */
  h2b_shim_set_bypass(1);
  clear_avector(y);
  addeval_h2matrix_avector(1.0, G, x, y);
  h2b_shim_set_bypass(0);
  snprintf(name, sizeof(name), "y%s_host", tag);
  dump_vec(name, y);
#endif
  del_avector(y);
}

int main(int argc, char **argv) {
  char path[4096];
  pmacrosurface3d mg;
  psurface3d gr;
  pcluster root;
  pblock broot;
  real eta = 1.4;
  uint iter;

  init_h2lib(&argc, &argv);
  if (argc < 2) {
    fprintf(stderr, "usage: %s outdir\n", argv[0]);
    return 2;
  }
  outdir = argv[1];
  snprintf(path, sizeof(path), "%s/manifest.txt", outdir);
  manifest = fopen(path, "w");
  if (!manifest) {
    perror(path);
    return 1;
  }
  mg = new_sphere_macrosurface3d();
  gr = build_from_macrosurface3d_surface3d(mg, 8);

#ifndef USE_COMPLEX
  {
    /* dense constant-basis single layer (assemble_bem3d_amatrix) */
    pbem3d slpc = new_slp_laplace_bem3d(gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D);
    pamatrix A = new_amatrix(gr->triangles, gr->triangles);
    assemble_bem3d_amatrix(slpc, A);
    dump_mat("dense_slp_cc", A);
    del_amatrix(A);
    del_laplace_bem3d(slpc);
  }
  {
    pbem3d slp = new_slp_laplace_bem3d(gr, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D);
    pbem3d dlp = new_dlp_laplace_bem3d(gr, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D, 0.5);
    ph2matrix V, K;
    pavector x, f, b, u;
    root = build_bem3d_cluster(slp, 16, BASIS_LINEAR_BEM3D);
    broot = build_strict_block(root, root, &eta, admissible_max_cluster);
    V = h2_of(slp, root, broot, 3);
    K = h2_of(dlp, root, broot, 3);
    x = new_avector(gr->vertices);
    seeded(x);
    products("V", V, x);
    products("K", K, x);
    /* interior Dirichlet problem V u = (K + M/2) g_D, GMRES(50) to 1e-8 */
    f = new_avector(gr->vertices);
    b = new_avector(gr->vertices);
    u = new_avector(gr->vertices);
    projectL2_bem3d_l_avector(dlp, eval_dirichlet_fundamental_laplacebem3d, f, NULL);
    clear_avector(b);
    addeval_h2matrix_avector(1.0, K, f, b);
    dump_vec("b", b);
    clear_avector(u);
    iter = solve_gmres_h2matrix_avector(V, b, u, 1.0e-8, 1000, 50);
    dump_num("gmres_iter", (double) iter);
    dump_vec("u", u);
    clear_avector(u);
    iter = solve_gmres_avector(V, (addeval_t) addeval_h2matrix_avector, b, u, 1.0e-8, 1000, 50);
    dump_num("gmres_iter2", (double) iter);
    dump_vec("u2", u);
    del_avector(x);
    del_avector(f);
    del_avector(b);
    del_avector(u);
    del_h2matrix(V);
    del_h2matrix(K);
    del_block(broot);
    freemem(root->idx);
    del_cluster(root);
    del_laplace_bem3d(slp);
    del_laplace_bem3d(dlp);
  }
  {
    /* greenhybrid single and double layer on the turned ellipsoid */
    psurface3d ge = build_from_macrosurface3d_surface3d(mg, 8);
    pbem3d slp, dlp;
    ph2matrix V, K;
    pavector x;
    turn(ge);
    slp = new_slp_laplace_bem3d(ge, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D);
    dlp = new_dlp_laplace_bem3d(ge, 2, 4, BASIS_LINEAR_BEM3D, BASIS_LINEAR_BEM3D, 0.5);
    root = build_bem3d_cluster(slp, 16, BASIS_LINEAR_BEM3D);
    broot = build_strict_block(root, root, &eta, admissible_max_cluster);
    V = green_of(slp, root, broot);
    K = green_of(dlp, root, broot);
    x = new_avector(ge->vertices);
    seeded(x);
    products("Vg", V, x);
    products("Kg", K, x);
    del_avector(x);
    del_h2matrix(V);
    del_h2matrix(K);
    del_block(broot);
    freemem(root->idx);
    del_cluster(root);
    del_laplace_bem3d(slp);
    del_laplace_bem3d(dlp);
    del_surface3d(ge);
  }
#else
  {
    const field k = 2.0;
    pbem3d slp = new_slp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D);
    pbem3d dlp =
        new_dlp_helmholtz_bem3d(k, gr, 2, 4, BASIS_CONSTANT_BEM3D, BASIS_CONSTANT_BEM3D, 0.5);
    ph2matrix V, K;
    pavector x, u;
    pamatrix B = new_amatrix(7, 5), A = new_amatrix(gr->triangles, gr->triangles);
    uint ridx[7] = {5, 9, 20, 33, 2, 61, 40}, cidx[5] = {1, 40, 2, 60, 65};
    /* one block of the single layer through the nearfield callback (the plugin point); the
     * double layer's identity term is placed differently by H2Lib when a triangle appears at
     * different positions of ridx and cidx (assemble_cc_near_bem3d writes aa[t + t ld]), so the
     * double layer is compared on the whole matrix */
    slp->nearfield(ridx, cidx, slp, false, B);
    dump_mat("block_slp", B);
    assemble_bem3d_amatrix(dlp, A);
    dump_mat("dense_dlp_cc", A);
    del_amatrix(B);
    del_amatrix(A);
    root = build_bem3d_cluster(slp, 16, BASIS_CONSTANT_BEM3D);
    broot = build_strict_block(root, root, &eta, admissible_max_cluster);
    V = h2_of(slp, root, broot, 3);
    K = h2_of(dlp, root, broot, 3);
    x = new_avector(gr->triangles);
    seeded(x);
    products("V", V, x);
    products("K", K, x);
    u = new_avector(gr->triangles);
    clear_avector(u);
    iter = solve_gmres_h2matrix_avector(V, x, u, 1.0e-8, 1000, 50);
    dump_num("gmres_iter", (double) iter);
    dump_vec("u", u);
    del_avector(x);
    del_avector(u);
    del_h2matrix(V);
    del_h2matrix(K);
    del_block(broot);
    freemem(root->idx);
    del_cluster(root);
    del_helmholtz_bem3d(slp);
    del_helmholtz_bem3d(dlp);
  }
#endif
#ifdef WITH_SHIM
  {
    unsigned long long c[6];
    double d[6];
    h2b_shim_counts(c);
    for (int i = 0; i < 6; i++) d[i] = (double) c[i];
    dump("shim_counts", d, 6, sizeof(double), "f8");
  }
#endif
  del_surface3d(gr);
  del_macrosurface3d(mg);
  fclose(manifest);
  uninit_h2lib();
  return 0;
}
