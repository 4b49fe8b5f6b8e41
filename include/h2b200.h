/* h2b200 — B200-native boundary-element quadrature, H2 matrix-vector product and GMRES.
 *
 * The C ABI below is the drop-in boundary for H2Lib's 3D BEM hot path.  Every entry point takes
 * plain pointers and sizes; no CUDA, torch or H2Lib types appear in a signature, so H2Lib (C), a
 * ctypes binding or any FFI can call it.  Each function names the H2Lib interface it replaces
 * (file:line in the H2Lib source tree).
 *
 * Conventions shared with H2Lib:
 *   - matrices are column-major, entry (i,j) at a[i + j*ld], ld >= rows  (Library/amatrix.h:43);
 *   - "field" arrays of complex operators (Helmholtz) are interleaved (re, im) doubles, i.e. the
 *     memory layout of C99 `double _Complex` used by H2Lib's USE_COMPLEX build;
 *   - index lists (ridx/cidx) may be NULL meaning the identity 0..n-1  (Library/bem3d.h:380);
 *   - basis identifiers equal H2Lib's basisfunctionbem3d values: 'c' constant, 'l' linear
 *     (Library/bem3d.h:167-175).
 * Pointers to matrix/vector data may be host or device pointers; the library detects which and
 * copies as needed (host buffers are staged through pinned memory).
 *
 * Errors: every function returning int returns H2B_OK (0) or a negative H2B_ERR_* code and leaves
 * a message for h2b_last_error().  H2Lib itself aborts on errors (Library/basic.c:106-117); the
 * replacement reports them instead, and never falls back to a CPU computation: without a usable
 * CUDA device every compute entry point fails with H2B_ERR_CUDA.
 *
 * Threading: handles may be used from several host threads if each thread uses its own handle; a
 * single handle serialises its work on its own CUDA stream.
 */
#ifndef H2B200_H
#define H2B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define H2B_OK 0
#define H2B_ERR_ARG (-1)
#define H2B_ERR_NOMEM (-2)
#define H2B_ERR_CUDA (-3)
#define H2B_ERR_INTERNAL (-4)
#define H2B_ERR_STATE (-5)
#define H2B_ERR_TIMEOUT (-6)

#define H2B_BASIS_CONSTANT 'c'
#define H2B_BASIS_LINEAR 'l'

#define H2B_LAPLACE 0
#define H2B_HELMHOLTZ 1

#define H2B_SLP 0
#define H2B_DLP 1
#define H2B_ADLP 2 /* adjoint double layer K' (normal derivative in x) */

#define H2B_MESH_SPHERE 0
#define H2B_MESH_CUBE 1

/* Precision of an assembled operator / matvec. */
#define H2B_FP64 0
#define H2B_FP32 1

typedef struct h2b_surface h2b_surface;
typedef struct h2b_bem h2b_bem;
typedef struct h2b_tree h2b_tree;
typedef struct h2b_h2matrix h2b_h2matrix;

/* ------------------------------------------------------------------------------------------
 * Status
 * ------------------------------------------------------------------------------------------ */

/* Message of the last failed call on this host thread ("" if none). */
const char *h2b_last_error(void);

/* Library version string. */
const char *h2b_version(void);

/* Select and initialise the CUDA device used by handles created afterwards on this thread.
 * Returns H2B_ERR_CUDA if no sm_100 device is usable. */
int h2b_device_init(int device);

/* Device memory of the current device: out[0] free and out[1] total bytes (cudaMemGetInfo), out[2]
 * bytes in use and out[3] bytes reserved by the device's default stream-ordered memory pool, from
 * which every handle allocates.  Diagnostics; no reference counterpart. */
int h2b_device_memory(uint64_t out[4]);

/* Kernels the library has launched directly since it was loaded (all host threads): the
 * assembly, classification and matrix-vector kernels (a GMRES CUDA-graph launch is not counted
 * here).  Diagnostics; no reference counterpart. */
int h2b_launch_count(uint64_t *n);

/* ------------------------------------------------------------------------------------------
 * Host-side geometry (no GPU needed)
 * ------------------------------------------------------------------------------------------ */

/* Sizes of a refined macro surface.  Replaces new_sphere_macrosurface3d (Library/
 * macrosurface3d.c:81) / new_cube_macrosurface3d (:390) + build_from_macrosurface3d_surface3d
 * (:707): kind H2B_MESH_SPHERE or H2B_MESH_CUBE, split >= 1. */
int h2b_macro_mesh_size(int kind, uint32_t split, uint32_t *vertices, uint32_t *triangles);

/* Vertex coordinates x[3*vertices] and triangles t[3*triangles] of the refined macro surface, with
 * H2Lib's vertex and triangle numbering. */
int h2b_macro_mesh_build(int kind, uint32_t split, double *x, uint32_t *t);

/* Unit normals n[3*triangles], Gram determinants g[triangles] (= 2*area) and (hmin, hmax).
 * Replaces prepare_surface3d (Library/surface3d.c:51). hminmax may be NULL. */
int h2b_prepare_surface(uint32_t vertices, const double *x, uint32_t triangles,
                        const uint32_t *t, double *n, double *g, double *hminmax);

/* Scale vertex coordinates per axis (used to make ellipsoids from the sphere). */
int h2b_scale_vertices(uint32_t vertices, double *x, const double scale[3]);

/* Quadrature tables, for inspection and tests.  which: 0 distant, 1 vertex, 2 edge, 3 identical
 * Sauter-Schwab rule (Library/singquad2d.c:50/80/129/206), 4 single-triangle rule (:25).  Any
 * output pointer may be NULL; w10 receives 10*n weights (rows 0..8 basis-weighted, row 9 raw;
 * 4*n for the single-triangle rule).  Call once with all NULL to get n. */
int h2b_quad_export(uint32_t q, uint32_t q2, int row_basis, int col_basis, int which,
                    uint32_t *n, double *x0, double *x1, double *y0, double *y1, double *w10);

/* ------------------------------------------------------------------------------------------
 * Cluster tree and block tree
 * ------------------------------------------------------------------------------------------ */

/* Build the row and column cluster trees (build_bem3d_cluster, Library/bem3d.c:932 ->
 * build_adaptive_cluster, Library/cluster.c:80) and the strict block tree with the max-norm
 * admissibility (build_strict_block, Library/block.c:258 + admissible_max_cluster, :52).
 * row_basis/col_basis choose triangles ('c') or vertices ('l') as indices. */
h2b_tree *h2b_tree_new(uint32_t vertices, const double *x, uint32_t triangles,
                       const uint32_t *t, int row_basis, int col_basis, uint32_t clf,
                       double eta);

/* The same trees as h2b_tree_new (index for index), built on the device: characteristic points
 * and support boxes, the cluster bisection level by level (one CTA per cluster: bounding box,
 * longest side, and the reference's in-place partition replayed exactly) and the block
 * admissibility level by level; the host lays out the levels and numbers the result.  Replaces
 * build_adaptive_cluster (Library/cluster.c:80) and build_strict_block (Library/block.c:258) as
 * h2b_tree_new does.  The mesh arrays are host arrays. */
h2b_tree *h2b_tree_new_device(uint32_t vertices, const double *x, uint32_t triangles,
                              const uint32_t *t, int row_basis, int col_basis, uint32_t clf,
                              double eta);

/* Build from explicit flattened trees (what an H2Lib integration passes after walking its own
 * pcluster / pblock): per cluster in pre-order off, size, sons (0 or 2) and the bounding box
 * (bmin[3], bmax[3]); idx the root index array; per leaf block (block-tree pre-order, sons
 * column-major) the pre-order ids of its row and column clusters and its admissibility flag. */
h2b_tree *h2b_tree_new_flat(uint32_t row_clusters, const uint32_t *row_off,
                            const uint32_t *row_size, const uint32_t *row_sons,
                            const double *row_box, uint32_t row_n, const uint32_t *row_idx,
                            uint32_t col_clusters, const uint32_t *col_off,
                            const uint32_t *col_size, const uint32_t *col_sons,
                            const double *col_box, uint32_t col_n, const uint32_t *col_idx,
                            uint32_t blocks, const uint32_t *block_rc,
                            const uint32_t *block_cc, const uint8_t *block_adm);

/* A forest of independent surfaces: surface m owns vertices [vertex_off[m], vertex_off[m+1]) and
 * triangles [triangle_off[m], triangle_off[m+1]) of x / t (t holds global vertex ids).  Each
 * surface gets its own cluster trees and block tree (as h2b_tree_new on that surface alone);
 * the forest concatenates them, so an H2 matrix on it is block diagonal: one assembly and one
 * matvec serve all surfaces.  No H2Lib counterpart (H2Lib builds one tree per surface). */
h2b_tree *h2b_tree_new_forest(uint32_t surfaces, const uint32_t *vertex_off,
                              const uint32_t *triangle_off, const double *x, const uint32_t *t,
                              int row_basis, int col_basis, uint32_t clf, double eta);

void h2b_tree_del(h2b_tree *tree);

/* Counts: clusters of the row/column tree, index-set sizes, leaf blocks, admissible blocks,
 * nearfield entries (sum over inadmissible blocks of rows*cols), depth of the row/column tree. */
int h2b_tree_info(const h2b_tree *tree, uint64_t info[8]);

/* Export one tree (which = 0 row, 1 column): rec[3*clusters] = (off, size, sons), box[6*clusters]
 * = (bmin, bmax), idx[n].  Any pointer may be NULL. */
int h2b_tree_export_clusters(const h2b_tree *tree, int which, uint32_t *rec, double *box,
                             uint32_t *idx);

/* Export the leaf blocks: rec[5*blocks] = (row off, row size, col off, col size, admissible). */
int h2b_tree_export_blocks(const h2b_tree *tree, uint32_t *rec);

/* ------------------------------------------------------------------------------------------
 * Device-resident surface and operators
 * ------------------------------------------------------------------------------------------ */

/* Upload a surface mesh (vertices x[3*nv], triangles t[3*nt], normals n[3*nt], Gram determinants
 * g[nt] — the fields of H2Lib's struct _surface3d, Library/surface3d.h:45). */
h2b_surface *h2b_surface_new(uint32_t vertices, const double *x, uint32_t triangles,
                             const uint32_t *t, const double *n, const double *g);
void h2b_surface_del(h2b_surface *s);

/* Boundary integral operator.  Replaces
 *   new_slp_laplace_bem3d(gr, q_regular, q_singular, row, col)        Library/laplacebem3d.c:844
 *   new_dlp_laplace_bem3d(gr, q_regular, q_singular, row, col, alpha) Library/laplacebem3d.c:1012
 *   new_slp_helmholtz_bem3d(k, gr, q_regular, q_singular, row, col)   Library/helmholtzbem3d.c:1008
 *   new_dlp_helmholtz_bem3d(k, gr, ..., alpha)                        Library/helmholtzbem3d.c:1177
 *   new_adlp_laplace_bem3d(gr, q_regular, q_singular, row, col, alpha) Library/laplacebem3d.c:1180
 *   new_adlp_helmholtz_bem3d(k, gr, ..., alpha)                       Library/helmholtzbem3d.c:1346
 * pde H2B_LAPLACE / H2B_HELMHOLTZ, layer H2B_SLP / H2B_DLP / H2B_ADLP; (k_re, k_im) the wave
 * number (Helmholtz only; H2Lib's convention e^{i k r} with damping for Im k > 0); (alpha_re,
 * alpha_im) the coefficient of the identity added to the DLP or adjoint DLP (H2Lib's bem->alpha:
 * 0.5*alpha*g on the cc diagonal, alpha*mass*g for linear bases).  The adjoint double layer's
 * H2 row basis carries the normal derivative of the interpolation polynomials. */
h2b_bem *h2b_bem_new(const h2b_surface *s, int pde, int layer, int row_basis, int col_basis,
                     uint32_t q_regular, uint32_t q_singular, double k_re, double k_im,
                     double alpha_re, double alpha_im);
void h2b_bem_del(h2b_bem *bem);

/* Nearfield block fill — the bem->nearfield callback (Library/bem3d.h:380; implementations
 * assemble_cc_near_bem3d, Library/bem3d.c:1151, and assemble_ll_near_bem3d, :3038):
 * N[i + j*ld] = entry (ridx[i], cidx[j]) for i < rows, j < cols; with ntrans the conjugate
 * transpose is written, N[j + i*ld].  ridx/cidx: triangle (c) or vertex (l) indices; NULL =
 * identity.  N may be a host or device pointer; complex operators write interleaved pairs. */
int h2b_bem_nearfield(const h2b_bem *bem, const uint32_t *ridx, uint32_t rows,
                      const uint32_t *cidx, uint32_t cols, int ntrans, double *N, uint64_t ld);

/* Dense matrix of the whole operator.  Replaces assemble_bem3d_amatrix (Library/bem3d.c:9988).
 * G has n rows and n columns (n = triangles or vertices by basis), column-major with ld. */
int h2b_bem_assemble_amatrix(const h2b_bem *bem, double *G, uint64_t ld);

/* Device time (ms, CUDA events on the surface's stream) of the last h2b_bem_nearfield or
 * h2b_bem_assemble_amatrix call on this operator: [0] distant pairs, [1] singular pairs.  No
 * reference counterpart (diagnostics). */
int h2b_bem_timings(const h2b_bem *bem, double ms[2]);

/* ------------------------------------------------------------------------------------------
 * H2 matrices
 * ------------------------------------------------------------------------------------------ */

/* Device H2 matrix with Chebyshev interpolation of order m in each direction (rank m^3) on the
 * given trees.  Replaces build_from_cluster_clusterbasis (Library/clusterbasis.c:251) +
 * build_from_block_h2matrix (Library/h2matrix.c:438) + setup_h2matrix_aprx_inter_bem3d
 * (Library/bem3d.c:9658).  All storage is FP64. */
h2b_h2matrix *h2b_h2matrix_new(const h2b_bem *bem, const h2b_tree *tree, uint32_t m);
/* A second operator on the structure of `like` (same surface, trees, bases, quadrature order and
 * PDE, e.g. the double layer beside the single layer of a Dirichlet problem): the device trees,
 * block lists and nearfield plan are shared, not rebuilt; only the operator's own bases,
 * coupling and nearfield storage are allocated.  `like` must outlive the new matrix.  No
 * reference counterpart (H2Lib builds the cluster bases of each operator separately). */
h2b_h2matrix *h2b_h2matrix_new_like(const h2b_bem *bem, const h2b_h2matrix *like);
/* H2 matrix with the greenhybrid farfield (setup_h2matrix_aprx_greenhybrid_bem3d,
 * Library/bem3d.c:9689, with the cube quadrature points build_bem3d_cube_quadpoints, :5063):
 * m Gauss points on each of l parts per axis of every face of the cluster box widened by
 * delta * (largest box side), cluster bases from full-pivoting ACA to the accuracy `accur` of the
 * kernel matrix on those points, coupling matrices = the operator's entries between the pivot
 * rows and columns.  Ranks vary per cluster; the bases and couplings are padded to
 * k = 12 (m l)^2 columns.  Laplace single and double layer; 1 <= m l <= 3.  The assembly calls
 * are those of h2b_h2matrix_new (h2b_h2matrix_assemble, or the three basis / farfield calls and
 * the nearfield); h2b_h2matrix_new_like on it gives a second operator with its own greenhybrid
 * bases on the same structure. */
h2b_h2matrix *h2b_h2matrix_new_greenhybrid(const h2b_bem *bem, const h2b_tree *tree, uint32_t m,
                                           uint32_t l, double delta, double accur);
/* Ranks of the greenhybrid cluster bases (side 0 row, 1 column), one per cluster in the tree's
 * pre-order: ranks[clusters]. */
int h2b_h2matrix_green_ranks(const h2b_h2matrix *h, int side, uint32_t *ranks);
/* The greenhybrid bases and couplings in H2Lib's layouts with their per-cluster ranks (what the
 * reference's assemble_bem3d_greenhybrid_* callbacks leave in the clusterbasis and uniform
 * structs): part 0 / 2 the row / column leaf bases V_t (|t| x k_t, column-major, leaves in
 * pre-order), 1 / 3 the transfers E_s (k_s x k_father, column-major, non-root clusters in
 * pre-order), 4 the coupling matrices S (k_row x k_col, column-major, admissible blocks in the
 * tree's block order).  The nearfield is h2b_h2matrix_export part 5.  out NULL: only the count
 * in *ndoubles. */
int h2b_h2matrix_export_green(const h2b_h2matrix *h, int part, double *out, uint64_t *ndoubles);
void h2b_h2matrix_del(h2b_h2matrix *h2);

/* Assembly.  Replace assemble_bem3d_h2matrix_row_clusterbasis (Library/bem3d.c:10407),
 * _col_clusterbasis (:10436), assemble_bem3d_nearfield_h2matrix (:10325),
 * assemble_bem3d_farfield_h2matrix (:10337) and assemble_bem3d_h2matrix (:10313; nearfield +
 * farfield).  h2b_h2matrix_assemble_all does all five in one pass. */
int h2b_h2matrix_assemble_row_clusterbasis(h2b_h2matrix *h2);
int h2b_h2matrix_assemble_col_clusterbasis(h2b_h2matrix *h2);
int h2b_h2matrix_assemble_nearfield(h2b_h2matrix *h2);
int h2b_h2matrix_assemble_farfield(h2b_h2matrix *h2);
int h2b_h2matrix_assemble(h2b_h2matrix *h2);
int h2b_h2matrix_assemble_all(h2b_h2matrix *h2);

/* Assemble the nearfield blocks of two operators on the same tree in one pass: a single layer
 * (a) and a double layer (b) of the same PDE (Laplace, or Helmholtz with the same wavenumber)
 * share every triangle pair and quadrature point, and for Helmholtz the sine and cosine of each
 * point's k r.  No reference counterpart (the reference fills each operator's blocks). */
int h2b_h2matrix_assemble_nearfield_pair(h2b_h2matrix *a, h2b_h2matrix *b);

/* Storage and counts: info[0] nearfield entries, [1] coupling entries, [2] leaf-basis entries,
 * [3] transfer entries, [4] bytes of device storage, [5] admissible blocks, [6] nearfield blocks,
 * [7] rank k. */
int h2b_h2matrix_info(const h2b_h2matrix *h2, uint64_t info[8]);

/* Precision of the regular (distant-pair) nearfield quadrature of later assembly calls:
 * H2B_FP64 (default; entries match the reference to 1e-12) or H2B_FP32 (points, kernel values
 * and sums in FP32 for q = 2, about 1e-7 relative in those entries; singular pairs, bases and
 * coupling matrices stay FP64).  The mixed-precision assembly of a solve whose FP64 residual is
 * driven to 1e-8 on this operator; no counterpart in the reference (FP64 only). */
int h2b_h2matrix_set_precision(h2b_h2matrix *h2, int precision);

/* Launch shape of the matrix-vector product (the knobs h2b_h2matrix_autotune searches):
 * shape[0] rows per forward slice of a flattened column basis, [1] rows per backward slice of the
 * row basis, [2] resident CTAs per SM of the item kernel, [3] shared-memory ring stages per
 * consumer warp (1..4), [4] largest panel of a work item in KiB at FP64 storage (4..64; blocks
 * and slices are split to fit; the FP32 product's items hold twice the entries), [5] leaf-basis
 * CTAs per leaf, [6] consumer warps per CTA of the item kernel (1..8).  A value of 0 keeps the
 * current setting.  Slice and panel sizes belong to the matrix's structure: while matrices made
 * with h2b_h2matrix_new_like share it, neither they nor the model matrix can change them (only
 * [2], [3], [5] and [6]; H2B_ERR_STATE otherwise).  No reference counterpart. */
#define H2B_SHAPE_N 7
int h2b_h2matrix_set_matvec_shape(h2b_h2matrix *h2, const uint32_t shape[H2B_SHAPE_N]);
int h2b_h2matrix_get_matvec_shape(const h2b_h2matrix *h2, uint32_t shape[H2B_SHAPE_N]);

/* Autotuner: times candidate launch shapes on the assembled matrix itself (CUDA events on its
 * stream) and keeps the fastest.  H2B_TUNE_MATVEC searches the matvec shape (panels of 12, 16
 * and 24 KiB with slices as wide, 2..8 CTAs per SM, 1..4 consumer warps, 1..2 stages per warp,
 * every candidate whose CTAs fit an SM together); the cost is the FP64 product's time, plus the
 * FP32 product's when the matrix has FP32 copies.  A matrix whose structure is shared
 * (h2b_h2matrix_new_like, either side) keeps its panel size, and matrices made like this one
 * before the call keep their own launch shape.  H2B_TUNE_LEAF times the assembly of both cluster
 * bases at 1, 2, 4 and 8 CTAs per leaf and leaves the bases as the chosen split assembles them
 * (the splits order a leaf's quadrature sums differently, so entries change by rounding only;
 * FP32 copies are remade afterwards).  The result goes to a process-wide cache keyed by
 * (complex, rank k, floor(log2(rows * columns))) that h2b_h2matrix_new applies to later matrices
 * of the same class.  shape (optional) receives the chosen shape, ms (optional) [0] the matvec
 * cost at the starting shape, [1] at the chosen one, [2] the basis assembly at the starting
 * split, [3] at the chosen one (0 where not tuned).  Every candidate gives the same product up
 * to FP64 rounding (only the grouping of the atomic additions changes).  No reference
 * counterpart (H2Lib's only knob is its OpenMP task depth, Library/basic.c). */
#define H2B_TUNE_MATVEC 1u
#define H2B_TUNE_LEAF 2u
int h2b_h2matrix_autotune(h2b_h2matrix *h2, uint32_t flags, uint32_t shape[H2B_SHAPE_N],
                          double ms[4]);
/* The autotuner's cache as text (one line per size class), to carry tuned shapes across
 * processes; load merges into the cache and rejects a malformed file; clear empties it. */
int h2b_autotune_save(const char *path);
int h2b_autotune_load(const char *path);
int h2b_autotune_clear(void);

/* FP32 copies of the nearfield blocks, coupling matrices and flattened cluster bases, read by the
 * mixed-precision matvec (half the bytes of the FP64 product).  Call after assembly; any later
 * assembly call drops the copies.  No counterpart in the reference (FP64 only). */
int h2b_h2matrix_make_single(h2b_h2matrix *h2);

/* y += alpha A x read from the FP32 copies (FP64 vectors and sums); same arguments as
 * h2b_h2matrix_addeval.  Needs h2b_h2matrix_make_single. */
int h2b_h2matrix_addeval_single(double alpha_re, double alpha_im, const h2b_h2matrix *h2,
                                const double *x, double *y);

/* Device time (ms, CUDA events on the matrix's stream) of the last run of each phase:
 * [0] row basis, [1] column basis, [2] coupling, [3] nearfield distant pairs, [4] nearfield
 * singular pairs, [5] last matvec.  No reference counterpart (diagnostics). */
int h2b_h2matrix_timings(const h2b_h2matrix *h2, double ms[6]);

/* Triangle pairs evaluated by one nearfield assembly, by Sauter-Schwab case: [0] distant,
 * [1] common vertex, [2] common edge, [3] identical.  Every nearfield block evaluates all pairs
 * of triangles touching its row and column index sets, as assemble_ll_near_bem3d does
 * (Library/bem3d.c:3038).  No reference counterpart (diagnostics). */
int h2b_h2matrix_pair_counts(const h2b_h2matrix *h2, uint64_t counts[4]);

/* Distinct triangle pairs among those h2b_h2matrix_pair_counts counts, by the same cases: a pair
 * of triangles that several nearfield blocks touch (the linear basis) counts once.  Counted on the
 * device in a bitmap of triangles^2 bits (at most 131072 triangles); synchronises the matrix's
 * stream.  No reference counterpart (diagnostics). */
int h2b_h2matrix_unique_pairs(const h2b_h2matrix *h2, uint64_t counts[4]);

/* Copy parts back for inspection, in H2Lib's layouts and orders (pre-order, column-major):
 * part 0: leaf bases of the row basis, 1: transfer matrices of the row basis (all non-root
 * clusters), 2/3 the same for the column basis, 4: coupling matrices of the admissible blocks,
 * 5: nearfield blocks.  'count' limits the number of matrices (block-tree order); out may be NULL
 * to query the number of doubles. */
int h2b_h2matrix_export(const h2b_h2matrix *h2, int part, uint32_t count, double *out,
                        uint64_t *ndoubles);

/* The same copy for parts 0, 1, 4 and 5, queued on the matrix's own copy stream and returning at
 * once, so that an H2Lib host matrix can be filled while later assembly calls run (for example the
 * coupling matrices while the nearfield is assembled).  `out` should be pinned host memory for the
 * copy to overlap; it must stay valid until h2b_h2matrix_export_wait returns. */
int h2b_h2matrix_export_async(h2b_h2matrix *h2, int part, uint32_t count, double *out);
int h2b_h2matrix_export_wait(h2b_h2matrix *h2);

/* y += alpha * A x.  Replaces addeval_h2matrix_avector (Library/h2matrix.c:1269): forward
 * transform (Library/clusterbasis.c:524), coupling and nearfield (fastaddeval, Library/h2matrix.c:
 * 1211), backward transform (Library/clusterbasis.c:749).  x has columns, y rows entries of the
 * operator (complex operators: interleaved).  Host or device pointers. */
int h2b_h2matrix_addeval(double alpha_re, double alpha_im, const h2b_h2matrix *h2,
                         const double *x, double *y);

/* Same with nrhs right-hand sides stored as columns of X (ldx) and Y (ldy). */
int h2b_h2matrix_addeval_multi(double alpha_re, double alpha_im, const h2b_h2matrix *h2,
                               uint32_t nrhs, const double *X, uint64_t ldx, double *Y,
                               uint64_t ldy);

/* ------------------------------------------------------------------------------------------
 * GMRES
 * ------------------------------------------------------------------------------------------ */

/* Restarted GMRES with Householder QR on the operator  A = sum_i coef_i * H_i  (nterms H2
 * matrices of the same size; nterms = 1, coef = 1 for a single matrix).  Replaces
 * solve_gmres_avector (Library/krylovsolvers.c:183) with addeval_h2matrix_avector as operator,
 * i.e. solve_gmres_h2matrix_avector (:254), and Brakhage-Werner style combinations.  Same
 * algorithm as init_gmres / step_gmres / finish_gmres (Library/krylov.c:612/659/725): stops when
 * the estimated residual |rhat_k| <= eps * ||b||, restarts every kmax-1 steps, at most
 * maxiter-1 steps.  x holds the start vector and receives the solution.  Returns the number of
 * iterations (>= 0) or a negative H2B_ERR_* code.  coef is interleaved complex (2*nterms).
 * Two terms on one structure (h2b_h2matrix_new_like) for the same PDE, wavenumber and row basis,
 * neither an adjoint double layer (a double layer beside its single layer), are applied as one
 * product that reads their common coupling matrices and row basis once. */
int h2b_solve_gmres(uint32_t nterms, const h2b_h2matrix *const *ops, const double *coef,
                    const double *b, double *x, double eps, uint32_t maxiter, uint32_t kmax);

/* Many independent systems at once: the operator must be block diagonal with diagonal blocks on
 * the row ranges [system_off[s], system_off[s+1]) (an H2 matrix on a forest, h2b_tree_new_forest;
 * system_off[0] = 0, system_off[systems] = the operator size).  Each system runs the GMRES of
 * h2b_solve_gmres on its own rows — own Krylov basis, residual estimate, restarts and stop at
 * eps * ||b_s|| or maxiter — while one operator application per step serves all of them.
 * iterations[s] (may be NULL) receives each system's step count.  No counterpart in the
 * reference, which solves one system per solve_gmres_avector call. */
#define H2B_SOLVE_MIXED 1u
/* Complex systems: Givens rotations in unitary form.  The reference's complex rotation
 * (Library/krylov.c:551/587) is not a unitary matrix, so for Helmholtz operators its residual
 * estimate |rhat_k| can lie orders of magnitude below the true residual and the solve stops
 * early; h2b_solve_gmres keeps that behaviour (same iteration counts as the reference).  With
 * this flag the rotation is unitary and |rhat_k| is the residual norm.  Real systems are
 * unaffected (both forms coincide); H2B_SOLVE_MIXED implies it. */
#define H2B_SOLVE_UNITARY 2u
int h2b_solve_gmres_batch(uint32_t nterms, const h2b_h2matrix *const *ops, const double *coef,
                          uint32_t systems, const uint32_t *system_off, uint32_t nrhs,
                          const double *b, double *x, double eps, uint32_t maxiter, uint32_t kmax,
                          uint32_t flags, uint32_t *iterations);
/* With nrhs > 1, b and x hold nrhs columns of the operator size (column r at r * size) and
 * system (s, r) is segment s of column r; iterations has systems * nrhs entries (s + r * systems).
 * flags: H2B_SOLVE_MIXED runs the Arnoldi steps on the FP32 copies of the matrices
 * (h2b_h2matrix_make_single) and keeps residuals in FP64: every (re)start computes the FP64
 * residual b - A x, and a system whose residual estimate reaches eps * ||b|| restarts once more
 * to confirm it with the FP64 residual, so the returned x meets eps in FP64 — restarted GMRES
 * as iterative refinement with a single-precision inner operator. */

/* h2b_solve_gmres with the mixed-precision iteration of H2B_SOLVE_MIXED (one system; unitary
 * rotations). */
int h2b_solve_gmres_mixed(uint32_t nterms, const h2b_h2matrix *const *ops, const double *coef,
                          const double *b, double *x, double eps, uint32_t maxiter,
                          uint32_t kmax);

/* GMRES that allocates nothing.  No counterpart in the reference (H2Lib allocates its Krylov work
 * space with new_avector / new_amatrix in solve_gmres_avector).  For callers that cannot allocate
 * device memory during a solve — a device-memory budget fixed at start-up, an allocator owned by
 * another framework, or a real-time loop that forbids allocation calls — this variant of
 * h2b_solve_gmres takes its work space (Householder vectors, compact-WY factor, staging vectors)
 * from a fixed device array of H2B_NOALLOC_SCRATCH_BYTES bytes compiled into the library, which
 * every GPU that loads the library holds until the process exits, and launches the step kernels
 * directly (no CUDA graph, one host round trip per Arnoldi step).  Problems whose work space
 * exceeds the array are rejected with H2B_ERR_ARG; the work space is slightly more than
 * 8 * (n * kmax + 4 n) bytes (twice that for complex operators): it is
 * 8 (W n (kmax + 4) + 2 kmax^2 + 8 kmax + 2 ceil(n / 256) (kmax + 1)) bytes plus about 1 KiB,
 * W = 1 real, 2 complex.  Same algorithm, arguments and result as h2b_solve_gmres; b and x may be host
 * or device pointers.  Every call looks up the array's device address (cudaGetSymbolAddress); the
 * first call on a device loads the module, so make it before any stream capture.  All calls share
 * the array and it keeps the last call's contents; calls that overlap on the GPU race, so
 * serialise them.  Every call, a failed one included, waits for its GPU work before returning. */
#define H2B_NOALLOC_SCRATCH_BYTES (24u << 20)
int h2b_solve_gmres_noalloc(uint32_t nterms, const h2b_h2matrix *const *ops, const double *coef,
                            const double *b, double *x, double eps, uint32_t maxiter,
                            uint32_t kmax);

/* Relative residual ||b - A x|| / ||b|| computed in FP64 on the device (diagnostic). */
int h2b_residual_norm(uint32_t nterms, const h2b_h2matrix *const *ops, const double *coef,
                      const double *b, const double *x, double *relres);

/* ------------------------------------------------------------------------------------------
 * Right-hand sides and errors (Laplace test data)
 * ------------------------------------------------------------------------------------------ */

/* L2 projection of the harmonic function g(x) = 1/|x - z| onto the linear basis.  Replaces
 * projectL2_bem3d_l_avector (Library/bem3d.c:9009) with f = eval_dirichlet_fundamental_
 * laplacebem3d (Library/laplacebem3d.c:1391; z = (1.2, 1.2, 1.2) there).  Result in w[vertices]
 * (host or device). */
int h2b_project_l2_harmonic(const h2b_bem *bem, const double z[3], double *w);

/* L2 norm of the difference between the linear-basis function u and the Neumann trace
 * d/dn 1/|x - z| (normL2diff_l_bem3d, Library/bem3d.c:8954 with
 * eval_neumann_fundamental_laplacebem3d, Library/laplacebem3d.c:1412), and the norm of the trace
 * itself (normL2_bem3d, :8704). */
int h2b_l2_error_harmonic(const h2b_bem *bem, const double z[3], const double *u, double *err,
                          double *norm);

/* The same for an operator on a union of surfaces (triangle ranges triangle_off[s] ..
 * triangle_off[s+1], triangle_off[surfaces] = all triangles) and nrhs columns: the source of
 * surface s in column r is zs[3 (s + r surfaces)]; w and u hold nrhs columns of the vertex count;
 * err / norm receive surfaces * nrhs values (s + r surfaces). */
int h2b_project_l2_harmonic_multi(const h2b_bem *bem, uint32_t surfaces,
                                  const uint32_t *triangle_off, uint32_t nrhs, const double *zs,
                                  double *w);
int h2b_l2_error_harmonic_multi(const h2b_bem *bem, uint32_t surfaces,
                                const uint32_t *triangle_off, uint32_t nrhs, const double *zs,
                                const double *u, double *err, double *norm);

/* b[t] = coef * int_{triangle t} exp(i kvec . (x - src)) dx for the constant basis (a plane wave
 * as Dirichlet datum).  Replaces integrate_bem3d_c_avector (Library/bem3d.c:8579) with
 * rhs_dirichlet_plane_helmholtzbem3d (Library/helmholtzbem3d.c:1611); coef = -1 gives the
 * datum -u_inc of a sound-soft scatterer.  b: interleaved complex, host or device. */
int h2b_integrate_plane_wave(const h2b_bem *bem, const double kvec[3], const double src[3],
                             double coef_re, double coef_im, double *b);

/* b = coef * int f(x) phi_i(x) dx for the point source f(x) = e^{ik|x - src|} / |x - src| (real
 * k >= 0), tested with the operator's row basis: b[t] per triangle for the constant basis, b[v]
 * per vertex for the linear basis.  Replaces integrate_bem3d_c_avector / _l_avector
 * (Library/bem3d.c:8579 / :8631) with rhs_dirichlet_point_helmholtzbem3d
 * (Library/helmholtzbem3d.c:1521), the Dirichlet datum of the reference's exterior test problem
 * (Tests/test_helmholtzbem3d.c:422) whose exact solution is f itself.  b: interleaved complex,
 * host or device. */
int h2b_integrate_point_source(const h2b_bem *bem, const double src[3], double k, double coef_re,
                               double coef_im, double *b);

/* u[p] = the Brakhage-Werner potential of the density w (the operator's column basis, complex) at
 * points[3 p] outside the surface: sum over triangles of int (d_n(y) G(x, y) - i eta G(x, y)) w(y)
 * dy with the operator's wavenumber, by the single-triangle rule.  The evaluation of
 * eval_brakhage_werner_c / _l (Tests/test_helmholtzbem3d.c:68 / :134), with which the reference
 * states a solve's error against the exact exterior field.  npoints <= 2^24; points, w, u host or
 * device (u interleaved complex). */
int h2b_eval_brakhage_werner(const h2b_bem *bem, uint32_t npoints, const double *points,
                             const double *w, double eta_re, double eta_im, double *u);

/* ------------------------------------------------------------------------------------------
 * Solve server: continuous admission of Dirichlet solves (no counterpart in the reference,
 * which solves one problem per program run)
 * ------------------------------------------------------------------------------------------ */

typedef struct h2b_server h2b_server;

/* One request.  pde = H2B_LAPLACE: interior Dirichlet problem of 1/|x - src| (src outside the
 * surface), V du/dn = (K + M/2) g_D with the linear basis (m = 4); the solution has `vertices`
 * entries.  pde = H2B_HELMHOLTZ: Brakhage-Werner ((K + M/2) - i k V) u = -int exp(i k src.x)
 * for the plane wave of unit direction src and wavenumber k, constant basis (m = 5); the solution
 * has `triangles` complex (interleaved) entries.  Both use q = 2/4, leaf size 64, eta = 1.4 and
 * GMRES(kmax) to eps (flags: H2B_SOLVE_MIXED for FP32 Arnoldi steps with FP64 residuals).  The
 * server always uses the unitary rotations of H2B_SOLVE_UNITARY, so every result meets eps in
 * the true residual. */
typedef struct {
  uint32_t vertices, triangles;
  const double *x;
  const uint32_t *t;
  int pde;
  double k;
  double src[3];
  double eps;
  uint32_t maxiter, kmax, flags;
} h2b_request;

typedef struct {
  int status;                /* H2B_OK or the error of the request */
  uint32_t iterations, unknowns;
  double rel_residual;       /* FP64 ||b - A u|| / ||b|| after the solve */
  double t_submit, t_start, t_done;  /* seconds since the server started */
  uint64_t bytes_reserved;   /* device-memory estimate charged against the budget */
  /* seconds spent in: surface + trees + H2 structure, assembly, right-hand side, solve */
  double t_setup, t_assembly, t_rhs, t_solve;
} h2b_request_result;

/* A server with `slots` worker threads on `device` admitting requests while their estimated
 * device memory fits hbm_budget_bytes.  Requests run concurrently on their own streams. */
h2b_server *h2b_server_new(int device, uint32_t slots, uint64_t hbm_budget_bytes);
/* Queue a request (the mesh is copied); returns its id (> 0) or a negative error. */
int64_t h2b_server_submit(h2b_server *server, const h2b_request *request);
/* Block until request `id` is done; copy its solution (may be NULL) and result, then forget it. */
int h2b_server_wait(h2b_server *server, int64_t id, double *solution, h2b_request_result *res);
/* queued, running, completed requests and reserved bytes */
int h2b_server_stats(h2b_server *server, uint64_t out[4]);
/* Continuous batching: a worker takes up to max_requests queued requests that can share one
 * operator (Laplace problems with equal flags, eps, maxiter and kmax) and solves them as one
 * forest H2 matrix with a batched GMRES (default 64; 1 solves every request alone). */
int h2b_server_set_batching(h2b_server *server, uint32_t max_requests);
/* Finish running requests, drop queued ones, stop the workers. */
void h2b_server_del(h2b_server *server);

#ifdef __cplusplus
}
#endif

#endif
