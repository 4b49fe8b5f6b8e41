// Greenhybrid cluster bases and coupling matrices (setup_h2matrix_aprx_greenhybrid_bem3d,
// Library/bem3d.c:9689) for the Laplace single and double layer.
//
// Per cluster t, bottom-up one tree level per launch: the matrix A_t of the row basis functions
// of t (a leaf's own, or its sons' pivot rows) against the fundamental solution and its normal
// derivative at the 6 (ml)^2 quadrature points of the surface of t's box widened by
// delta * diam_max(t) (build_bem3d_cube_quadpoints, Library/bem3d.c:5063), compressed by ACA with
// full pivoting to the accuracy `accur` (decomp_fullaca_rkmatrix, Library/aca.c:18); the basis is
// the cross approximation's row factor normalised to the identity on the pivot rows
// (assemble_bem3d_greenhybrid_leaf_row_clusterbasis / _transfer_row_, Library/bem3d.c:6194 and
// :6262; column side :6343 and :6412).  Every rank is padded to K = 12 (ml)^2 with zero columns,
// so the flattened bases and the coupling matrices have the layout of the interpolation path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"

#define H2B_GREEN_MLMAX 3   // K = 12 (ml)^2 <= 108

struct GreenArgs {
  const TriRec *tri;
  const uint32_t *vt_off, *vt_tri;   // vertex -> triangles
  const double *xs, *ys, *ws, *wsl;  // single-triangle rule: raw weights, corner-weighted (3 ns)
  int ns;
  int linear;      // this side's basis functions are the piecewise linear ones (vertices)
  int dcol;        // column side of the double layer (fill_dcol / fill_dnzdcol kernels)
  int transposed;  // column side: leaf bases stored as V^T
  double kconst;
  const uint32_t *clusters;  // the clusters of this launch (one tree level)
  uint32_t n;
  const uint32_t *off, *size, *son0, *son1, *idx;
  const double *box;         // per cluster: bmin[3], bmax[3]
  const uint64_t *voff;      // leaf basis offsets
  double tg[3 * H2B_GREEN_MLMAX], wg[3 * H2B_GREEN_MLMAX];  // per-axis rule on [-1, 1]
  int ml, K;
  double delta, accur;
  uint32_t max_rows;         // bound on the rows of A_t over the launch
  uint32_t *rank;            // per cluster
  uint32_t *piv;             // per cluster: K global basis ids of the pivot rows
  double *V;                 // leaf bases
  double *E;                 // per cluster: K x K transfer to the father (column-major)
};

#define H2B_GREEN_FLAT_ROWS 64  // rows of a son per flatten item

struct GreenFlatArgs {
  const uint32_t *items;  // per item (father, son, first row, rows) of one level
  uint32_t n;
  const uint32_t *off, *size, *son0, *son1, *rank;
  const uint64_t *woff;
  const double *E;
  double *W;
  int K;
};

struct GreenCouplingArgs {
  const TriRec *tri;
  const uint32_t *vt_off, *vt_tri;
  const uint32_t *adm_rc, *adm_cc;
  const uint32_t *rrank, *rpiv, *crank, *cpiv;
  double *S;
  uint32_t n;
  int K, q, rlinear, clinear, dlp;
  double kconst;
  uint32_t max_elems;  // bound on a block's column triangles over its pivots (K x the largest
                       // vertex degree, or K for constant bases)
};

extern "C" {
size_t h2b_green_smem(uint32_t max_rows, int K);
int h2b_green_basis(const GreenArgs *a, cudaStream_t st);
int h2b_green_flatten(const GreenFlatArgs *a, cudaStream_t st);
int h2b_green_coupling(const GreenCouplingArgs *a, cudaStream_t st);
}
