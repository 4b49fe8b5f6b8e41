// H2 matrix handle layout shared by api_h2.cu and api_solve.cu.
#pragma once

#include <atomic>

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "api_internal.h"
#include "farfield.h"
#include "h2b200_tree.h"
#include "h2mvm.h"

struct DevCTree {
  uint32_t n = 0, nidx = 0, depth = 0, nleaves = 0, max_rows = 0, nnonroot = 0;
  uint64_t vtotal = 0;
  uint32_t *d_off = nullptr, *d_size = nullptr, *d_father = nullptr, *d_son0 = nullptr,
           *d_son1 = nullptr, *d_idx = nullptr, *d_leaves = nullptr, *d_nonroot = nullptr;
  uint64_t *d_voff = nullptr;
  double *d_pts = nullptr, *d_V = nullptr, *d_E = nullptr;
  TriRef *d_refs = nullptr;
  uint32_t *d_tr_off = nullptr, *d_tr_len = nullptr;
  std::vector<uint32_t> leaves;
  // flattened bases (flatbasis.cu): W_t for every cluster of an admissible block and below
  double *d_W = nullptr;
  uint64_t *d_woff = nullptr;
  uint64_t wtotal = 0;
  uint32_t *d_fitems = nullptr;  // flatten items (4 uint32 each: pair, first row, rows, 0)
  uint32_t *d_wleaves = nullptr; // leaves that carry a W (W_leaf = V_leaf)
  // (leaf, ancestor) pairs of the flattened bases: d_ppairs[2 p] = leaf, [2 p + 1] = ancestor;
  // the pairs of needed leaf i are d_pfirst[i] .. d_pfirst[i + 1] - 1, nearest ancestor first
  uint32_t *d_ppairs = nullptr, *d_pfirst = nullptr;
  uint32_t nwleaves = 0, npairs = 0, nfitems = 0;
  double *d_P = nullptr;  // per pair: the three m x m products of one-dimensional transfers
  std::vector<uint64_t> h_woff;  // host copy of d_woff
  std::vector<char> h_adm;       // 1: the cluster belongs to an admissible block
  std::vector<uint32_t> h_seg;   // host copy of d_seg
  float *f_W = nullptr;  // FP32 copy of W (h2b_h2matrix_make_single)
  // surfaces of a forest: the surface of every cluster (device) and the roots (host)
  uint32_t *d_seg = nullptr;
  std::vector<uint32_t> roots;
  const uint32_t *h_idx = nullptr, *h_off = nullptr, *h_size = nullptr;  // the host tree
  // greenhybrid bases (green.cu).  Structure: per cluster box (bmin, bmax), the clusters by
  // level (deepest first, with a bound on the rows of A_t per level) and the flatten items of the
  // needed non-leaf clusters by level (4 uint32 each).  Per operator: ranks, pivots (K per cluster), transfers (K x K).
  double *d_gbox = nullptr;
  uint32_t *d_glev = nullptr, *d_gflat = nullptr;
  std::vector<uint32_t> h_glev_off, h_glev_rows, h_gflat_off;
  uint32_t *d_grank = nullptr, *d_gpiv = nullptr;
  double *d_gE = nullptr;
};

struct h2b_h2matrix {
  const h2b_bem *bem = nullptr;
  const h2b_tree *tree = nullptr;
  uint32_t m = 0, k = 0, ns = 0;
  // greenhybrid farfield (h2b_h2matrix_new_greenhybrid): points per axis and face ml = m l, the
  // one-dimensional rule on [-1, 1], the box widening delta and the ACA accuracy; k = 12 ml^2
  int green = 0;
  int g_ml = 0;
  // 1: equal row and column trees and bases (the column basis of the single layer is then the
  // row basis); g_row_ready: the row basis of the current assembly is in place
  int g_same = 0, g_row_ready = 0;
  int g_col_copied = 0;  // the column basis was copied (its leaf bases are the row side's)
  double g_tg[9] = {}, g_wg[9] = {}, g_delta = 0.0, g_accur = 0.0;
  int cx = 0, num_sms = 148;
  int quad_fp32 = 0;  // distant-pair quadrature in FP32 (h2b_h2matrix_set_precision)
  // matvec work items (h2mvm.h), owned by the structure's owner, and the knobs they were built
  // with: rows per forward / backward slice, largest panel; CTAs per SM, consumer warps and
  // stages per consumer warp of the item kernel
  MvItem *d_items = nullptr, *d_items_single = nullptr;
  MvItems mvitems = {}, mvitems_single = {};  // the FP64 product's and the FP32 product's
  uint32_t mv_fwd_rows = 32, mv_back_rows = 32;
  int mv_ctas = 4, mv_warps = 3, mv_stages = 1;
  uint32_t mv_panel_bytes = H2B_MV_PANEL_BYTES;
  int leaf_split = 2;  // CTAs per leaf of the leaf-basis kernel (each a range of the k columns)
  int *d_mverr = nullptr;  // the item kernel's error flag (one per matrix)
  // host copies of the block lists: admissible (row, column cluster), nearfield (row, column
  // cluster, offset of the block in N)
  std::vector<uint32_t> h_arc, h_acc, h_nrc, h_ncc;
  std::vector<uint64_t> h_noff;
  // 1: the tree, block and nearfield-plan arrays belong to another matrix (h2b_h2matrix_new_like);
  // only the operator's own data (bases, transfers, W, S, N, work vectors) are freed here
  int shared = 0;
  // the matrix whose structure this one shares, and (on that matrix) how many matrices share its
  // structure: while any do, its slice and panel sizes (the shared work items) stay fixed
  const h2b_h2matrix *owner = nullptr;
  struct Count {  // a copy (h2b_h2matrix_new_like) starts at zero
    std::atomic<int> n{0};
    Count() = default;
    Count(const Count &) {}
    Count &operator=(const Count &) { return *this; }
  };
  mutable Count sharers;
  cudaStream_t st = nullptr;
  DevCTree rt, ct;
  uint32_t nadm = 0, nnear = 0, ntiles = 0, nsing = 0;
  uint64_t near_total = 0;
  uint32_t *d_adm_rc = nullptr, *d_adm_cc = nullptr;
  double *d_S = nullptr;
  uint32_t *d_near_rc = nullptr, *d_near_cc = nullptr;
  uint64_t *d_near_off = nullptr;
  double *d_N = nullptr;
  float *f_S = nullptr, *f_N = nullptr;  // FP32 copies (h2b_h2matrix_make_single)
  h2b_tile *d_tiles = nullptr;
  h2b_triref *d_refs = nullptr;
  h2b_sing *d_sing = nullptr;
  double *d_xp = nullptr, *d_yp = nullptr, *d_xt = nullptr, *d_yt = nullptr;
  double *d_xio = nullptr, *d_yio = nullptr;  // staging of host vectors
  double *d_xs = nullptr, *d_ys = nullptr, *d_ws = nullptr, *d_wsl = nullptr;
  MvmPlan mvm;
  // pair counts of the nearfield plan by Sauter-Schwab case (distant, vertex, edge, identical)
  uint64_t pairs[4] = {0, 0, 0, 0};
  // device timings of the last assembly phases (ms): row basis, column basis, coupling,
  // nearfield distant, nearfield singular, matvec
  cudaEvent_t ev[12] = {};
  cudaStream_t cst = nullptr;     // copy stream of h2b_h2matrix_export_async
  cudaEvent_t ev_copy = nullptr;
  float ms[6] = {0, 0, 0, 0, 0, 0};
};

void h2b_h2_fill_mvm_plan(h2b_h2matrix *h);
// (Re)build the matvec work items from the structure and the matrix's slice knobs (owner only).
int h2b_h2_build_mv_items(h2b_h2matrix *h);
// Applies the autotuner's cached shape for h's size class, if any (before the items are built).
void h2b_tune_lookup(h2b_h2matrix *h);
// H2B_ERR_TIMEOUT (and the flag cleared) if a matvec of h lost a panel copy; synchronises h->st.
int h2b_h2_check_mv_error(const h2b_h2matrix *h);
// Bytes of slack after every panel array: a panel copy may read up to 15 bytes past its panel.
#define H2B_MV_SLACK 64
int h2b_h2_addeval_dev(const h2b_h2matrix *h, double ar, double ai, const double *dx, double *dy,
                       cudaStream_t st);
