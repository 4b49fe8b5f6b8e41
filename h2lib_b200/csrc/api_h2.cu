// C-ABI implementation: H2 matrices (structure upload, assembly, export, matvec).
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "api_h2.h"
#include "green.h"

// ------------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------------

template <typename T>
static int upload(T **dst, const std::vector<T> &src, cudaStream_t st) {
  *dst = nullptr;
  if (src.empty()) return H2B_OK;
  H2B_CUDA_TRY(cudaMallocAsync((void **) dst, sizeof(T) * src.size(), st));
  H2B_CUDA_TRY(cudaMemcpyAsync(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice,
                               st));
  return H2B_OK;
}

// Device memory of the H2 structures is stream-ordered (cudaMallocAsync / cudaFreeAsync on the
// matrix's stream, served from the device's memory pool): creating and releasing matrices never
// synchronises the device, so matrices of concurrent requests do not stall each other.
template <typename T>
static void dfree(T *&p, cudaStream_t st) {
  if (p) cudaFreeAsync((void *) p, st);
  p = nullptr;
}

// Chebyshev nodes cos(pi (2i+1)/(2m)) (setup_interpolation_bem3d, Library/bem3d.c:4978) mapped to
// the box [a, b] of each axis, widened by 5e-3 on both sides when narrower than 5e-3
// (assemble_interpoints3d_realavector, Library/bem3d.c:5236).
static void box_points(const double *bmin, const double *bmax, uint32_t m, double *out) {
  const double e = 1.0 / (2.0 * m);
  for (int d = 0; d < 3; d++) {
    double a = bmin[d], b = bmax[d];
    if (b - a < 5.0e-3) {
      b += 5.0e-3;
      a -= 5.0e-3;
    }
    const double c = (b + a) * 0.5, h = (b - a) * 0.5;
    for (uint32_t i = 0; i < m; i++) out[d * m + i] = c + h * cos(M_PI * (2.0 * i * e + e));
  }
}

static void devtree_free(DevCTree &t, cudaStream_t st) {
  dfree(t.d_off, st); dfree(t.d_size, st); dfree(t.d_father, st); dfree(t.d_son0, st); dfree(t.d_son1, st);
  dfree(t.d_idx, st); dfree(t.d_leaves, st); dfree(t.d_nonroot, st); dfree(t.d_voff, st);
  dfree(t.d_pts, st); dfree(t.d_V, st); dfree(t.d_E, st); dfree(t.d_refs, st);
  dfree(t.d_tr_off, st); dfree(t.d_tr_len, st);
  dfree(t.d_W, st); dfree(t.d_woff, st); dfree(t.d_fitems, st); dfree(t.d_wleaves, st);
  dfree(t.d_ppairs, st); dfree(t.d_pfirst, st); dfree(t.d_P, st);
  dfree(t.d_seg, st);
  dfree(t.d_gbox, st); dfree(t.d_glev, st); dfree(t.d_gflat, st);
}

// Flattened bases: W_t for the clusters of admissible blocks (`adm`, ids of this tree) and all
// their descendants.  W_t is formed from the leaves below t directly: the rows of leaf l inside
// W_t are W_l times the product of the transfers on the path from l up to t, and that product is
// the tensor product of three m x m products of one-dimensional transfers.  One flatten item per
// (leaf, needed ancestor) pair and slice of at most H2B_FLAT_ROWS of the leaf's rows; the items
// write disjoint rows, so one launch covers every level.  W is allocated with H2B_MV_SLACK bytes
// at its end.
static int devtree_flat_setup(DevCTree &t, const h2b_ctree &c, const std::vector<uint32_t> &adm,
                              uint32_t m, uint32_t k, cudaStream_t st) {
  std::vector<char> in_adm(c.n, 0), need(c.n, 0);
  for (uint32_t a : adm) in_adm[a] = 1;
  // pre-order: a father precedes its sons
  for (uint32_t i = 0; i < c.n; i++)
    need[i] = in_adm[i] || (c.father[i] != UINT32_MAX && need[c.father[i]]);
  std::vector<uint64_t> woff(c.n, 0);
  uint64_t tot = 0;
  for (uint32_t i = 0; i < c.n; i++)
    if (need[i]) {
      woff[i] = tot;
      tot += (uint64_t) c.size[i] * k;
    }
  t.wtotal = tot;
  std::vector<uint32_t> wleaves, pairs, pfirst, fitems;
  for (uint32_t i = 0; i < c.n; i++)
    if (need[i] && c.sons[i] == 0) wleaves.push_back(i);
  for (uint32_t l : wleaves) {
    pfirst.push_back((uint32_t) (pairs.size() / 2));
    for (uint32_t f = c.father[l]; f != UINT32_MAX && need[f]; f = c.father[f]) {
      const uint32_t pid = (uint32_t) (pairs.size() / 2);
      pairs.insert(pairs.end(), {l, f});
      for (uint32_t r0 = 0; r0 < c.size[l]; r0 += H2B_FLAT_ROWS)
        fitems.insert(fitems.end(),
                      {pid, r0, std::min<uint32_t>(H2B_FLAT_ROWS, c.size[l] - r0), 0u});
    }
  }
  pfirst.push_back((uint32_t) (pairs.size() / 2));
  t.nwleaves = (uint32_t) wleaves.size();
  t.npairs = (uint32_t) (pairs.size() / 2);
  t.nfitems = (uint32_t) (fitems.size() / 4);
  t.h_woff = woff;
  t.h_adm = in_adm;
  int rc;
  if ((rc = upload(&t.d_woff, woff, st)) || (rc = upload(&t.d_wleaves, wleaves, st)) ||
      (rc = upload(&t.d_fitems, fitems, st)) || (rc = upload(&t.d_ppairs, pairs, st)) ||
      (rc = upload(&t.d_pfirst, pfirst, st)))
    return rc;
  H2B_CUDA_TRY(cudaMallocAsync(&t.d_W, sizeof(double) * std::max<uint64_t>(tot, 1) + H2B_MV_SLACK,
                               st));
  H2B_CUDA_TRY(cudaMallocAsync(
      &t.d_P, sizeof(double) * std::max<uint64_t>((uint64_t) t.npairs * 3 * m * m, 1), st));
  return H2B_OK;
}

// W^T from V: the leaves first, then the paths' transfer products, then the rows of every
// needed ancestor in one launch.  `transposed`: the basis stores V^T (column side); otherwise V
// (row side).
static int devtree_flatten(DevCTree &t, uint32_t m, uint32_t k, int transposed, cudaStream_t st) {
  FlatLeafArgs la{t.d_wleaves, t.d_size, t.d_voff, t.d_woff, t.d_V, t.d_W, t.nwleaves, (int) k,
                  !transposed};
  int rc = h2b_flat_leaves(&la, st);
  FlatArgs fa{t.d_fitems, t.d_ppairs, t.d_pfirst, t.d_wleaves, t.d_off, t.d_size, t.d_woff,
              t.d_pts, t.d_P, t.d_W, t.nfitems, t.nwleaves, (int) m, (int) k};
  if (rc == H2B_OK) rc = h2b_flat_paths(&fa, st);
  if (rc == H2B_OK) rc = h2b_flat_rows(&fa, st);
  return rc;
}

static int devtree_build(DevCTree &t, const h2b_ctree &c, int basis, uint32_t m, uint32_t k,
                         h2b_adjacency *adj, cudaStream_t st) {
  t.n = c.n;
  t.nidx = c.nidx;
  t.depth = c.depth;
  std::vector<uint32_t> leaves, nonroot, seg(c.n, 0);
  t.roots.clear();
  t.h_idx = c.idx;
  t.h_off = c.off;
  t.h_size = c.size;
  std::vector<uint64_t> voff(c.n, 0);
  std::vector<double> pts((size_t) c.n * 3 * m);
  uint64_t vtot = 0;
  t.max_rows = 0;
  for (uint32_t i = 0; i < c.n; i++) {
    if (c.sons[i] == 0) {
      leaves.push_back(i);
      voff[i] = vtot;
      vtot += (uint64_t) c.size[i] * k;
      t.max_rows = std::max(t.max_rows, c.size[i]);
    }
    if (c.father[i] != UINT32_MAX) nonroot.push_back(i);  // every root of a forest excluded
    else t.roots.push_back(i);
    seg[i] = (uint32_t) t.roots.size() - 1;  // pre-order: a surface's clusters follow its root
    box_points(c.bmin + 3 * (size_t) i, c.bmax + 3 * (size_t) i, m, pts.data() + (size_t) i * 3 * m);
  }
  t.vtotal = vtot;
  t.h_seg = seg;
  t.nnonroot = (uint32_t) nonroot.size();
  t.nleaves = (uint32_t) leaves.size();
  t.leaves = leaves;
  // triangle lists of the leaves (basis assembly)
  h2b_nearplan tmp;
  h2b_nearplan_init(&tmp);
  std::vector<uint32_t> tr_off(leaves.size()), tr_len(leaves.size());
  for (size_t i = 0; i < leaves.size(); i++) {
    const uint32_t cl = leaves[i];
    if (h2b_nearplan_add_reflist(&tmp, adj, basis == H2B_BASIS_LINEAR, c.idx + c.off[cl],
                                 c.size[cl], &tr_off[i], &tr_len[i]) != H2B_OK) {
      h2b_nearplan_free(&tmp);
      h2b_set_error("h2matrix: out of host memory");
      return H2B_ERR_NOMEM;
    }
  }
  std::vector<TriRef> refs(tmp.nrefs);
  memcpy(refs.data(), tmp.refs, sizeof(TriRef) * tmp.nrefs);
  h2b_nearplan_free(&tmp);

  std::vector<uint32_t> off(c.off, c.off + c.n), size(c.size, c.size + c.n),
      father(c.father, c.father + c.n), son0(c.son0, c.son0 + c.n), son1(c.son1, c.son1 + c.n),
      idx(c.idx, c.idx + c.nidx);
  int rc;
  if ((rc = upload(&t.d_off, off, st)) || (rc = upload(&t.d_size, size, st)) ||
      (rc = upload(&t.d_father, father, st)) || (rc = upload(&t.d_son0, son0, st)) ||
      (rc = upload(&t.d_son1, son1, st)) || (rc = upload(&t.d_idx, idx, st)) ||
      (rc = upload(&t.d_leaves, leaves, st)) || (rc = upload(&t.d_nonroot, nonroot, st)) ||
      (rc = upload(&t.d_voff, voff, st)) ||
      (rc = upload(&t.d_pts, pts, st)) || (rc = upload(&t.d_refs, refs, st)) ||
      (rc = upload(&t.d_tr_off, tr_off, st)) || (rc = upload(&t.d_tr_len, tr_len, st)) ||
      (rc = upload(&t.d_seg, seg, st)))
    return rc;
  H2B_CUDA_TRY(cudaMallocAsync(&t.d_V, sizeof(double) * std::max<uint64_t>(vtot, 1), st));
  H2B_CUDA_TRY(cudaMallocAsync(&t.d_E, sizeof(double) * std::max<uint64_t>((uint64_t) (c.n - 1) * k * k, 1), st));
  return H2B_OK;
}

// ------------------------------------------------------------------------------------------
// construction
// ------------------------------------------------------------------------------------------

extern "C" void h2b_h2matrix_del(h2b_h2matrix *h) {
  if (!h) return;
  cudaStream_t st = h->st;
  if (st) cudaStreamSynchronize(st);
  if (h->cst) cudaStreamSynchronize(h->cst);  // pending asynchronous exports read the blocks
  if (h->shared && h->owner) h->owner->sharers.n--;
  // the operator's own data
  for (DevCTree *t : {&h->rt, &h->ct}) {
    dfree(t->d_V, st); dfree(t->d_E, st); dfree(t->d_W, st); dfree(t->d_P, st);
    dfree(t->f_W, st); dfree(t->d_grank, st); dfree(t->d_gpiv, st); dfree(t->d_gE, st);
  }
  dfree(h->f_N, st); dfree(h->f_S, st); dfree(h->d_S, st); dfree(h->d_N, st);
  dfree(h->d_xp, st); dfree(h->d_yp, st); dfree(h->d_xt, st); dfree(h->d_yt, st);
  dfree(h->d_xio, st); dfree(h->d_yio, st); dfree(h->d_mverr, st);
  // the structure, unless it belongs to the matrix this one was made like
  if (!h->shared) {
    dfree(h->d_items, st);
    dfree(h->d_items_single, st);
    devtree_free(h->rt, st);
    devtree_free(h->ct, st);
    dfree(h->d_adm_rc, st); dfree(h->d_adm_cc, st);
    dfree(h->d_near_rc, st); dfree(h->d_near_cc, st); dfree(h->d_near_off, st);
    dfree(h->d_tiles, st); dfree(h->d_refs, st); dfree(h->d_sing, st);
    dfree(h->d_xs, st); dfree(h->d_ys, st); dfree(h->d_ws, st); dfree(h->d_wsl, st);
  }
  for (int e = 0; e < 12; e++)
    if (h->ev[e]) cudaEventDestroy(h->ev[e]);
  if (h->cst) {
    cudaStreamSynchronize(h->cst);
    cudaStreamDestroy(h->cst);
  }
  if (h->ev_copy) cudaEventDestroy(h->ev_copy);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

// Singular pairs of the uploaded tiles (found on the device) and the pair counts per case.
static int classify_singular(h2b_h2matrix *h, uint64_t all_pairs) {
  uint32_t cnt[4] = {0, 0, 0, 0};
  const int rc = h2b_classify_device(h->bem->s, h->d_refs, h->d_tiles, h->ntiles, h->st,
                                     &h->d_sing, cnt);
  if (rc != H2B_OK) return rc;
  const uint64_t nsing = (uint64_t) cnt[1] + cnt[2] + cnt[3];
  h->nsing = (uint32_t) nsing;
  for (int c = 1; c <= 3; c++) h->pairs[c] = cnt[c];
  h->pairs[0] = all_pairs - nsing;
  return H2B_OK;
}

// The structure of an H2 matrix of rank k (every cluster basis padded to k columns); m is the
// interpolation order of the Chebyshev path (1 for the greenhybrid bases, which use no nodes).
static h2b_h2matrix *h2matrix_create(const h2b_bem *bem, const h2b_tree *tree, uint32_t m,
                                     uint32_t k) {
  const uint32_t nr = h2b_bem_rows(bem), nc = h2b_bem_cols(bem);
  if (tree->row.nidx != nr || tree->col.nidx != nc) {
    h2b_set_error("h2b_h2matrix_new: tree index sets (%u, %u) do not match the operator (%u, %u)",
                  tree->row.nidx, tree->col.nidx, nr, nc);
    return NULL;
  }
  if (h2b_ensure_device() != H2B_OK) return NULL;
  h2b_h2matrix *h = new h2b_h2matrix();
  h->bem = bem;
  h->tree = tree;
  h->m = m;
  h->k = k;
  h->cx = bem->pde == H2B_HELMHOLTZ;
  h->num_sms = bem->s->num_sms;
  int rc = H2B_OK;
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
    h2b_set_error("h2b_h2matrix_new: %s", cudaGetErrorString(cudaGetLastError()));
    delete h;
    return NULL;
  }
  h2b_adjacency *adj = const_cast<h2b_adjacency *>(&bem->s->adj);
  rc = devtree_build(h->rt, tree->row, bem->row_basis, m, h->k, adj, h->st);
  if (rc == H2B_OK) rc = devtree_build(h->ct, tree->col, bem->col_basis, m, h->k, adj, h->st);

  // blocks
  std::vector<uint32_t> arc, acc, nrc, ncc;
  std::vector<uint64_t> noff;
  uint64_t ntot = 0;
  h2b_nearplan plan;
  h2b_nearplan_init(&plan);
  plan.skip_sing = 1;  // singular pairs are found on the device below
  for (uint32_t b = 0; rc == H2B_OK && b < tree->blocks.n; b++) {
    const uint32_t r = tree->blocks.rc[b], c = tree->blocks.cc[b];
    if (tree->blocks.adm[b]) {
      arc.push_back(r);
      acc.push_back(c);
    } else {
      nrc.push_back(r);
      ncc.push_back(c);
      noff.push_back(ntot);
      const uint32_t rows = tree->row.size[r], cols = tree->col.size[c];
      rc = h2b_nearplan_add_block(&plan, adj, bem->row_basis, bem->col_basis,
                                  tree->row.idx + tree->row.off[r], rows,
                                  tree->col.idx + tree->col.off[c], cols, ntot, rows, 0, 64);
      ntot += (uint64_t) rows * cols;
    }
  }
  uint64_t all_pairs = 0;
  if (rc == H2B_OK)
    for (uint32_t t = 0; t < plan.ntiles; t++)
      all_pairs += (uint64_t) plan.tiles[t].tr_len * plan.tiles[t].sc_len;
  for (int e = 0; rc == H2B_OK && e < 12; e++)
    if (cudaEventCreate(&h->ev[e]) != cudaSuccess) {
      h2b_set_error("h2b_h2matrix_new: %s", cudaGetErrorString(cudaGetLastError()));
      rc = H2B_ERR_CUDA;
    }
  h->nadm = (uint32_t) arc.size();
  h->nnear = (uint32_t) nrc.size();
  h->near_total = ntot;
  h->ntiles = plan.ntiles;
  if (rc == H2B_OK) {
    const size_t W = h->cx ? 2 : 1;
    std::vector<h2b_tile> tiles(plan.tiles, plan.tiles + plan.ntiles);
    std::vector<h2b_triref> refs(plan.refs, plan.refs + plan.nrefs);
    if ((rc = upload(&h->d_adm_rc, arc, h->st)) || (rc = upload(&h->d_adm_cc, acc, h->st)) ||
        (rc = upload(&h->d_near_rc, nrc, h->st)) || (rc = upload(&h->d_near_cc, ncc, h->st)) ||
        (rc = upload(&h->d_near_off, noff, h->st)) || (rc = upload(&h->d_tiles, tiles, h->st)) ||
        (rc = upload(&h->d_refs, refs, h->st)) ||
        (rc = classify_singular(h, all_pairs))) {
    } else if (cudaMallocAsync(&h->d_S, sizeof(double) * W * std::max<uint64_t>((uint64_t) h->nadm * h->k * h->k, 1) + H2B_MV_SLACK, h->st) != cudaSuccess ||
               cudaMallocAsync(&h->d_N, sizeof(double) * W * std::max<uint64_t>(ntot, 1) + H2B_MV_SLACK, h->st) != cudaSuccess ||
               cudaMallocAsync(&h->d_mverr, sizeof(int), h->st) != cudaSuccess ||
               cudaMemsetAsync(h->d_mverr, 0, sizeof(int), h->st) != cudaSuccess ||
               cudaMallocAsync(&h->d_xp, sizeof(double) * W * nc + H2B_MV_SLACK, h->st) != cudaSuccess ||
               cudaMallocAsync(&h->d_yp, sizeof(double) * W * nr, h->st) != cudaSuccess ||
               cudaMallocAsync(&h->d_xt, sizeof(double) * W * h->k * tree->col.n + H2B_MV_SLACK, h->st) != cudaSuccess ||
               cudaMallocAsync(&h->d_yt, sizeof(double) * W * h->k * tree->row.n + H2B_MV_SLACK, h->st) != cudaSuccess ||
               cudaMallocAsync(&h->d_xio, sizeof(double) * W * nc, h->st) != cudaSuccess ||
               cudaMallocAsync(&h->d_yio, sizeof(double) * W * nr, h->st) != cudaSuccess) {
      h2b_set_error("h2b_h2matrix_new: device allocation failed: %s",
                    cudaGetErrorString(cudaGetLastError()));
      rc = H2B_ERR_NOMEM;
    }
  }
  h2b_nearplan_free(&plan);
  // flattened bases over the admissible clusters, and the matvec work items
  if (rc == H2B_OK) rc = devtree_flat_setup(h->rt, tree->row, arc, m, h->k, h->st);
  if (rc == H2B_OK) rc = devtree_flat_setup(h->ct, tree->col, acc, m, h->k, h->st);
  if (rc == H2B_OK) {
    h->h_arc = arc;
    h->h_acc = acc;
    h->h_nrc = nrc;
    h->h_ncc = ncc;
    h->h_noff = noff;
    h2b_tune_lookup(h);
    rc = h2b_h2_build_mv_items(h);
  }
  // single-triangle rule (raw and linear-basis weighted)
  if (rc == H2B_OK) {
    const h2b_quad &qd = bem->quad;
    std::vector<double> xs(qd.xs, qd.xs + qd.ns), ys(qd.ys, qd.ys + qd.ns),
        ws(qd.ws + 3 * qd.ns, qd.ws + 4 * qd.ns), wsl(qd.ws, qd.ws + 3 * qd.ns);
    h->ns = qd.ns;
    if ((rc = upload(&h->d_xs, xs, h->st)) || (rc = upload(&h->d_ys, ys, h->st)) ||
        (rc = upload(&h->d_ws, ws, h->st)) || (rc = upload(&h->d_wsl, wsl, h->st))) {
    }
  }
  if (rc == H2B_OK && cudaStreamSynchronize(h->st) != cudaSuccess) {
    h2b_set_error("h2b_h2matrix_new: %s", cudaGetErrorString(cudaGetLastError()));
    rc = H2B_ERR_CUDA;
  }
  if (rc != H2B_OK) {
    h2b_h2matrix_del(h);
    return NULL;
  }
  h2b_h2_fill_mvm_plan(h);
  return h;
}

extern "C" h2b_h2matrix *h2b_h2matrix_new(const h2b_bem *bem, const h2b_tree *tree, uint32_t m) {
  if (!bem || !tree) {
    h2b_set_error("h2b_h2matrix_new: NULL operator or tree");
    return NULL;
  }
  if (m < 1 || m > 5) {
    h2b_set_error("h2b_h2matrix_new: interpolation order %u outside 1..5", m);
    return NULL;
  }
  return h2matrix_create(bem, tree, m, m * m * m);
}

// Per operator: ranks, pivots and transfers of the greenhybrid bases of one tree.
static int green_alloc(DevCTree &t, uint32_t k, cudaStream_t st) {
  H2B_CUDA_TRY(cudaMallocAsync(&t.d_grank, sizeof(uint32_t) * t.n, st));
  H2B_CUDA_TRY(cudaMallocAsync(&t.d_gpiv, sizeof(uint32_t) * (size_t) t.n * k, st));
  H2B_CUDA_TRY(cudaMallocAsync(&t.d_gE, sizeof(double) * (size_t) t.n * k * k, st));
  return H2B_OK;
}

// Structure of the greenhybrid bases of one tree: boxes, clusters by level (deepest first) with
// the rows bound of A_t (a leaf's size; a father's size, at most the 2k pivot rows of its two
// sons), and by level the flatten items of the needed non-leaf clusters (father, son, first
// row, rows: slices of at most H2B_GREEN_FLAT_ROWS rows of each son).
static int green_setup(DevCTree &t, const h2b_ctree &c, uint32_t k, cudaStream_t st) {
  uint32_t maxlev = 0;
  for (uint32_t i = 0; i < c.n; i++) maxlev = std::max(maxlev, c.level[i]);
  std::vector<char> need(c.n, 0);
  for (uint32_t i = 0; i < c.n; i++)
    need[i] = t.h_adm[i] || (c.father[i] != UINT32_MAX && need[c.father[i]]);
  std::vector<uint32_t> lev, flat;
  std::vector<double> box((size_t) c.n * 6);
  t.h_glev_off.assign(1, 0);
  t.h_gflat_off.assign(1, 0);
  t.h_glev_rows.clear();
  for (uint32_t L = maxlev + 1; L-- > 0;) {
    uint32_t rows = 1;
    for (uint32_t i = 0; i < c.n; i++) {
      if (c.level[i] != L) continue;
      lev.push_back(i);
      rows = std::max(rows, c.sons[i] == 0 ? c.size[i] : std::min(c.size[i], 2 * k));
      if (c.sons[i] != 0 && need[i])
        for (uint32_t so : {c.son0[i], c.son1[i]}) {
          if (so == UINT32_MAX) continue;
          for (uint32_t r0 = 0; r0 < c.size[so]; r0 += H2B_GREEN_FLAT_ROWS)
            flat.insert(flat.end(),
                        {i, so, r0, std::min<uint32_t>(H2B_GREEN_FLAT_ROWS, c.size[so] - r0)});
        }
    }
    t.h_glev_off.push_back((uint32_t) lev.size());
    t.h_gflat_off.push_back((uint32_t) (flat.size() / 4));
    t.h_glev_rows.push_back(rows);
  }
  for (uint32_t i = 0; i < c.n; i++)
    for (int d = 0; d < 3; d++) {
      box[6 * (size_t) i + d] = c.bmin[3 * (size_t) i + d];
      box[6 * (size_t) i + 3 + d] = c.bmax[3 * (size_t) i + d];
    }
  int rc;
  if ((rc = upload(&t.d_gbox, box, st)) || (rc = upload(&t.d_glev, lev, st)) ||
      (rc = upload(&t.d_gflat, flat, st)))
    return rc;
  return green_alloc(t, k, st);
}

extern "C" h2b_h2matrix *h2b_h2matrix_new_greenhybrid(const h2b_bem *bem, const h2b_tree *tree,
                                                      uint32_t m, uint32_t l, double delta,
                                                      double accur) {
  if (!bem || !tree) {
    h2b_set_error("h2b_h2matrix_new_greenhybrid: NULL operator or tree");
    return NULL;
  }
  if (bem->pde != H2B_LAPLACE || (bem->layer != H2B_SLP && bem->layer != H2B_DLP)) {
    h2b_set_error("h2b_h2matrix_new_greenhybrid: built for the Laplace single and double layer");
    return NULL;
  }
  if (m < 1 || l < 1 || m * l > H2B_GREEN_MLMAX || !(accur > 0.0) || !(delta >= 0.0)) {
    h2b_set_error("h2b_h2matrix_new_greenhybrid: m %u, l %u (m l at most %d), delta %g, "
                  "accuracy %g", m, l, H2B_GREEN_MLMAX, delta, accur);
    return NULL;
  }
  // the one-dimensional rule: m Gauss points on each of l equal parts of [-1, 1]
  // (setup_green_bem3d, Library/bem3d.c:4999)
  double g01[H2B_GREEN_MLMAX], w01[H2B_GREEN_MLMAX], ht[H2B_GREEN_MLMAX], hw[H2B_GREEN_MLMAX];
  if (m == 1) {
    ht[0] = 0.0;
    hw[0] = 2.0;
  } else {
    if (h2b_gauss_legendre01(m, g01, w01) != H2B_OK) return NULL;
    for (uint32_t i = 0; i < m; i++) {
      ht[i] = 2.0 * g01[i] - 1.0;
      hw[i] = 2.0 * w01[i];
    }
  }
  const uint32_t ml = m * l, k = 12 * ml * ml;
  h2b_h2matrix *h = h2matrix_create(bem, tree, 1, k);
  if (!h) return NULL;
  h->green = 1;
  h->g_ml = (int) ml;
  h->g_delta = delta;
  h->g_accur = accur;
  const double cw = 2.0 / (double) l;
  for (uint32_t j = 1; j <= l; j++) {
    const double s0 = -1.0 + cw * (j - 1), s1 = -1.0 + cw * j, hh = 0.5 * (s1 - s0);
    for (uint32_t i = 0; i < m; i++) {
      h->g_tg[i + (j - 1) * m] = hh * ht[i] + 0.5 * (s1 + s0);
      h->g_wg[i + (j - 1) * m] = hh * hw[i];
    }
  }
  int rc = green_setup(h->rt, tree->row, k, h->st);
  if (rc == H2B_OK) rc = green_setup(h->ct, tree->col, k, h->st);
  {
    const h2b_ctree &r = tree->row, &c = tree->col;
    h->g_same = bem->row_basis == bem->col_basis && r.n == c.n && r.nidx == c.nidx &&
                !memcmp(r.off, c.off, sizeof(uint32_t) * r.n) &&
                !memcmp(r.size, c.size, sizeof(uint32_t) * r.n) &&
                !memcmp(r.sons, c.sons, sizeof(uint32_t) * r.n) &&
                !memcmp(r.idx, c.idx, sizeof(uint32_t) * r.nidx) &&
                !memcmp(r.bmin, c.bmin, sizeof(double) * 3 * r.n) &&
                !memcmp(r.bmax, c.bmax, sizeof(double) * 3 * r.n);
  }
  if (rc == H2B_OK && cudaStreamSynchronize(h->st) != cudaSuccess) {
    h2b_set_error("h2b_h2matrix_new_greenhybrid: %s", cudaGetErrorString(cudaGetLastError()));
    rc = H2B_ERR_CUDA;
  }
  if (rc != H2B_OK) {
    h2b_h2matrix_del(h);
    return NULL;
  }
  return h;
}

extern "C" h2b_h2matrix *h2b_h2matrix_new_like(const h2b_bem *bem, const h2b_h2matrix *like) {
  if (!bem || !like) {
    h2b_set_error("h2b_h2matrix_new_like: NULL operator or matrix");
    return NULL;
  }
  const h2b_bem *b0 = like->bem;
  if (bem->s != b0->s || bem->row_basis != b0->row_basis || bem->col_basis != b0->col_basis ||
      bem->q != b0->q || bem->pde != b0->pde) {
    h2b_set_error("h2b_h2matrix_new_like: the operator must share the surface, bases, quadrature "
                  "order and PDE of the model matrix");
    return NULL;
  }
  if (h2b_ensure_device() != H2B_OK) return NULL;
  // copy every field, then replace what belongs to the new operator
  h2b_h2matrix *h = new h2b_h2matrix(*like);
  h->bem = bem;
  h->shared = 1;
  // the structure's owner: the model matrix itself, or the matrix it shares with
  h->owner = like->shared ? like->owner : like;
  h->owner->sharers.n++;
  h->st = nullptr;
  h->cst = nullptr;
  h->ev_copy = nullptr;
  for (int e = 0; e < 12; e++) h->ev[e] = nullptr;
  for (int i = 0; i < 6; i++) h->ms[i] = 0.0f;
  h->quad_fp32 = 0;
  h->g_row_ready = 0;
  h->g_col_copied = 0;
  h->f_S = h->f_N = nullptr;
  h->d_S = h->d_N = h->d_xp = h->d_yp = h->d_xt = h->d_yt = h->d_xio = h->d_yio = nullptr;
  h->d_mverr = nullptr;
  for (DevCTree *t : {&h->rt, &h->ct}) {
    t->d_V = t->d_E = t->d_W = t->d_P = t->d_gE = nullptr;
    t->f_W = nullptr;
    t->d_grank = t->d_gpiv = nullptr;
  }
  int rc = H2B_OK;
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) rc = H2B_ERR_CUDA;
  for (int e = 0; rc == H2B_OK && e < 12; e++)
    if (cudaEventCreate(&h->ev[e]) != cudaSuccess) rc = H2B_ERR_CUDA;
  const size_t W = h->cx ? 2 : 1;
  const uint64_t kk = (uint64_t) h->k * h->k;
  const uint32_t nr = h->rt.nidx, nc = h->ct.nidx;
  for (DevCTree *t : {&h->rt, &h->ct}) {
    if (rc != H2B_OK) break;
    if (cudaMallocAsync(&t->d_V, sizeof(double) * std::max<uint64_t>(t->vtotal, 1), h->st) ||
        cudaMallocAsync(&t->d_E, sizeof(double) * std::max<uint64_t>((uint64_t) (t->n - 1) * kk, 1),
                        h->st) ||
        cudaMallocAsync(&t->d_W, sizeof(double) * std::max<uint64_t>(t->wtotal, 1) + H2B_MV_SLACK,
                        h->st) ||
        cudaMallocAsync(&t->d_P,
                        sizeof(double) * std::max<uint64_t>((uint64_t) t->npairs * 3 * h->m * h->m, 1),
                        h->st))
      rc = H2B_ERR_NOMEM;
  }
  for (DevCTree *t : {&h->rt, &h->ct})
    if (rc == H2B_OK && h->green) rc = green_alloc(*t, h->k, h->st);
  if (rc == H2B_OK &&
      (cudaMallocAsync(&h->d_S, sizeof(double) * W * std::max<uint64_t>(h->nadm * kk, 1) + H2B_MV_SLACK, h->st) ||
       cudaMallocAsync(&h->d_N, sizeof(double) * W * std::max<uint64_t>(h->near_total, 1) + H2B_MV_SLACK, h->st) ||
       cudaMallocAsync(&h->d_mverr, sizeof(int), h->st) ||
       cudaMemsetAsync(h->d_mverr, 0, sizeof(int), h->st) ||
       cudaMallocAsync(&h->d_xp, sizeof(double) * W * nc + H2B_MV_SLACK, h->st) ||
       cudaMallocAsync(&h->d_yp, sizeof(double) * W * nr, h->st) ||
       cudaMallocAsync(&h->d_xt, sizeof(double) * W * h->k * h->ct.n + H2B_MV_SLACK, h->st) ||
       cudaMallocAsync(&h->d_yt, sizeof(double) * W * h->k * h->rt.n + H2B_MV_SLACK, h->st) ||
       cudaMallocAsync(&h->d_xio, sizeof(double) * W * nc, h->st) ||
       cudaMallocAsync(&h->d_yio, sizeof(double) * W * nr, h->st)))
    rc = H2B_ERR_NOMEM;
  if (rc == H2B_OK && cudaStreamSynchronize(h->st) != cudaSuccess) rc = H2B_ERR_CUDA;
  if (rc != H2B_OK) {
    h2b_set_error("h2b_h2matrix_new_like: %s", cudaGetErrorString(cudaGetLastError()));
    h2b_h2matrix_del(h);
    return NULL;
  }
  h2b_h2_fill_mvm_plan(h);
  return h;
}

int h2b_h2_check_mv_error(const h2b_h2matrix *h) {
  int flag = 0;
  H2B_CUDA_TRY(cudaMemcpyAsync(&flag, h->d_mverr, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  H2B_CUDA_TRY(cudaStreamSynchronize(h->st));
  if (flag) {
    cudaMemsetAsync(h->d_mverr, 0, sizeof(int), h->st);
    h2b_set_error("matvec: a panel copy to shared memory did not complete (bounded wait)");
    return H2B_ERR_TIMEOUT;
  }
  return H2B_OK;
}

// The item list of a product for panels of pb bytes at FP64 storage, ordered by kind: forward,
// nearfield, coupling, backward (the matvec runs the first two kinds in one launch, then the
// coupling, then the backward slices).
static void build_items(const h2b_h2matrix *h, uint32_t pb, uint32_t fwd_rows, uint32_t back_rows,
                        std::vector<MvItem> &it, MvItems &m) {
  const h2b_ctree &R = h->tree->row, &C = h->tree->col;
  const uint32_t k = h->k, W = h->cx ? 2 : 1;
  uint32_t start[4] = {0, 0, 0, 0};
  it.clear();
  auto slice_rows = [&](uint32_t want) {
    const uint32_t cap = std::max<uint32_t>(1, pb / (8u * k));
    return std::max<uint32_t>(1, std::min(want, cap));
  };
  // columns per panel of a block with `rows` rows and complex entries when W = 2
  auto panel_cols = [&](uint32_t rows) {
    return std::max<uint32_t>(1, pb / (8u * W * std::max<uint32_t>(rows, 1)));
  };
  const uint32_t fr = slice_rows(fwd_rows), br = slice_rows(back_rows);
  // forward slices, x_t -> xt_t, over every admissible column cluster
  for (uint32_t t = 0; t < C.n; t++) {
    if (!h->ct.h_adm[t]) continue;
    for (uint32_t r0 = 0; r0 < C.size[t]; r0 += fr)
      it.push_back(MvItem{h->ct.h_woff[t] + (uint64_t) r0 * k, k, std::min(fr, C.size[t] - r0),
                          C.off[t] + r0, k * t, h->ct.h_seg[t], H2B_MV_FORWARD});
  }
  // nearfield blocks, in column panels
  start[H2B_MV_NEAR] = (uint32_t) it.size();
  for (size_t b = 0; b < h->h_nrc.size(); b++) {
    const uint32_t r = h->h_nrc[b], c = h->h_ncc[b], rows = R.size[r], cols = C.size[c];
    const uint32_t pc = panel_cols(rows);
    for (uint32_t c0 = 0; c0 < cols; c0 += pc)
      it.push_back(MvItem{h->h_noff[b] + (uint64_t) c0 * rows, rows, std::min(pc, cols - c0),
                          C.off[c] + c0, R.off[r], h->rt.h_seg[r], H2B_MV_NEAR});
  }
  // coupling blocks, in column panels
  start[H2B_MV_COUPLING] = (uint32_t) it.size();
  for (size_t b = 0; b < h->h_arc.size(); b++) {
    const uint32_t r = h->h_arc[b], c = h->h_acc[b], pc = panel_cols(k);
    for (uint32_t c0 = 0; c0 < k; c0 += pc)
      it.push_back(MvItem{(uint64_t) b * k * k + (uint64_t) c0 * k, k, std::min(pc, k - c0),
                          k * c + c0, k * r, h->rt.h_seg[r], H2B_MV_COUPLING});
  }
  // backward slices, yt_t -> y_t (W_t^T transposed), over every admissible row cluster
  start[H2B_MV_BACKWARD] = (uint32_t) it.size();
  for (uint32_t t = 0; t < R.n; t++) {
    if (!h->rt.h_adm[t]) continue;
    for (uint32_t r0 = 0; r0 < R.size[t]; r0 += br)
      it.push_back(MvItem{h->rt.h_woff[t] + (uint64_t) r0 * k, k, std::min(br, R.size[t] - r0),
                          k * t, R.off[t] + r0, h->rt.h_seg[t], H2B_MV_BACKWARD | H2B_MV_TRANS});
  }
  m.n = (uint32_t) it.size();
  for (int q = 0; q < 4; q++) m.start[q] = start[q];
  m.max_bytes = m.max_rows = m.max_cols_t = m.max_x = 0;
  for (const MvItem &e : it) {
    const uint32_t kind = e.flags & H2B_MV_KIND;
    const bool cpx = kind == H2B_MV_NEAR || kind == H2B_MV_COUPLING;
    m.max_bytes = std::max<uint32_t>(m.max_bytes, e.rows * e.cols * 8u * (cpx ? W : 1u));
    if (!(e.flags & H2B_MV_TRANS)) m.max_rows = std::max(m.max_rows, e.rows);
    else m.max_cols_t = std::max(m.max_cols_t, e.cols);
    m.max_x = std::max(m.max_x, (e.flags & H2B_MV_TRANS) ? e.rows : e.cols);
  }
}

// Two lists: one for the FP64 product, and one for the product from the FP32 copies with twice
// the entries per panel (the same bytes per copy).
int h2b_h2_build_mv_items(h2b_h2matrix *h) {
  std::vector<MvItem> it, its;
  build_items(h, h->mv_panel_bytes, h->mv_fwd_rows, h->mv_back_rows, it, h->mvitems);
  build_items(h, 2 * h->mv_panel_bytes, 2 * h->mv_fwd_rows, 2 * h->mv_back_rows, its,
              h->mvitems_single);
  dfree(h->d_items, h->st);
  dfree(h->d_items_single, h->st);
  int rc;
  if ((rc = upload(&h->d_items, it, h->st)) || (rc = upload(&h->d_items_single, its, h->st)))
    return rc;
  h->mvitems.items = h->d_items;
  h->mvitems_single.items = h->d_items_single;
  return H2B_OK;
}

void h2b_h2_fill_mvm_plan(h2b_h2matrix *h) {
  MvmPlan &p = h->mvm;
  memset(&p, 0, sizeof(p));
  p.cx = h->cx;
  p.num_sms = h->num_sms;
  p.k = (int) h->k;
  p.nrow = h->rt.nidx;
  p.ncol = h->ct.nidx;
  p.nrow_clusters = h->rt.n;
  p.ncol_clusters = h->ct.n;
  p.ridx = h->rt.d_idx;
  p.cidx = h->ct.d_idx;
  p.xp = h->d_xp;
  p.yp = h->d_yp;
  p.xt = h->d_xt;
  p.yt = h->d_yt;
  p.items = h->mvitems;
  p.items_single = h->mvitems_single;
  p.Wc = h->ct.d_W;
  p.Wr = h->rt.d_W;
  p.N = h->d_N;
  p.S = h->d_S;
  p.fWc = h->ct.f_W;
  p.fWr = h->rt.f_W;
  p.fN = h->f_N;
  p.fS = h->f_S;
  p.err = h->d_mverr;
  p.ctas_per_sm = h->mv_ctas;
  p.warps = h->mv_warps;
  p.stages = h->mv_stages;
  h2b_mvm_prepare();
}

// ------------------------------------------------------------------------------------------
// assembly
// ------------------------------------------------------------------------------------------

// The column basis is stored transposed (V^T, E^T), the layout the forward transform reads.
static int assemble_basis(h2b_h2matrix *h, DevCTree &t, int basis, int dn) {
  const int transposed = (&t == &h->ct);
  FarLeafArgs la;
  la.transposed = transposed;
  la.tri = h->bem->s->d_tri;
  la.refs = t.d_refs;
  la.leaves = t.d_leaves;
  la.tr_off = t.d_tr_off;
  la.tr_len = t.d_tr_len;
  la.size = t.d_size;
  la.voff = t.d_voff;
  la.pts = t.d_pts;
  la.xs = h->d_xs;
  la.ys = h->d_ys;
  la.ws = h->d_ws;
  la.wsl = h->d_wsl;
  la.V = t.d_V;
  la.nleaves = t.nleaves;
  la.max_rows = t.max_rows;
  la.m = (int) h->m;
  la.k = (int) h->k;
  la.ns = (int) h->ns;
  la.split = std::max(1, std::min((int) h->k, h->leaf_split));
  int rc = h2b_far_leaf_basis(&la, basis == H2B_BASIS_LINEAR, dn, h->st);
  if (rc != H2B_OK) return rc;
  FarTransferArgs ta{t.d_nonroot, t.d_father, t.d_pts, t.d_E, t.nnonroot, (int) h->m, (int) h->k,
                     transposed};
  rc = h2b_far_transfer(&ta, h->st);
  if (rc == H2B_OK) rc = devtree_flatten(t, h->m, h->k, transposed, h->st);
  return rc;
}

// Greenhybrid bases of one tree: ranks, pivots and transfers level by level (deepest first),
// then the flattened bases (the leaves' copies, then the fathers' rows level by level).
static int green_basis(h2b_h2matrix *h, DevCTree &t, int basis, int dcol) {
  const int transposed = (&t == &h->ct);
  const uint32_t K = h->k;
  H2B_CUDA_TRY(cudaMemsetAsync(t.d_gE, 0, sizeof(double) * (size_t) t.n * K * K, h->st));
  GreenArgs g;
  memset(&g, 0, sizeof(g));
  g.tri = h->bem->s->d_tri;
  g.vt_off = h->bem->s->d_vt_off;
  g.vt_tri = h->bem->s->d_vt_tri;
  g.xs = h->d_xs;
  g.ys = h->d_ys;
  g.ws = h->d_ws;
  g.wsl = h->d_wsl;
  g.ns = (int) h->ns;
  g.linear = basis == H2B_BASIS_LINEAR;
  g.dcol = dcol;
  g.transposed = transposed;
  g.kconst = h->bem->kconst;
  g.off = t.d_off;
  g.size = t.d_size;
  g.son0 = t.d_son0;
  g.son1 = t.d_son1;
  g.idx = t.d_idx;
  g.box = t.d_gbox;
  g.voff = t.d_voff;
  memcpy(g.tg, h->g_tg, sizeof(g.tg));
  memcpy(g.wg, h->g_wg, sizeof(g.wg));
  g.ml = h->g_ml;
  g.K = (int) K;
  g.delta = h->g_delta;
  g.accur = h->g_accur;
  g.rank = t.d_grank;
  g.piv = t.d_gpiv;
  g.V = t.d_V;
  g.E = t.d_gE;
  int rc = H2B_OK;
  for (size_t L = 0; rc == H2B_OK && L + 1 < t.h_glev_off.size(); L++) {
    g.clusters = t.d_glev + t.h_glev_off[L];
    g.n = t.h_glev_off[L + 1] - t.h_glev_off[L];
    g.max_rows = t.h_glev_rows[L];
    rc = h2b_green_basis(&g, h->st);
  }
  if (rc != H2B_OK) return rc;
  FlatLeafArgs la{t.d_wleaves, t.d_size, t.d_voff, t.d_woff, t.d_V, t.d_W, t.nwleaves, (int) K,
                  !transposed};
  rc = h2b_flat_leaves(&la, h->st);
  GreenFlatArgs fa{nullptr, 0, t.d_off, t.d_size, t.d_son0, t.d_son1, t.d_grank, t.d_woff,
                   t.d_gE, t.d_W, (int) K};
  for (size_t L = 0; rc == H2B_OK && L + 1 < t.h_gflat_off.size(); L++) {
    fa.items = t.d_gflat + 4 * (size_t) t.h_gflat_off[L];
    fa.n = t.h_gflat_off[L + 1] - t.h_gflat_off[L];
    rc = h2b_green_flatten(&fa, h->st);
  }
  return rc;
}

// Phase timings: events 2i / 2i+1 bracket phase i (0 row basis, 1 column basis, 2 coupling,
// 3 nearfield; event 7 separates the distant and singular nearfield kernels; 9/10 the matvec).
static void mark(h2b_h2matrix *h, int e) { cudaEventRecord(h->ev[e], h->st); }

// Free the FP32 copies (they no longer match the matrix once any part is reassembled).
static void drop_single(h2b_h2matrix *h) {
  if (!h->f_N && !h->f_S && !h->rt.f_W && !h->ct.f_W) return;
  cudaStream_t st = h->st;
  dfree(h->f_N, st);
  dfree(h->f_S, st);
  dfree(h->rt.f_W, st);
  dfree(h->ct.f_W, st);
  h2b_h2_fill_mvm_plan(h);
}

extern "C" int h2b_h2matrix_set_precision(h2b_h2matrix *h, int precision) {
  if (!h || (precision != H2B_FP64 && precision != H2B_FP32)) {
    h2b_set_error("h2b_h2matrix_set_precision: precision must be H2B_FP64 or H2B_FP32");
    return H2B_ERR_ARG;
  }
  if (precision == H2B_FP32 && h->bem->q != 2) {
    h2b_set_error("h2b_h2matrix_set_precision: FP32 quadrature needs the regular order q = 2");
    return H2B_ERR_ARG;
  }
  h->quad_fp32 = precision == H2B_FP32;
  return H2B_OK;
}

extern "C" int h2b_h2matrix_set_matvec_shape(h2b_h2matrix *h, const uint32_t shape[H2B_SHAPE_N]) {
  if (!h || !shape) return H2B_ERR_ARG;
  const uint32_t fr = shape[0] ? shape[0] : h->mv_fwd_rows;
  const uint32_t br = shape[1] ? shape[1] : h->mv_back_rows;
  const uint32_t pb = shape[4] ? shape[4] * 1024u : h->mv_panel_bytes;
  if (shape[2] > 8 || shape[3] > 4 || (shape[4] && (shape[4] < 4 || shape[4] > 64)) ||
      shape[5] > h->k || shape[6] > 8) {
    h2b_set_error("h2b_h2matrix_set_matvec_shape: CTAs per SM <= 8, stages per warp <= 4, panels "
                  "4..64 KiB, leaf CTAs <= k, consumer warps <= 8");
    return H2B_ERR_ARG;
  }
  if (fr != h->mv_fwd_rows || br != h->mv_back_rows || pb != h->mv_panel_bytes) {
    if (h->shared || h->sharers.n > 0) {
      h2b_set_error("h2b_h2matrix_set_matvec_shape: slice and panel sizes belong to a structure "
                    "that other matrices share");
      return H2B_ERR_STATE;
    }
    H2B_CUDA_TRY(cudaStreamSynchronize(h->st));  // no product reads the old items
    h->mv_fwd_rows = fr;
    h->mv_back_rows = br;
    h->mv_panel_bytes = pb;
    int rc = h2b_h2_build_mv_items(h);
    if (rc != H2B_OK) return rc;
    H2B_CUDA_TRY(cudaStreamSynchronize(h->st));
  }
  if (shape[2]) h->mv_ctas = (int) shape[2];
  if (shape[3]) h->mv_stages = (int) shape[3];
  if (shape[5]) h->leaf_split = (int) shape[5];
  if (shape[6]) h->mv_warps = (int) shape[6];
  h2b_h2_fill_mvm_plan(h);
  return H2B_OK;
}

extern "C" int h2b_h2matrix_get_matvec_shape(const h2b_h2matrix *h, uint32_t shape[H2B_SHAPE_N]) {
  if (!h || !shape) return H2B_ERR_ARG;
  shape[0] = h->mv_fwd_rows;
  shape[1] = h->mv_back_rows;
  shape[2] = (uint32_t) h->mv_ctas;
  shape[3] = (uint32_t) h->mv_stages;
  shape[4] = h->mv_panel_bytes / 1024u;
  shape[5] = (uint32_t) h->leaf_split;
  shape[6] = (uint32_t) h->mv_warps;
  return H2B_OK;
}

extern "C" int h2b_h2matrix_make_single(h2b_h2matrix *h) {
  if (!h) return H2B_ERR_ARG;
  drop_single(h);
  const uint64_t W = h->cx ? 2 : 1;
  const uint64_t nN = W * h->near_total, nS = W * (uint64_t) h->nadm * h->k * h->k;
  const size_t sl = H2B_MV_SLACK;
  if (cudaMallocAsync(&h->f_N, sizeof(float) * std::max<uint64_t>(nN, 1) + sl, h->st) != cudaSuccess ||
      cudaMallocAsync(&h->f_S, sizeof(float) * std::max<uint64_t>(nS, 1) + sl, h->st) != cudaSuccess ||
      cudaMallocAsync(&h->rt.f_W, sizeof(float) * std::max<uint64_t>(h->rt.wtotal, 1) + sl, h->st) != cudaSuccess ||
      cudaMallocAsync(&h->ct.f_W, sizeof(float) * std::max<uint64_t>(h->ct.wtotal, 1) + sl, h->st) != cudaSuccess) {
    cudaGetLastError();
    drop_single(h);
    h2b_set_error("h2b_h2matrix_make_single: device allocation failed");
    return H2B_ERR_NOMEM;
  }
  int rc = h2b_to_single(h->d_N, h->f_N, nN, h->num_sms, h->st);
  if (rc == H2B_OK) rc = h2b_to_single(h->d_S, h->f_S, nS, h->num_sms, h->st);
  if (rc == H2B_OK) rc = h2b_to_single(h->rt.d_W, h->rt.f_W, h->rt.wtotal, h->num_sms, h->st);
  if (rc == H2B_OK) rc = h2b_to_single(h->ct.d_W, h->ct.f_W, h->ct.wtotal, h->num_sms, h->st);
  if (rc == H2B_OK && cudaStreamSynchronize(h->st) != cudaSuccess) {
    h2b_set_error("h2b_h2matrix_make_single: %s", cudaGetErrorString(cudaGetLastError()));
    rc = H2B_ERR_CUDA;
  }
  if (rc != H2B_OK) {
    drop_single(h);
    return rc;
  }
  h2b_h2_fill_mvm_plan(h);
  return H2B_OK;
}

static int finish(h2b_h2matrix *h, int rc, unsigned phases) {
  drop_single(h);
  if (rc != H2B_OK) return rc;
  if (cudaStreamSynchronize(h->st) != cudaSuccess) {
    h2b_set_error("h2matrix: %s", cudaGetErrorString(cudaGetLastError()));
    return H2B_ERR_CUDA;
  }
  float t;
  if ((phases & 1) && cudaEventElapsedTime(&t, h->ev[0], h->ev[1]) == cudaSuccess) h->ms[0] = t;
  if ((phases & 2) && cudaEventElapsedTime(&t, h->ev[2], h->ev[3]) == cudaSuccess) h->ms[1] = t;
  if ((phases & 4) && cudaEventElapsedTime(&t, h->ev[4], h->ev[5]) == cudaSuccess) h->ms[2] = t;
  if (phases & 8) {
    if (cudaEventElapsedTime(&t, h->ev[6], h->ev[7]) == cudaSuccess) h->ms[3] = t;
    if (cudaEventElapsedTime(&t, h->ev[7], h->ev[8]) == cudaSuccess) h->ms[4] = t;
  }
  cudaGetLastError();
  return H2B_OK;
}

// The single layer's column kernels are its row kernels (kernel_col = fundamental_row,
// dnz_kernel_col = dnz_fundamental_row, Library/laplacebem3d.c:870/897): on equal trees the
// column basis is the row basis, and its ranks, pivots, transfers and flattened bases are copied.
static int green_copy_col(h2b_h2matrix *h) {
  const uint32_t K = h->k;
  DevCTree &r = h->rt, &c = h->ct;
  H2B_CUDA_TRY(cudaMemcpyAsync(c.d_grank, r.d_grank, sizeof(uint32_t) * r.n,
                               cudaMemcpyDeviceToDevice, h->st));
  H2B_CUDA_TRY(cudaMemcpyAsync(c.d_gpiv, r.d_gpiv, sizeof(uint32_t) * (size_t) r.n * K,
                               cudaMemcpyDeviceToDevice, h->st));
  H2B_CUDA_TRY(cudaMemcpyAsync(c.d_gE, r.d_gE, sizeof(double) * (size_t) r.n * K * K,
                               cudaMemcpyDeviceToDevice, h->st));
  H2B_CUDA_TRY(cudaMemcpyAsync(c.d_W, r.d_W, sizeof(double) * r.wtotal, cudaMemcpyDeviceToDevice,
                               h->st));
  return H2B_OK;
}

static int row_basis(h2b_h2matrix *h) {
  mark(h, 0);
  // row side: Lagrange polynomials (assemble_bem3d_lagrange_{c,l}_amatrix); normal derivatives
  // for the adjoint double layer (assemble_bem3d_dn_lagrange_*, Library/laplacebem3d.c:1180)
  int rc = h->green ? green_basis(h, h->rt, h->bem->row_basis, 0)
                    : assemble_basis(h, h->rt, h->bem->row_basis, h->bem->layer == H2B_ADLP);
  h->g_row_ready = h->green && rc == H2B_OK;
  mark(h, 1);
  return rc;
}

static int col_basis(h2b_h2matrix *h) {
  mark(h, 2);
  // column side of the double layer: normal derivatives (assemble_bem3d_dn_lagrange_*)
  int rc;
  if (h->green && h->g_same && h->g_row_ready && h->bem->layer == H2B_SLP &&
      h->rt.h_woff == h->ct.h_woff) {
    rc = green_copy_col(h);
    h->g_col_copied = 1;
  } else {
    rc = h->green ? green_basis(h, h->ct, h->bem->col_basis, h->bem->layer == H2B_DLP)
                  : assemble_basis(h, h->ct, h->bem->col_basis, h->bem->layer == H2B_DLP);
    h->g_col_copied = 0;
  }
  mark(h, 3);
  return rc;
}

static int coupling(h2b_h2matrix *h) {
  mark(h, 4);
  if (h->green) {
    GreenCouplingArgs ga{h->bem->s->d_tri, h->bem->s->d_vt_off, h->bem->s->d_vt_tri,
                         h->d_adm_rc, h->d_adm_cc, h->rt.d_grank, h->rt.d_gpiv, h->ct.d_grank,
                         h->ct.d_gpiv, h->d_S, h->nadm, (int) h->k, (int) h->bem->q,
                         h->bem->row_basis == H2B_BASIS_LINEAR,
                         h->bem->col_basis == H2B_BASIS_LINEAR, h->bem->layer == H2B_DLP,
                         h->bem->kconst, 0};
    uint32_t deg = 1;
    if (h->bem->col_basis == H2B_BASIS_LINEAR) {
      const h2b_adjacency &adj = h->bem->s->adj;
      for (uint32_t v = 0; v < adj.nv; v++) deg = std::max(deg, adj.off[v + 1] - adj.off[v]);
    }
    ga.max_elems = h->k * deg;
    const int rc = h2b_green_coupling(&ga, h->st);
    mark(h, 5);
    return rc;
  }
  FarCouplingArgs ca{h->d_adm_rc, h->d_adm_cc, h->rt.d_pts, h->ct.d_pts, h->d_S, h->nadm,
                     (int) h->m, (int) h->k, h->bem->kconst, h->bem->k_re, -h->bem->k_im};
  int rc = h2b_far_coupling(&ca, h->cx, h->st);
  mark(h, 5);
  return rc;
}

static int launch_near(h2b_h2matrix *h, h2b_h2matrix *h2) {
  h2b_near_launch L;
  h2b_fill_launch(h->bem, &L);
  L.refs = h->d_refs;
  L.tiles = h->d_tiles;
  L.ntiles = h->ntiles;
  L.sing = h->d_sing;
  L.nsing = h->nsing;
  L.nvert = h->pairs[1];
  L.out0 = h->d_N;
  L.ev_between = h->ev[7];
  L.fp32 = h->quad_fp32;
  if (h2) {
    L.kk = h->bem->pde == H2B_LAPLACE ? H2B_KK_LBOTH : H2B_KK_HBOTH;
    L.out1 = h2->d_N;
    L.alpha_re = h2->bem->alpha_re;
    L.alpha_im = h2->bem->alpha_im;
  }
  mark(h, 6);
  int rc = h2b_near_launch_kernels(&L, h->st);
  mark(h, 8);
  if (rc == H2B_OK) rc = h2b_check_err_flag(h->bem, h->st);
  return rc;
}

extern "C" int h2b_h2matrix_assemble_row_clusterbasis(h2b_h2matrix *h) {
  if (!h) return H2B_ERR_ARG;
  return finish(h, row_basis(h), 1);
}

extern "C" int h2b_h2matrix_assemble_col_clusterbasis(h2b_h2matrix *h) {
  if (!h) return H2B_ERR_ARG;
  return finish(h, col_basis(h), 2);
}

extern "C" int h2b_h2matrix_assemble_farfield(h2b_h2matrix *h) {
  if (!h) return H2B_ERR_ARG;
  return finish(h, coupling(h), 4);
}

extern "C" int h2b_h2matrix_assemble_nearfield(h2b_h2matrix *h) {
  if (!h) return H2B_ERR_ARG;
  return finish(h, launch_near(h, nullptr), 8);
}

extern "C" int h2b_h2matrix_assemble_nearfield_pair(h2b_h2matrix *a, h2b_h2matrix *b) {
  if (!a || !b) return H2B_ERR_ARG;
  const h2b_bem *A = a->bem, *B = b->bem;
  if (a->tree != b->tree || A->s != B->s || A->pde != B->pde || A->k_re != B->k_re ||
      A->k_im != B->k_im || A->layer != H2B_SLP || B->layer != H2B_DLP ||
      A->row_basis != B->row_basis || A->col_basis != B->col_basis || A->q != B->q ||
      A->q2 != B->q2) {
    h2b_set_error("h2b_h2matrix_assemble_nearfield_pair: needs a single and a double layer of "
                  "the same PDE and wavenumber on the same tree, surface, bases and quadrature "
                  "orders");
    return H2B_ERR_ARG;
  }
  // b's storage must be idle before a's stream writes it
  H2B_CUDA_TRY(cudaEventRecord(b->ev[11], b->st));
  H2B_CUDA_TRY(cudaStreamWaitEvent(a->st, b->ev[11], 0));
  int rc = finish(a, launch_near(a, b), 8);
  if (rc == H2B_OK) {
    b->ms[3] = b->ms[4] = 0.0f;  // the pass is accounted to a
  }
  return rc;
}

extern "C" int h2b_h2matrix_assemble(h2b_h2matrix *h) {
  if (!h) return H2B_ERR_ARG;
  int rc = coupling(h);
  if (rc == H2B_OK) rc = launch_near(h, nullptr);
  return finish(h, rc, 4 | 8);
}

extern "C" int h2b_h2matrix_assemble_all(h2b_h2matrix *h) {
  if (!h) return H2B_ERR_ARG;
  int rc = row_basis(h);
  if (rc == H2B_OK) rc = col_basis(h);
  if (rc == H2B_OK) rc = coupling(h);
  if (rc == H2B_OK) rc = launch_near(h, nullptr);
  return finish(h, rc, 1 | 2 | 4 | 8);
}

extern "C" int h2b_h2matrix_green_ranks(const h2b_h2matrix *h, int side, uint32_t *ranks) {
  if (!h || !ranks || (side != 0 && side != 1)) {
    h2b_set_error("h2b_h2matrix_green_ranks: NULL matrix or output, or side not 0 / 1");
    return H2B_ERR_ARG;
  }
  if (!h->green) {
    h2b_set_error("h2b_h2matrix_green_ranks: not a greenhybrid H2 matrix");
    return H2B_ERR_ARG;
  }
  const DevCTree &t = side ? h->ct : h->rt;
  H2B_CUDA_TRY(cudaMemcpyAsync(ranks, t.d_grank, sizeof(uint32_t) * t.n, cudaMemcpyDeviceToHost,
                               h->st));
  H2B_CUDA_TRY(cudaStreamSynchronize(h->st));
  return H2B_OK;
}

extern "C" int h2b_h2matrix_export_green(const h2b_h2matrix *h, int part, double *out,
                                         uint64_t *ndoubles) {
  if (!h || !ndoubles || part < 0 || part > 4) {
    h2b_set_error("h2b_h2matrix_export_green: NULL matrix or count, or part outside 0..4");
    return H2B_ERR_ARG;
  }
  if (!h->green) {
    h2b_set_error("h2b_h2matrix_export_green: not a greenhybrid H2 matrix");
    return H2B_ERR_ARG;
  }
  const uint32_t K = h->k;
  std::vector<uint32_t> rr(h->rt.n), rcr(h->ct.n);
  H2B_CUDA_TRY(cudaMemcpyAsync(rr.data(), h->rt.d_grank, sizeof(uint32_t) * h->rt.n,
                               cudaMemcpyDeviceToHost, h->st));
  H2B_CUDA_TRY(cudaMemcpyAsync(rcr.data(), h->ct.d_grank, sizeof(uint32_t) * h->ct.n,
                               cudaMemcpyDeviceToHost, h->st));
  H2B_CUDA_TRY(cudaStreamSynchronize(h->st));
  uint64_t n = 0;
  if (part == 4) {
    for (uint32_t b = 0; b < h->nadm; b++) n += (uint64_t) rr[h->h_arc[b]] * rcr[h->h_acc[b]];
  } else {
    const int col = part >= 2;
    const h2b_ctree &c = col ? h->tree->col : h->tree->row;
    const std::vector<uint32_t> &rk = col ? rcr : rr;
    for (uint32_t i = 0; i < c.n; i++) {
      if (part % 2 == 0 && c.sons[i] == 0) n += (uint64_t) c.size[i] * rk[i];
      if (part % 2 == 1 && c.father[i] != UINT32_MAX) n += (uint64_t) rk[i] * rk[c.father[i]];
    }
  }
  *ndoubles = n;
  if (!out) return H2B_OK;
  uint64_t o = 0;
  if (part == 4) {
    std::vector<double> S((size_t) h->nadm * K * K);
    H2B_CUDA_TRY(cudaMemcpy(S.data(), h->d_S, sizeof(double) * S.size(), cudaMemcpyDeviceToHost));
    for (uint32_t b = 0; b < h->nadm; b++) {
      const uint32_t kr = rr[h->h_arc[b]], kc = rcr[h->h_acc[b]];
      for (uint32_t j = 0; j < kc; j++)
        for (uint32_t i = 0; i < kr; i++) out[o++] = S[(size_t) b * K * K + i + (size_t) j * K];
    }
    return H2B_OK;
  }
  const int col = part >= 2;
  const h2b_ctree &c = col ? h->tree->col : h->tree->row;
  const std::vector<uint32_t> &rk = col ? rcr : rr;
  const DevCTree &t = col ? h->ct : h->rt;
  if (part % 2 == 1) {
    std::vector<double> E((size_t) c.n * K * K);
    H2B_CUDA_TRY(cudaMemcpy(E.data(), t.d_gE, sizeof(double) * E.size(), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < c.n; i++) {
      if (c.father[i] == UINT32_MAX) continue;
      const uint32_t ks = rk[i], kf = rk[c.father[i]];
      for (uint32_t j = 0; j < kf; j++)
        for (uint32_t r = 0; r < ks; r++) out[o++] = E[(size_t) i * K * K + r + (size_t) j * K];
    }
    return H2B_OK;
  }
  // leaf bases: the row side stores V (size x K, column-major), the column side V^T; a copied
  // column basis has only the row side's
  const int from_row = col && h->g_col_copied;
  const DevCTree &tv = from_row ? h->rt : t;
  std::vector<double> V(tv.vtotal);
  H2B_CUDA_TRY(cudaMemcpy(V.data(), tv.d_V, sizeof(double) * V.size(), cudaMemcpyDeviceToHost));
  uint64_t voff = 0;
  for (uint32_t i = 0; i < c.n; i++) {
    if (c.sons[i] != 0) continue;
    const uint32_t sz = c.size[i], k = rk[i];
    const double *v = V.data() + voff;
    for (uint32_t j = 0; j < k; j++)
      for (uint32_t r = 0; r < sz; r++)
        out[o++] = (col && !from_row) ? v[j + (size_t) r * K] : v[r + (size_t) j * sz];
    voff += (uint64_t) sz * K;
  }
  return H2B_OK;
}

extern "C" int h2b_h2matrix_timings(const h2b_h2matrix *h, double ms[6]) {
  if (!h || !ms) return H2B_ERR_ARG;
  for (int i = 0; i < 6; i++) ms[i] = h->ms[i];
  return H2B_OK;
}

extern "C" int h2b_h2matrix_pair_counts(const h2b_h2matrix *h, uint64_t counts[4]) {
  if (!h || !counts) return H2B_ERR_ARG;
  for (int i = 0; i < 4; i++) counts[i] = h->pairs[i];
  return H2B_OK;
}

extern "C" int h2b_h2matrix_unique_pairs(const h2b_h2matrix *h, uint64_t counts[4]) {
  if (!h || !counts) return H2B_ERR_ARG;
  return h2b_near_unique_pairs(h->bem->s->d_tri, h->d_refs, h->d_tiles, h->ntiles, h->bem->s->nt,
                               counts, h->st);
}

// ------------------------------------------------------------------------------------------
// inspection
// ------------------------------------------------------------------------------------------

extern "C" int h2b_h2matrix_info(const h2b_h2matrix *h, uint64_t info[8]) {
  if (!h || !info) return H2B_ERR_ARG;
  const uint64_t W = h->cx ? 2 : 1;
  info[0] = h->near_total;
  info[1] = (uint64_t) h->nadm * h->k * h->k;
  info[2] = h->rt.vtotal + h->ct.vtotal;
  info[3] = (uint64_t) (h->rt.n - 1 + h->ct.n - 1) * h->k * h->k;
  info[4] = 8 * (W * (info[0] + info[1]) + info[2] + info[3]);
  info[5] = h->nadm;
  info[6] = h->nnear;
  info[7] = h->k;
  return H2B_OK;
}

extern "C" int h2b_h2matrix_export(const h2b_h2matrix *h, int part, uint32_t count, double *out,
                                   uint64_t *ndoubles) {
  if (!h || !ndoubles) return H2B_ERR_ARG;
  if (h->green && part >= 0 && part <= 3) {
    h2b_set_error("h2b_h2matrix_export: the bases of a greenhybrid H2 matrix have per-cluster "
                  "ranks; only parts 4 and 5 are exported");
    return H2B_ERR_ARG;
  }
  const uint64_t W = h->cx ? 2 : 1, kk = (uint64_t) h->k * h->k;
  const double *src = nullptr;
  uint64_t n = 0;
  switch (part) {
    case 0:
    case 2: {
      const DevCTree &t = part == 0 ? h->rt : h->ct;
      const h2b_ctree &c = part == 0 ? h->tree->row : h->tree->col;
      uint32_t got = 0;
      for (uint32_t i = 0; i < c.n && got < count; i++)
        if (c.sons[i] == 0) {
          n += (uint64_t) c.size[i] * h->k;
          got++;
        }
      src = t.d_V;
      break;
    }
    case 1:
    case 3: {
      const DevCTree &t = part == 1 ? h->rt : h->ct;
      n = (uint64_t) std::min<uint32_t>(count, t.n - 1) * kk;
      src = t.d_E;
      break;
    }
    case 4:
      n = (uint64_t) std::min<uint32_t>(count, h->nadm) * kk * W;
      src = h->d_S;
      break;
    case 5: {
      const uint32_t nb = std::min<uint32_t>(count, h->nnear);
      uint64_t e = 0;
      for (uint32_t b = 0, j = 0; b < h->tree->blocks.n && j < nb; b++)
        if (!h->tree->blocks.adm[b]) {
          e += (uint64_t) h->tree->row.size[h->tree->blocks.rc[b]] *
               h->tree->col.size[h->tree->blocks.cc[b]];
          j++;
        }
      n = e * W;
      src = h->d_N;
      break;
    }
    default:
      h2b_set_error("h2b_h2matrix_export: part %d outside 0..5", part);
      return H2B_ERR_ARG;
  }
  *ndoubles = n;
  if (out && n) {
    H2B_CUDA_TRY(cudaMemcpyAsync(out, src, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
    H2B_CUDA_TRY(cudaStreamSynchronize(h->st));
    if (part == 2 || part == 3) {
      // the column basis is stored transposed on the device: return H2Lib's layout
      const h2b_ctree &c = h->tree->col;
      std::vector<double> tmp;
      uint64_t pos = 0;
      uint32_t got = 0;
      for (uint32_t i = (part == 2 ? 0 : 1); i < c.n && got < count && pos < n; i++) {
        if (part == 2 && c.sons[i] != 0) continue;
        const uint64_t rows = part == 2 ? c.size[i] : h->k, k = h->k;
        tmp.assign(out + pos, out + pos + rows * k);
        for (uint64_t r = 0; r < rows; r++)
          for (uint64_t nu = 0; nu < k; nu++) out[pos + r + nu * rows] = tmp[nu + r * k];
        pos += rows * k;
        got++;
      }
    }
  }
  return H2B_OK;
}

extern "C" int h2b_h2matrix_export_async(h2b_h2matrix *h, int part, uint32_t count,
                                         double *out) {
  if (!h || !out || part == 2 || part == 3 || part < 0 || part > 5) {
    h2b_set_error("h2b_h2matrix_export_async: parts 0, 1, 4, 5 into a non-NULL buffer");
    return H2B_ERR_ARG;
  }
  uint64_t n = 0;
  int rc = h2b_h2matrix_export(h, part, count, nullptr, &n);
  if (rc != H2B_OK || n == 0) return rc;
  const double *src = part == 0 ? h->rt.d_V : part == 1 ? h->rt.d_E : part == 4 ? h->d_S : h->d_N;
  if (!h->cst) H2B_CUDA_TRY(cudaStreamCreateWithFlags(&h->cst, cudaStreamNonBlocking));
  if (!h->ev_copy) H2B_CUDA_TRY(cudaEventCreateWithFlags(&h->ev_copy, cudaEventDisableTiming));
  // after everything already queued on the matrix's stream, on the copy stream
  H2B_CUDA_TRY(cudaEventRecord(h->ev_copy, h->st));
  H2B_CUDA_TRY(cudaStreamWaitEvent(h->cst, h->ev_copy, 0));
  H2B_CUDA_TRY(cudaMemcpyAsync(out, src, sizeof(double) * n, cudaMemcpyDeviceToHost, h->cst));
  return H2B_OK;
}

extern "C" int h2b_h2matrix_export_wait(h2b_h2matrix *h) {
  if (!h) return H2B_ERR_ARG;
  if (h->cst) H2B_CUDA_TRY(cudaStreamSynchronize(h->cst));
  return H2B_OK;
}

// ------------------------------------------------------------------------------------------
// matvec
// ------------------------------------------------------------------------------------------

int h2b_h2_addeval_dev(const h2b_h2matrix *h, double ar, double ai, const double *dx, double *dy,
                       cudaStream_t st) {
  return h2b_mvm_launch(&h->mvm, dx, dy, ar, ai, st);
}

extern "C" int h2b_h2matrix_addeval_multi(double alpha_re, double alpha_im,
                                          const h2b_h2matrix *h, uint32_t nrhs, const double *X,
                                          uint64_t ldx, double *Y, uint64_t ldy) {
  if (!h || !X || !Y) {
    h2b_set_error("h2b_h2matrix_addeval_multi: NULL argument");
    return H2B_ERR_ARG;
  }
  if (ldx < h->ct.nidx || ldy < h->rt.nidx) {
    h2b_set_error("h2b_h2matrix_addeval_multi: leading dimensions too small");
    return H2B_ERR_ARG;
  }
  const size_t W = h->cx ? 2 : 1;
  for (uint32_t r = 0; r < nrhs; r++) {
    int rc = h2b_h2matrix_addeval(alpha_re, alpha_im, h, X + W * ldx * r, Y + W * ldy * r);
    if (rc != H2B_OK) return rc;
  }
  return H2B_OK;
}

static int addeval_prec(double alpha_re, double alpha_im, const h2b_h2matrix *h, const double *x,
                        double *y, int single);

extern "C" int h2b_h2matrix_addeval(double alpha_re, double alpha_im, const h2b_h2matrix *h,
                                    const double *x, double *y) {
  return addeval_prec(alpha_re, alpha_im, h, x, y, 0);
}

extern "C" int h2b_h2matrix_addeval_single(double alpha_re, double alpha_im,
                                           const h2b_h2matrix *h, const double *x, double *y) {
  return addeval_prec(alpha_re, alpha_im, h, x, y, 1);
}

static int addeval_prec(double alpha_re, double alpha_im, const h2b_h2matrix *h, const double *x,
                        double *y, int single) {
  if (!h || !x || !y) {
    h2b_set_error("h2b_h2matrix_addeval: NULL argument");
    return H2B_ERR_ARG;
  }
  const size_t W = h->cx ? 2 : 1;
  const bool dx = h2b_is_device_ptr(x), dy = h2b_is_device_ptr(y);
  const double *xd = x;
  double *yd = y;
  if (!dx) {
    H2B_CUDA_TRY(cudaMemcpyAsync(h->d_xio, x, sizeof(double) * W * h->ct.nidx,
                                 cudaMemcpyHostToDevice, h->st));
    xd = h->d_xio;
  }
  if (!dy) {
    H2B_CUDA_TRY(cudaMemcpyAsync(h->d_yio, y, sizeof(double) * W * h->rt.nidx,
                                 cudaMemcpyHostToDevice, h->st));
    yd = h->d_yio;
  }
  cudaEventRecord(h->ev[9], h->st);
  int rc = single ? h2b_mvm_launch_single(&h->mvm, xd, yd, alpha_re, alpha_im, h->st)
                  : h2b_h2_addeval_dev(h, alpha_re, alpha_im, xd, yd, h->st);
  cudaEventRecord(h->ev[10], h->st);
  if (rc == H2B_OK && !dy) {
    if (cudaMemcpyAsync(y, yd, sizeof(double) * W * h->rt.nidx, cudaMemcpyDeviceToHost,
                        h->st) != cudaSuccess) {
      h2b_set_error("h2b_h2matrix_addeval: %s", cudaGetErrorString(cudaGetLastError()));
      rc = H2B_ERR_CUDA;
    }
  }
  if (rc == H2B_OK && cudaStreamSynchronize(h->st) != cudaSuccess) {
    h2b_set_error("h2b_h2matrix_addeval: %s", cudaGetErrorString(cudaGetLastError()));
    rc = H2B_ERR_CUDA;
  }
  if (rc == H2B_OK) rc = h2b_h2_check_mv_error(h);
  float t;
  if (rc == H2B_OK && cudaEventElapsedTime(&t, h->ev[9], h->ev[10]) == cudaSuccess)
    const_cast<h2b_h2matrix *>(h)->ms[5] = t;
  return rc;
}
