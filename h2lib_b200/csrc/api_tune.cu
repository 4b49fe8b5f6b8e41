// Autotuner of the launch shapes of an H2 matrix (h2b_h2matrix_autotune, include/h2b200.h).
//
// The reference has no counterpart: its only scheduling knob is the OpenMP task depth
// (max_pardepth, Library/basic.c).  Here the matrix-vector product's item kernel has a launch
// shape (panel size of a work item, resident CTAs per SM, consumer warps per CTA, ring stages per
// consumer warp) and the leaf-basis kernel a split (CTAs per leaf).  The tuner times every
// candidate that fits the SM with CUDA events on the matrix's own stream and data, keeps the
// fastest, and records it in a process-wide cache keyed by the matrix's size class, so that the
// next matrix of that class starts from the tuned shape (h2b_h2matrix_new looks it up).  The
// cache can be written to and read from a text file.
//
// No matvec candidate changes the product's arithmetic per entry, only the grouping of the
// atomic additions into the outputs, so every shape gives the same product up to FP64 rounding.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "api_h2.h"
#include "device_common.cuh"
#include "h2b200_internal.h"
#include "h2mvm.h"

namespace {

// size class: operator kind, rank and the binary magnitude of the rows x columns
using TuneKey = std::tuple<int, uint32_t, int>;
struct TuneVal {
  uint32_t shape[H2B_SHAPE_N];
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;

TuneKey key_of(int cx, uint32_t k, uint64_t rows, uint64_t cols) {
  const double rc = (double) std::max<uint64_t>(rows, 1) * (double) std::max<uint64_t>(cols, 1);
  return TuneKey(cx, k, (int) floor(log2(rc)));
}

struct Events {
  cudaEvent_t a = nullptr, b = nullptr;
  Events() {
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) a = b = nullptr;
  }
  ~Events() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// Mean device ms of `reps` products (FP64 or from the FP32 copies) after one warm-up product, on
// the matrix's input/output staging vectors; a negative value on an error.
double time_products(h2b_h2matrix *h, int single, int reps, Events &ev) {
  const double *x = h->d_xio;
  double *y = h->d_yio;
  auto once = [&]() {
    return single ? h2b_mvm_launch_single(&h->mvm, x, y, 1.0, 0.0, h->st)
                  : h2b_mvm_launch(&h->mvm, x, y, 1.0, 0.0, h->st);
  };
  if (once() != H2B_OK) return -1.0;
  cudaEventRecord(ev.a, h->st);
  for (int r = 0; r < reps; r++)
    if (once() != H2B_OK) return -1.0;
  cudaEventRecord(ev.b, h->st);
  if (cudaEventSynchronize(ev.b) != cudaSuccess) return -1.0;
  if (h2b_h2_check_mv_error(h) != H2B_OK) return -1.0;
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, ev.a, ev.b) != cudaSuccess) return -1.0;
  return (double) ms / reps;
}

// Device ms of one assembly of both cluster bases at the matrix's current leaf split.
double time_bases(h2b_h2matrix *h, Events &ev) {
  cudaEventRecord(ev.a, h->st);
  if (h2b_h2matrix_assemble_row_clusterbasis(h) != H2B_OK ||
      h2b_h2matrix_assemble_col_clusterbasis(h) != H2B_OK)
    return -1.0;
  cudaEventRecord(ev.b, h->st);
  if (cudaEventSynchronize(ev.b) != cudaSuccess) return -1.0;
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, ev.a, ev.b) != cudaSuccess) return -1.0;
  return (double) ms;
}

}  // namespace

// Applies a cached shape of h's size class to a new matrix (before its items are built).
void h2b_tune_lookup(h2b_h2matrix *h) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = g_tune.find(key_of(h->cx, h->k, h->rt.nidx, h->ct.nidx));
  if (it == g_tune.end()) return;
  const uint32_t *s = it->second.shape;
  h->mv_fwd_rows = s[0];
  h->mv_back_rows = s[1];
  h->mv_ctas = (int) s[2];
  h->mv_stages = (int) s[3];
  h->mv_panel_bytes = s[4] * 1024u;
  h->leaf_split = (int) std::min<uint32_t>(s[5], h->k);
  h->mv_warps = (int) s[6];
}

extern "C" int h2b_h2matrix_autotune(h2b_h2matrix *h, uint32_t flags,
                                     uint32_t shape_out[H2B_SHAPE_N], double ms_out[4]) {
  if (!h) return H2B_ERR_ARG;
  if (flags & ~(uint32_t) (H2B_TUNE_MATVEC | H2B_TUNE_LEAF)) {
    h2b_set_error("h2b_h2matrix_autotune: unknown flags 0x%x", flags);
    return H2B_ERR_ARG;
  }
  Events ev;
  if (!ev.a) {
    h2b_set_error("h2b_h2matrix_autotune: event creation failed");
    return H2B_ERR_CUDA;
  }
  H2B_CUDA_TRY(cudaStreamSynchronize(h->st));
  double res[4] = {0.0, 0.0, 0.0, 0.0};  // matvec ms: start, tuned; bases ms: start, tuned
  int rc = H2B_OK;

  if (flags & H2B_TUNE_LEAF) {
    const bool had_single = h->f_N != nullptr;
    const int start = h->leaf_split;
    double best = time_bases(h, ev);
    if (best < 0.0) return H2B_ERR_CUDA;
    res[2] = best;
    int arg = start, last = start;
    for (int split : {1, 2, 4, 8}) {
      if (split == start || (uint32_t) split > h->k) continue;
      h->leaf_split = last = split;
      const double t = time_bases(h, ev);
      if (t < 0.0) {
        h->leaf_split = start;
        return H2B_ERR_CUDA;
      }
      if (t < best) best = t, arg = split;
    }
    h->leaf_split = arg;
    res[3] = best;
    // the splits sum a leaf's quadrature in different orders (entries agree to rounding): the
    // bases are left as the chosen split assembles them
    if (last != arg && time_bases(h, ev) < 0.0) return H2B_ERR_CUDA;
    if (had_single && (rc = h2b_h2matrix_make_single(h)) != H2B_OK) return rc;
  }

  if (flags & H2B_TUNE_MATVEC) {
    const bool single = h->f_N != nullptr;
    const uint32_t k = std::max<uint32_t>(h->k, 1);
    const uint32_t fr0 = h->mv_fwd_rows, br0 = h->mv_back_rows, pb0 = h->mv_panel_bytes;
    const int ct0 = h->mv_ctas, nw0 = h->mv_warps, sp0 = h->mv_stages;
    auto cost = [&]() {
      const double a = time_products(h, 0, 3, ev);
      if (a < 0.0) return -1.0;
      if (!single) return a;
      const double b = time_products(h, 1, 3, ev);
      return b < 0.0 ? -1.0 : a + b;
    };
    double best = cost();
    if (best < 0.0) return H2B_ERR_CUDA;
    res[0] = best;
    uint32_t bpb = pb0, bfr = fr0, bbr = br0;
    int bct = ct0, bnw = nw0, bsp = sp0;
    // slices and panels belong to the structure: fixed while it is shared
    std::vector<uint32_t> panels;
    if (h->shared || h->sharers.n > 0) panels.push_back(pb0);
    else panels = {12u * 1024u, 16u * 1024u, 24u * 1024u};
    int smem_sm = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    for (uint32_t pb : panels) {
      if (rc != H2B_OK) break;
      if (pb != h->mv_panel_bytes) {
        h->mv_panel_bytes = pb;
        // slices of W^T as wide as a panel, at least 8 columns
        h->mv_fwd_rows = h->mv_back_rows = std::max<uint32_t>(8u, pb / (8u * k));
        if ((rc = h2b_h2_build_mv_items(h)) != H2B_OK) break;
        if (cudaStreamSynchronize(h->st) != cudaSuccess) {
          rc = H2B_ERR_CUDA;
          break;
        }
      }
      for (int ct : {2, 3, 4, 5, 6, 8})
        for (int nw : {1, 2, 3, 4})
          for (int sp : {1, 2}) {
            if (rc != H2B_OK) continue;
            h->mv_ctas = ct, h->mv_warps = nw, h->mv_stages = sp;
            h2b_h2_fill_mvm_plan(h);
            // the candidate's CTAs must be resident together (1 KiB per CTA is reserved)
            size_t smem = h2b_mvm_smem_bytes(&h->mvm, 0);
            if (single) smem = std::max(smem, h2b_mvm_smem_bytes(&h->mvm, 1));
            if (smem > H2B_MAX_DYN_SMEM || (size_t) ct * (smem + 1024) > (size_t) smem_sm)
              continue;
            const double t = cost();
            if (t < 0.0) {
              rc = H2B_ERR_CUDA;
              continue;
            }
            if (t < best) {
              best = t;
              bpb = pb, bfr = h->mv_fwd_rows, bbr = h->mv_back_rows;
              bct = ct, bnw = nw, bsp = sp;
            }
          }
    }
    // leave the matrix at the best shape found (or back at its own after an error)
    if (rc != H2B_OK) bpb = pb0, bfr = fr0, bbr = br0, bct = ct0, bnw = nw0, bsp = sp0;
    h->mv_ctas = bct, h->mv_warps = bnw, h->mv_stages = bsp;
    if (h->mv_panel_bytes != bpb || h->mv_fwd_rows != bfr || h->mv_back_rows != bbr) {
      h->mv_panel_bytes = bpb, h->mv_fwd_rows = bfr, h->mv_back_rows = bbr;
      const int rc2 = h2b_h2_build_mv_items(h);
      if (rc == H2B_OK) rc = rc2;
      cudaStreamSynchronize(h->st);
    }
    h2b_h2_fill_mvm_plan(h);
    if (rc != H2B_OK) return rc;
    res[1] = best;
  }

  uint32_t shape[H2B_SHAPE_N];
  h2b_h2matrix_get_matvec_shape(h, shape);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    TuneVal v;
    memcpy(v.shape, shape, sizeof(shape));
    g_tune[key_of(h->cx, h->k, h->rt.nidx, h->ct.nidx)] = v;
  }
  if (shape_out) memcpy(shape_out, shape, sizeof(shape));
  if (ms_out) memcpy(ms_out, res, sizeof(res));
  return H2B_OK;
}

extern "C" int h2b_autotune_save(const char *path) {
  if (!path) return H2B_ERR_ARG;
  FILE *f = fopen(path, "w");
  if (!f) {
    h2b_set_error("h2b_autotune_save: cannot write %s", path);
    return H2B_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_tune_mu);
  fprintf(f, "# h2b autotune cache: complex rank size-class shape[%d]\n", H2B_SHAPE_N);
  for (const auto &e : g_tune) {
    fprintf(f, "%d %u %d", std::get<0>(e.first), std::get<1>(e.first), std::get<2>(e.first));
    for (int i = 0; i < H2B_SHAPE_N; i++) fprintf(f, " %u", e.second.shape[i]);
    fprintf(f, "\n");
  }
  const int bad = ferror(f);
  fclose(f);
  if (bad) {
    h2b_set_error("h2b_autotune_save: write error on %s", path);
    return H2B_ERR_ARG;
  }
  return H2B_OK;
}

extern "C" int h2b_autotune_load(const char *path) {
  if (!path) return H2B_ERR_ARG;
  FILE *f = fopen(path, "r");
  if (!f) {
    h2b_set_error("h2b_autotune_load: cannot read %s", path);
    return H2B_ERR_ARG;
  }
  char line[512];
  std::vector<std::pair<TuneKey, TuneVal>> got;
  int rc = H2B_OK;
  while (fgets(line, sizeof(line), f)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    int cx, cls, used = 0;
    unsigned k;
    TuneVal v;
    char *p = line;
    if (sscanf(p, "%d %u %d%n", &cx, &k, &cls, &used) != 3) {
      rc = H2B_ERR_ARG;
      break;
    }
    p += used;
    for (int i = 0; i < H2B_SHAPE_N && rc == H2B_OK; i++) {
      if (sscanf(p, "%u%n", &v.shape[i], &used) != 1) rc = H2B_ERR_ARG;
      p += used;
    }
    // the ranges h2b_h2matrix_set_matvec_shape accepts
    if (rc == H2B_OK && (v.shape[0] == 0 || v.shape[1] == 0 || v.shape[2] < 1 ||
                         v.shape[2] > 8 || v.shape[3] < 1 || v.shape[3] > 4 || v.shape[4] < 4 ||
                         v.shape[4] > 64 || v.shape[5] < 1 || v.shape[6] < 1 || v.shape[6] > 8))
      rc = H2B_ERR_ARG;
    if (rc != H2B_OK) break;
    got.emplace_back(TuneKey(cx, k, cls), v);
  }
  fclose(f);
  if (rc != H2B_OK) {
    h2b_set_error("h2b_autotune_load: malformed line in %s", path);
    return rc;
  }
  std::lock_guard<std::mutex> lock(g_tune_mu);
  for (auto &e : got) g_tune[e.first] = e.second;
  return H2B_OK;
}

extern "C" int h2b_autotune_clear(void) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune.clear();
  return H2B_OK;
}
