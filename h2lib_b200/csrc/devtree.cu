// Cluster and block trees built on the device (h2b_tree_new_device, include/h2b200.h).
//
// The trees equal the host builder's (host_tree.c) index for index, which restates
// build_bem3d_cluster (Library/bem3d.c:932: characteristic points and support boxes, :811/:850),
// build_adaptive_cluster (Library/cluster.c:80) and build_strict_block with
// admissible_max_cluster (Library/block.c:258 / :52):
//   * characteristic points (triangle centroids, or vertices) and support boxes (triangle boxes,
//     or per vertex the union of the boxes of its triangles) are formed on the device; a box is a
//     min / max, exact in any order of accumulation, so atomic updates give the same bits;
//   * the cluster tree grows level by level, one CTA per cluster of the level: the CTA reduces
//     the bounding box of its points, picks the longest side (the first of equal extents) and its
//     midpoint, and partitions its index range.  The reference partitions in place, swapping every
//     index whose point lies below the midpoint to the front in one pass; that pass fixes the
//     order of both halves, so it is replayed exactly: the CTA evaluates the comparisons in
//     parallel, then one thread runs the swaps over the range staged in shared memory.  A cluster
//     that does not split reduces its support box;
//   * the block tree grows level by level, one thread per pair of clusters evaluating the
//     max-norm admissibility with the reference's arithmetic.
// Between levels the host reads the small per-level records (split sizes, block codes) and lays
// out the next level; it numbers the clusters in pre-order and the block leaves in the block
// tree's pre-order (sons column-major) from counts, and the result fills the same host tree
// structure h2b_tree_new fills, so everything downstream is shared.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "api_internal.h"
#include "device_common.cuh"
#include "h2b200_tree.h"

extern "C" int h2b_tree_finish(h2b_tree *tr);
extern "C" int h2b_ctree_copy(h2b_ctree *dst, const h2b_ctree *src);

namespace {

constexpr int SPLIT_TPB = 256;       // a level whose clusters all fit the shared-memory stage
constexpr int SPLIT_TPB_BIG = 1024;  // a level with longer ranges (partitioned in global memory)
constexpr uint32_t LEAF = 0xFFFFFFFFu;

// Order-preserving map of finite doubles to unsigned integers (for atomic min / max).
__device__ __forceinline__ unsigned long long ord_of(double v) {
  const unsigned long long b = (unsigned long long) __double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double of_ord(unsigned long long o) {
  const unsigned long long b = (o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
  return __longlong_as_double((long long) b);
}

// Constant basis: index = triangle; point = centroid (a + b + c) / 3, support = triangle box.
__global__ void geom_const_kernel(const double *__restrict__ x, const uint32_t *__restrict__ t,
                                  uint32_t nt, double *cx, double *smin, double *smax) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
    const double *a = x + 3 * (size_t) t[3 * (size_t) i], *b = x + 3 * (size_t) t[3 * (size_t) i + 1],
                 *c = x + 3 * (size_t) t[3 * (size_t) i + 2];
    for (int d = 0; d < 3; d++) {
      cx[3 * (size_t) i + d] = (a[d] + b[d] + c[d]) / 3.0;
      smin[3 * (size_t) i + d] = fmin(a[d], fmin(b[d], c[d]));
      smax[3 * (size_t) i + d] = fmax(a[d], fmax(b[d], c[d]));
    }
  }
}

// Linear basis: index = vertex; point = vertex, support box starts as the point ...
__global__ void geom_lin_init_kernel(const double *__restrict__ x, uint32_t nv, double *cx,
                                     unsigned long long *omin, unsigned long long *omax) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * nv;
       i += gridDim.x * blockDim.x) {
    cx[i] = x[i];
    omin[i] = omax[i] = ord_of(x[i]);
  }
}

// ... and grows by the box of every triangle at the vertex.
__global__ void geom_lin_tri_kernel(const double *__restrict__ x, const uint32_t *__restrict__ t,
                                    uint32_t nt, unsigned long long *omin,
                                    unsigned long long *omax) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
    const uint32_t v[3] = {t[3 * (size_t) i], t[3 * (size_t) i + 1], t[3 * (size_t) i + 2]};
    for (int d = 0; d < 3; d++) {
      const double a = x[3 * (size_t) v[0] + d], b = x[3 * (size_t) v[1] + d],
                   c = x[3 * (size_t) v[2] + d];
      const unsigned long long lo = ord_of(fmin(a, fmin(b, c))), hi = ord_of(fmax(a, fmax(b, c)));
      for (int k = 0; k < 3; k++) {
        atomicMin(&omin[3 * (size_t) v[k] + d], lo);
        atomicMax(&omax[3 * (size_t) v[k] + d], hi);
      }
    }
  }
}

__global__ void geom_lin_fini_kernel(uint32_t n3, const unsigned long long *omin,
                                     const unsigned long long *omax, double *smin, double *smax) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    smin[i] = of_ord(omin[i]);
    smax[i] = of_ord(omax[i]);
  }
}

struct SplitArgs {
  const uint32_t *off, *size;  // the level's clusters
  uint32_t ncl, clf;
  const double *cx, *smin, *smax;
  uint32_t *idx;
  uint8_t *flag;               // ranges too long for shared memory: one byte per index,
  uint32_t *orig, *nxt;        // the original indices and the chain links
  uint32_t *size0;             // out: size of the first son, or LEAF
  double *box;                 // out: 6 per cluster, the support box of a leaf
  uint32_t cap;                // indices the shared-memory stage holds (9 bytes each)
};

// min / max of three coordinates over the CTA (every thread gets the result)
template <int TPB>
__device__ void box_reduce(double lo[3], double hi[3]) {
  __shared__ double slo[3][TPB / 32], shi[3][TPB / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int d = 0; d < 3; d++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(0xFFFFFFFFu, lo[d], o));
      hi[d] = fmax(hi[d], __shfl_xor_sync(0xFFFFFFFFu, hi[d], o));
    }
    if (lane == 0) {
      slo[d][w] = lo[d];
      shi[d][w] = hi[d];
    }
  }
  __syncthreads();
  for (int d = 0; d < 3; d++) {
    lo[d] = slo[d][0];
    hi[d] = shi[d][0];
    for (int q = 1; q < TPB / 32; q++) {
      lo[d] = fmin(lo[d], slo[d][q]);
      hi[d] = fmax(hi[d], shi[d][q]);
    }
  }
  __syncthreads();
}

// Exclusive prefix sum of one value per thread over the CTA; *total receives the sum.
template <int TPB>
__device__ uint32_t block_excl_scan(uint32_t v, uint32_t *total) {
  __shared__ uint32_t wsum[TPB / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  uint32_t before = 0, all = 0;
  for (int q = 0; q < TPB / 32; q++) {
    if (q < w) before += wsum[q];
    all += wsum[q];
  }
  if (threadIdx.x == 0) *total = all;
  __syncthreads();
  return before + incl - v;
}

template <int TPB>
__global__ void __launch_bounds__(TPB) split_kernel(SplitArgs a) {
  // stage of a range that fits: cap original indices, cap chain links, cap flag bytes
  extern __shared__ uint32_t sidx[];
  __shared__ uint32_t s0_sh;
  __shared__ int split_sh;
  const uint32_t c = blockIdx.x, off = a.off[c], size = a.size[c];
  uint32_t *idx = a.idx + off;
  if (threadIdx.x == 0) {
    s0_sh = 0;
    split_sh = 0;
  }
  __syncthreads();
  if (size > a.clf) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = threadIdx.x; i < size; i += TPB)
      for (int d = 0; d < 3; d++) {
        const double v = a.cx[3 * (size_t) idx[i] + d];
        lo[d] = fmin(lo[d], v);
        hi[d] = fmax(hi[d], v);
      }
    box_reduce<TPB>(lo, hi);
    // the longest side, the first of equal ones, and its midpoint (host_tree.c build_cluster)
    double ext = hi[0] - lo[0];
    int dir = 0;
    for (int d = 1; d < 3; d++)
      if (ext < hi[d] - lo[d]) {
        ext = hi[d] - lo[d];
        dir = d;
      }
    if (ext > 0.0) {
      const double mid = (hi[dir] + lo[dir]) / 2.0;
      // The reference's pass (for i: if point(idx[i]) < mid: swap(idx[i], idx[s]); s++) leaves
      // the m indices below the midpoint at the front in input order, and at every later position
      // p the index found by following p -> (number of "below" flags before p) while p is a
      // "below" position, up to the first position that is not: a prefix count and pointer
      // jumping give the same permutation in log2(size) parallel rounds.
      uint32_t *orig, *nxt;
      uint8_t *fl;
      if (size <= a.cap) {
        orig = sidx;
        nxt = sidx + a.cap;
        fl = reinterpret_cast<uint8_t *>(sidx + 2 * (size_t) a.cap);
      } else {
        orig = a.orig + off;
        nxt = a.nxt + off;
        fl = a.flag + off;
      }
      for (uint32_t i = threadIdx.x; i < size; i += TPB) {
        const uint32_t v = idx[i];
        orig[i] = v;
        fl[i] = a.cx[3 * (size_t) v + dir] < mid ? 1 : 0;
      }
      __syncthreads();
      // exclusive prefix count of the flags, contiguous chunks per thread
      const uint32_t chunk = (size + TPB - 1) / TPB;
      const uint32_t c0 = min(size, threadIdx.x * chunk), c1 = min(size, c0 + chunk);
      uint32_t cnt = 0;
      for (uint32_t i = c0; i < c1; i++) cnt += fl[i];
      const uint32_t base = block_excl_scan<TPB>(cnt, &s0_sh);  // s0_sh: the total
      uint32_t run = base;
      for (uint32_t i = c0; i < c1; i++) {
        nxt[i] = fl[i] ? run : i;
        run += fl[i];
      }
      __syncthreads();
      const uint32_t m = s0_sh;
      for (uint32_t i = threadIdx.x; i < size; i += TPB)
        if (fl[i]) idx[nxt[i]] = orig[i];
      uint32_t rounds = 1;
      while ((1u << rounds) < size) rounds++;
      // (four links per thread in flight; a link read while another thread replaces it is
      // still a link of the same chain, so the jumps need no ordering within a round)
      for (uint32_t r = 0; r <= rounds; r++) {
        for (uint32_t i0 = threadIdx.x; i0 < size; i0 += 4 * TPB) {
          uint32_t l[4];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const uint32_t i = i0 + k * TPB;
            l[k] = i < size ? nxt[i] : 0u;
          }
#pragma unroll
          for (int k = 0; k < 4; k++) l[k] = nxt[l[k]];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const uint32_t i = i0 + k * TPB;
            if (i < size) nxt[i] = l[k];
          }
        }
        __syncthreads();
      }
      for (uint32_t p = m + threadIdx.x; p < size; p += TPB) idx[p] = orig[nxt[p]];
      __syncthreads();
      if (threadIdx.x == 0) split_sh = s0_sh > 0 && s0_sh < size;
      __syncthreads();
    }
  }
  if (split_sh) {
    if (threadIdx.x == 0) a.size0[c] = s0_sh;
    return;
  }
  // leaf: the union of the support boxes of its indices
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = threadIdx.x; i < size; i += TPB)
    for (int d = 0; d < 3; d++) {
      lo[d] = fmin(lo[d], a.smin[3 * (size_t) idx[i] + d]);
      hi[d] = fmax(hi[d], a.smax[3 * (size_t) idx[i] + d]);
    }
  box_reduce<TPB>(lo, hi);
  if (threadIdx.x == 0) {
    a.size0[c] = LEAF;
    for (int d = 0; d < 3; d++) {
      a.box[6 * (size_t) c + d] = lo[d];
      a.box[6 * (size_t) c + 3 + d] = hi[d];
    }
  }
}

struct BlockArgs {
  const uint32_t *rc, *cc;     // the level's pairs (pre-order cluster ids)
  uint32_t n;
  const double *rbox, *cbox;   // 6 per cluster: bmin, bmax
  const uint32_t *rsons, *csons;
  double eta;
  uint8_t *code;               // out: 0 inadmissible leaf, 1 admissible leaf, 2 refined
};

// admissible_max_cluster with getdiam_max_cluster / getdist_max_cluster (host_tree.c build_block)
__global__ void block_kernel(BlockArgs a) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
    const double *r = a.rbox + 6 * (size_t) a.rc[p], *c = a.cbox + 6 * (size_t) a.cc[p];
    double dist = 0.0, dr = 0.0, dc = 0.0;
    for (int d = 0; d < 3; d++) {
      double v = 0.0;
      if (r[3 + d] < c[d]) v = c[d] - r[3 + d];
      else if (c[3 + d] < r[d]) v = r[d] - c[3 + d];
      if (v > dist) dist = v;
      const double er = r[3 + d] - r[d], ec = c[3 + d] - c[d];
      if (er > dr) dr = er;
      if (ec > dc) dc = ec;
    }
    uint8_t code;
    if (dr <= a.eta * dist && dc <= a.eta * dist) code = 1;
    else if (a.rsons[a.rc[p]] == 0 && a.csons[a.cc[p]] == 0) code = 0;
    else code = 2;
    a.code[p] = code;
  }
}

// Stream-ordered device buffer, freed on scope exit.
struct Buf {
  void *p = nullptr;
  cudaStream_t st = nullptr;
  ~Buf() { reset(); }
  void reset() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
  }
  template <typename T> T *as() const { return (T *) p; }
};

int alloc(Buf &b, size_t bytes, cudaStream_t st) {
  b.st = st;
  if (cudaMallocAsync(&b.p, std::max<size_t>(bytes, 16), st) != cudaSuccess) {
    cudaGetLastError();
    h2b_set_error("h2b_tree_new_device: device allocation of %zu bytes failed", bytes);
    return H2B_ERR_NOMEM;
  }
  return H2B_OK;
}

// One cluster tree.  x / t are device arrays; the result is the host tree of host_tree.c.
int build_ctree(const double *dx, uint32_t nv, const uint32_t *dt, uint32_t nt, int basis,
                uint32_t clf, int grid, cudaStream_t st, h2b_ctree *out) {
  const uint32_t n = basis == H2B_BASIS_LINEAR ? nv : nt;
  Buf geo, ord, idx, flag, lv, res;
  int rc;
  // idx, then the partition scratch of ranges longer than the shared-memory stage: original
  // indices and chain links (4 B each) and flags (1 B)
  if ((rc = alloc(geo, sizeof(double) * 9 * (size_t) n, st)) ||
      (rc = alloc(idx, sizeof(uint32_t) * 3 * (size_t) n, st)) ||
      (rc = alloc(flag, (size_t) n, st)))
    return rc;
  double *cx = geo.as<double>(), *smin = cx + 3 * (size_t) n, *smax = smin + 3 * (size_t) n;
  if (basis == H2B_BASIS_LINEAR) {
    if ((rc = alloc(ord, sizeof(unsigned long long) * 6 * (size_t) n, st))) return rc;
    unsigned long long *omin = ord.as<unsigned long long>(), *omax = omin + 3 * (size_t) n;
    geom_lin_init_kernel<<<grid, 256, 0, st>>>(dx, nv, cx, omin, omax);
    geom_lin_tri_kernel<<<grid, 256, 0, st>>>(dx, dt, nt, omin, omax);
    geom_lin_fini_kernel<<<grid, 256, 0, st>>>(3 * n, omin, omax, smin, smax);
    h2b_note_launch(); h2b_note_launch(); h2b_note_launch();
  } else {
    geom_const_kernel<<<grid, 256, 0, st>>>(dx, dt, nt, cx, smin, smax);
    h2b_note_launch();
  }
  std::vector<uint32_t> hidx(n);
  for (uint32_t i = 0; i < n; i++) hidx[i] = i;
  H2B_CUDA_TRY(cudaMemcpyAsync(idx.p, hidx.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice,
                               st));
  // shared-memory stage: as many indices (original index, chain link, flag byte: 9 B) as fit
  // the opt-in limit
  const uint32_t cap = (uint32_t) ((H2B_MAX_DYN_SMEM - 64u) / 9u) & ~3u;
  H2B_CUDA_TRY((h2b_allow_smem<split_kernel<SPLIT_TPB>>()));
  H2B_CUDA_TRY((h2b_allow_smem<split_kernel<SPLIT_TPB_BIG>>()));
  // clusters in creation (breadth-first) order
  std::vector<uint32_t> c_off{0}, c_size{n}, c_level{0}, c_father{LEAF}, c_s0, c_s1;
  std::vector<double> c_box;
  uint32_t first = 0;  // first cluster of the current level
  std::vector<uint32_t> size0;
  std::vector<double> box;
  while (first < c_off.size()) {
    const uint32_t ncl = (uint32_t) c_off.size() - first;
    if ((rc = alloc(lv, sizeof(uint32_t) * 2 * (size_t) ncl, st)) ||
        (rc = alloc(res, sizeof(uint32_t) * ncl + sizeof(double) * 6 * (size_t) ncl, st)))
      return rc;
    uint32_t *doff = lv.as<uint32_t>(), *dsize = doff + ncl;
    H2B_CUDA_TRY(cudaMemcpyAsync(doff, c_off.data() + first, sizeof(uint32_t) * ncl,
                                 cudaMemcpyHostToDevice, st));
    H2B_CUDA_TRY(cudaMemcpyAsync(dsize, c_size.data() + first, sizeof(uint32_t) * ncl,
                                 cudaMemcpyHostToDevice, st));
    double *dbox = res.as<double>();
    uint32_t *ds0 = reinterpret_cast<uint32_t *>(dbox + 6 * (size_t) ncl);
    uint32_t maxsize = 0;
    for (uint32_t c = 0; c < ncl; c++) maxsize = std::max(maxsize, c_size[first + c]);
    // the stage this launch allocates: every cluster of the level fits it, or the longest ones
    // (above the opt-in limit) partition in global memory
    const uint32_t stage = (std::min(cap, maxsize) + 3u) & ~3u;
    uint32_t *didx = idx.as<uint32_t>();
    SplitArgs sa{doff, dsize, ncl, clf, cx, smin, smax, didx, flag.as<uint8_t>(),
                 didx + n, didx + 2 * (size_t) n, ds0, dbox, stage};
    const size_t smem = (size_t) stage * 9 + 16;
    if (maxsize > cap) split_kernel<SPLIT_TPB_BIG><<<ncl, SPLIT_TPB_BIG, smem, st>>>(sa);
    else split_kernel<SPLIT_TPB><<<ncl, SPLIT_TPB, smem, st>>>(sa);
    h2b_note_launch();
    H2B_CUDA_TRY(cudaGetLastError());
    size0.resize(ncl);
    box.resize(6 * (size_t) ncl);
    H2B_CUDA_TRY(cudaMemcpyAsync(size0.data(), ds0, sizeof(uint32_t) * ncl,
                                 cudaMemcpyDeviceToHost, st));
    H2B_CUDA_TRY(cudaMemcpyAsync(box.data(), dbox, sizeof(double) * 6 * ncl,
                                 cudaMemcpyDeviceToHost, st));
    H2B_CUDA_TRY(cudaStreamSynchronize(st));
    lv.reset();
    res.reset();
    const uint32_t end = (uint32_t) c_off.size();
    c_s0.resize(end, LEAF);
    c_s1.resize(end, LEAF);
    c_box.resize(6 * (size_t) end, 0.0);
    for (uint32_t c = 0; c < ncl; c++) {
      const uint32_t id = first + c;
      if (size0[c] == LEAF) {
        for (int e = 0; e < 6; e++) c_box[6 * (size_t) id + e] = box[6 * (size_t) c + e];
        continue;
      }
      c_s0[id] = (uint32_t) c_off.size();
      c_off.push_back(c_off[id]);
      c_size.push_back(size0[c]);
      c_level.push_back(c_level[id] + 1);
      c_father.push_back(id);
      c_s1[id] = (uint32_t) c_off.size();
      c_off.push_back(c_off[id] + size0[c]);
      c_size.push_back(c_size[id] - size0[c]);
      c_level.push_back(c_level[id] + 1);
      c_father.push_back(id);
    }
    first = end;
  }
  const uint32_t ncl = (uint32_t) c_off.size();
  c_s0.resize(ncl, LEAF);
  c_s1.resize(ncl, LEAF);
  c_box.resize(6 * (size_t) ncl, 0.0);
  // pre-order numbering (son0's subtree before son1's), then the host tree arrays
  std::vector<uint32_t> pre(ncl), stack{0};
  uint32_t next = 0;
  while (!stack.empty()) {
    const uint32_t id = stack.back();
    stack.pop_back();
    pre[id] = next++;
    if (c_s0[id] != LEAF) {
      stack.push_back(c_s1[id]);
      stack.push_back(c_s0[id]);
    }
  }
  memset(out, 0, sizeof(*out));
  out->n = ncl;
  out->nidx = n;
  out->off = (uint32_t *) malloc(sizeof(uint32_t) * ncl);
  out->size = (uint32_t *) malloc(sizeof(uint32_t) * ncl);
  out->sons = (uint32_t *) malloc(sizeof(uint32_t) * ncl);
  out->son0 = (uint32_t *) malloc(sizeof(uint32_t) * ncl);
  out->son1 = (uint32_t *) malloc(sizeof(uint32_t) * ncl);
  out->father = (uint32_t *) malloc(sizeof(uint32_t) * ncl);
  out->level = (uint32_t *) malloc(sizeof(uint32_t) * ncl);
  out->bmin = (double *) malloc(sizeof(double) * 3 * ncl);
  out->bmax = (double *) malloc(sizeof(double) * 3 * ncl);
  out->idx = (uint32_t *) malloc(sizeof(uint32_t) * n);
  if (!out->off || !out->size || !out->sons || !out->son0 || !out->son1 || !out->father ||
      !out->level || !out->bmin || !out->bmax || !out->idx) {
    h2b_ctree_free(out);
    h2b_set_error("h2b_tree_new_device: out of host memory");
    return H2B_ERR_NOMEM;
  }
  for (uint32_t id = 0; id < ncl; id++) {
    const uint32_t p = pre[id];
    out->off[p] = c_off[id];
    out->size[p] = c_size[id];
    out->sons[p] = c_s0[id] != LEAF ? 2 : 0;
    out->son0[p] = c_s0[id] != LEAF ? pre[c_s0[id]] : UINT32_MAX;
    out->son1[p] = c_s1[id] != LEAF ? pre[c_s1[id]] : UINT32_MAX;
    out->father[p] = c_father[id] != LEAF ? pre[c_father[id]] : UINT32_MAX;
    out->level[p] = c_level[id];
    out->depth = std::max(out->depth, c_level[id] + 1);
    for (int d = 0; d < 3; d++) {
      out->bmin[3 * p + d] = c_box[6 * (size_t) id + d];
      out->bmax[3 * p + d] = c_box[6 * (size_t) id + 3 + d];
    }
  }
  // inner clusters: the union of their sons' boxes, sons first (larger pre-order ids)
  for (uint32_t p = ncl; p-- > 0;)
    if (out->sons[p])
      for (int d = 0; d < 3; d++) {
        out->bmin[3 * p + d] = fmin(out->bmin[3 * out->son0[p] + d], out->bmin[3 * out->son1[p] + d]);
        out->bmax[3 * p + d] = fmax(out->bmax[3 * out->son0[p] + d], out->bmax[3 * out->son1[p] + d]);
      }
  H2B_CUDA_TRY(cudaMemcpyAsync(out->idx, idx.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost,
                               st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  return H2B_OK;
}

int upload_boxes(const h2b_ctree *t, Buf &b, cudaStream_t st) {
  int rc;
  if ((rc = alloc(b, sizeof(double) * 6 * (size_t) t->n + sizeof(uint32_t) * t->n, st)))
    return rc;
  std::vector<double> h(6 * (size_t) t->n);
  for (uint32_t c = 0; c < t->n; c++)
    for (int d = 0; d < 3; d++) {
      h[6 * (size_t) c + d] = t->bmin[3 * c + d];
      h[6 * (size_t) c + 3 + d] = t->bmax[3 * c + d];
    }
  H2B_CUDA_TRY(cudaMemcpyAsync(b.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice,
                               st));
  H2B_CUDA_TRY(cudaMemcpyAsync(b.as<double>() + h.size(), t->sons, sizeof(uint32_t) * t->n,
                               cudaMemcpyHostToDevice, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));  // h is a local
  return H2B_OK;
}

// The block tree: pairs level by level on the device, leaves in pre-order on the host.
int build_blist(const h2b_ctree *rt, const h2b_ctree *ct, double eta, int grid, cudaStream_t st,
                h2b_blist *out) {
  Buf rb, cb, lv;
  int rc;
  if ((rc = upload_boxes(rt, rb, st)) || (rc = upload_boxes(ct, cb, st))) return rc;
  const double *rbox = rb.as<double>(), *cbox = cb.as<double>();
  const uint32_t *rsons = reinterpret_cast<const uint32_t *>(rbox + 6 * (size_t) rt->n);
  const uint32_t *csons = reinterpret_cast<const uint32_t *>(cbox + 6 * (size_t) ct->n);
  // pair nodes in breadth-first order: clusters, code, first child, children
  std::vector<uint32_t> prc{0}, pcc{0}, child0, nchild;
  std::vector<uint8_t> code;
  uint32_t first = 0;
  while (first < prc.size()) {
    const uint32_t n = (uint32_t) prc.size() - first;
    if ((rc = alloc(lv, sizeof(uint32_t) * 2 * (size_t) n + n, st))) return rc;
    uint32_t *drc = lv.as<uint32_t>(), *dcc = drc + n;
    uint8_t *dcode = reinterpret_cast<uint8_t *>(dcc + n);
    H2B_CUDA_TRY(cudaMemcpyAsync(drc, prc.data() + first, sizeof(uint32_t) * n,
                                 cudaMemcpyHostToDevice, st));
    H2B_CUDA_TRY(cudaMemcpyAsync(dcc, pcc.data() + first, sizeof(uint32_t) * n,
                                 cudaMemcpyHostToDevice, st));
    BlockArgs ba{drc, dcc, n, rbox, cbox, rsons, csons, eta, dcode};
    block_kernel<<<std::min<uint32_t>((n + 255) / 256, (uint32_t) grid), 256, 0, st>>>(ba);
    h2b_note_launch();
    H2B_CUDA_TRY(cudaGetLastError());
    code.resize(first + n);
    H2B_CUDA_TRY(cudaMemcpyAsync(code.data() + first, dcode, n, cudaMemcpyDeviceToHost, st));
    H2B_CUDA_TRY(cudaStreamSynchronize(st));
    lv.reset();
    const uint32_t end = first + n;
    child0.resize(end, 0);
    nchild.resize(end, 0);
    for (uint32_t p = first; p < end; p++) {
      if (code[p] != 2) continue;
      const uint32_t r = prc[p], c = pcc[p];
      const uint32_t nr = rt->sons[r] ? 2 : 1, nc = ct->sons[c] ? 2 : 1;
      const uint32_t rs[2] = {rt->sons[r] ? rt->son0[r] : r, rt->son1[r]};
      const uint32_t cs[2] = {ct->sons[c] ? ct->son0[c] : c, ct->son1[c]};
      child0[p] = (uint32_t) prc.size();
      nchild[p] = nr * nc;
      for (uint32_t j = 0; j < nc; j++)  // sons column-major: column son outer
        for (uint32_t i = 0; i < nr; i++) {
          prc.push_back(rs[i]);
          pcc.push_back(cs[j]);
        }
    }
    first = end;
  }
  const uint32_t np = (uint32_t) prc.size();
  child0.resize(np, 0);
  nchild.resize(np, 0);
  // leaves below each node (children come after their father), then the pre-order position
  std::vector<uint32_t> leaves(np), pos(np);
  for (uint32_t p = np; p-- > 0;) {
    if (code[p] != 2) {
      leaves[p] = 1;
      continue;
    }
    uint32_t s = 0;
    for (uint32_t q = 0; q < nchild[p]; q++) s += leaves[child0[p] + q];
    leaves[p] = s;
  }
  pos[0] = 0;
  for (uint32_t p = 0; p < np; p++) {
    if (code[p] != 2) continue;
    uint32_t o = pos[p];
    for (uint32_t q = 0; q < nchild[p]; q++) {
      pos[child0[p] + q] = o;
      o += leaves[child0[p] + q];
    }
  }
  memset(out, 0, sizeof(*out));
  out->n = leaves[0];
  out->rc = (uint32_t *) malloc(sizeof(uint32_t) * std::max<uint32_t>(out->n, 1));
  out->cc = (uint32_t *) malloc(sizeof(uint32_t) * std::max<uint32_t>(out->n, 1));
  out->adm = (uint8_t *) malloc(std::max<uint32_t>(out->n, 1));
  if (!out->rc || !out->cc || !out->adm) {
    h2b_blist_free(out);
    h2b_set_error("h2b_tree_new_device: out of host memory");
    return H2B_ERR_NOMEM;
  }
  for (uint32_t p = 0; p < np; p++)
    if (code[p] != 2) {
      out->rc[pos[p]] = prc[p];
      out->cc[pos[p]] = pcc[p];
      out->adm[pos[p]] = code[p];
    }
  return H2B_OK;
}

}  // namespace

extern "C" h2b_tree *h2b_tree_new_device(uint32_t vertices, const double *x, uint32_t triangles,
                                        const uint32_t *t, int row_basis, int col_basis,
                                        uint32_t clf, double eta) {
  if (!x || !t || vertices == 0 || triangles == 0) {
    h2b_set_error("h2b_tree_new_device: empty mesh");
    return NULL;
  }
  if ((row_basis != H2B_BASIS_CONSTANT && row_basis != H2B_BASIS_LINEAR) ||
      (col_basis != H2B_BASIS_CONSTANT && col_basis != H2B_BASIS_LINEAR) || !(eta > 0.0) ||
      clf < 1) {
    h2b_set_error("h2b_tree_new_device: invalid basis, leaf size or eta");
    return NULL;
  }
  for (uint64_t i = 0; i < 3 * (uint64_t) triangles; i++)
    if (t[i] >= vertices) {
      h2b_set_error("h2b_tree_new_device: triangle vertex %u out of range", t[i]);
      return NULL;
    }
  if (h2b_ensure_device() != H2B_OK) return NULL;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = 4 * sms;
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    h2b_set_error("h2b_tree_new_device: stream creation failed");
    return NULL;
  }
  h2b_tree *tr = (h2b_tree *) calloc(1, sizeof(h2b_tree));
  int rc = tr ? H2B_OK : H2B_ERR_NOMEM;
  {
    Buf mesh;
    if (rc == H2B_OK)
      rc = alloc(mesh, sizeof(double) * 3 * (size_t) vertices + sizeof(uint32_t) * 3 * (size_t) triangles, st);
    double *dx = mesh.as<double>();
    uint32_t *dt = reinterpret_cast<uint32_t *>(dx + 3 * (size_t) vertices);
    if (rc == H2B_OK &&
        (cudaMemcpyAsync(dx, x, sizeof(double) * 3 * (size_t) vertices, cudaMemcpyHostToDevice, st) != cudaSuccess ||
         cudaMemcpyAsync(dt, t, sizeof(uint32_t) * 3 * (size_t) triangles, cudaMemcpyHostToDevice, st) != cudaSuccess)) {
      h2b_set_error("h2b_tree_new_device: %s", cudaGetErrorString(cudaGetLastError()));
      rc = H2B_ERR_CUDA;
    }
    if (rc == H2B_OK) {
      tr->row_basis = row_basis;
      tr->col_basis = col_basis;
      rc = build_ctree(dx, vertices, dt, triangles, row_basis, clf, grid, st, &tr->row);
      // equal bases give equal trees: copy the row tree (as h2b_tree_new does)
      if (rc == H2B_OK)
        rc = col_basis == row_basis
                 ? h2b_ctree_copy(&tr->col, &tr->row)
                 : build_ctree(dx, vertices, dt, triangles, col_basis, clf, grid, st, &tr->col);
      if (rc == H2B_OK) rc = build_blist(&tr->row, &tr->col, eta, grid, st, &tr->blocks);
    }
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (rc != H2B_OK) {
    if (rc == H2B_ERR_NOMEM && tr) h2b_set_error("h2b_tree_new_device: out of memory");
    if (tr) h2b_tree_del(tr);
    return NULL;
  }
  h2b_tree_finish(tr);
  return tr;
}
