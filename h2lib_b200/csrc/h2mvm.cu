// H2 matrix-vector product y += alpha A x on the device (sm_100a).
//
// Follows addeval_h2matrix_avector (Library/h2matrix.c:1269):
//   forward transform   xt_t = V_t^T x_t (leaves), xt_t = sum_s E_s^T xt_s (Library/clusterbasis.c:524)
//   coupling / near     yt_t += S_b xt_s,  y_t += N_b x_s      (fastaddeval, Library/h2matrix.c:1211)
//   backward transform  yt_s += E_s yt_t,  y_t += V_t yt_t     (Library/clusterbasis.c:749)
// The nested transforms are multiplied out once after assembly (flatbasis.cu): for every cluster
// t of an admissible block, W_t = V_t (leaf) or [W_s E_s] over the sons s, the |t| x k basis on
// t's own indices, stored transposed (k x |t|).  The forward transform is then xt_t = W_t^T x_t
// and the backward transform y_t += W_t yt_t for every such cluster independently.
//
// Every product is a list of small dense GEMV work items (h2mvm.h: MvItem), ordered by kind and
// run by three launches of one persistent kernel between a gather (xp = x[idx], accumulators
// cleared) and a scatter (y[idx] += alpha yp):
//   1. forward     xt_t += (W_t^T slice) x_slice,   and nearfield   y_r += N_b x_c
//   2. coupling    yt_r += S_b xt_c
//   3. backward    y_slice += (W_t^T slice)^T yt_t
// Vectors are kept in cluster order, so every item's x and y are contiguous slices.  (Running
// all three in one launch, with counters per cluster carrying the dependences, measured slower:
// the counter and claim atomics cost more than the two launch boundaries.)
//
// The kernel streams each item's panel — a contiguous column-major block of N, S or W^T — and its
// x slice into a ring of shared-memory stages with bulk asynchronous copies (cp.async.bulk
// global -> shared, completion counted on an mbarrier per stage), issued by a producer warp, so
// that several panels per SM are in flight while consumer warps multiply earlier ones from
// shared memory.  The copies are local to this GPU and have no cluster multicast.  Every wait is
// bounded: on time-out the kernel sets the plan's error flag, waits (bounded) for its copies in
// flight and returns.  Partial sums reach their outputs with FP64 atomics.
// CX: complex coefficients (Helmholtz) — S, N, x, y complex (interleaved); W real.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <type_traits>

#include "device_common.cuh"
#include "h2mvm.h"

namespace {

constexpr int MAXTHREADS = 288;              // up to 8 consumer warps and the producer warp
constexpr int MAXROWS = 128;                 // rows of an untransposed item, columns of a transposed
                                             // one (four 32-lane slots)
constexpr uint32_t WAIT_LIMIT = 1u << 24;    // try_wait polls before a stage counts as lost

// Vectors of a product with nrhs right-hand sides.  With a mask (batched solves on a forest:
// mask[surface + r * nseg] for column r) an item skips the columns whose system is done.
struct MvmVecs {
  double *xp, *yp, *xt, *yt;      // work vectors, column r at r * stride
  size_t sxp, syp, sxt, syt;
  uint32_t nrhs, nseg;
  const uint32_t *mask;           // NULL: every column
};

__device__ __forceinline__ bool col_on(const uint32_t *mask, uint32_t nseg, uint32_t seg,
                                       uint32_t r) {
  return !mask || mask[seg + r * nseg] != 0;
}

// xp = x[idx] per column; the accumulators yp, xt, yt are cleared.
template <bool CX>
__global__ void gather_zero_kernel(const double *__restrict__ x, size_t ldx,
                                   const uint32_t *__restrict__ idx, uint32_t n, MvmVecs v,
                                   size_t nyp, size_t nxt, size_t nyt) {
  const size_t i0 = blockIdx.x * (size_t) blockDim.x + threadIdx.x, st = (size_t) gridDim.x * blockDim.x;
  for (uint32_t r = 0; r < v.nrhs; r++) {
    const double *xr = x + r * ldx;
    double *xp = v.xp + r * v.sxp;
    for (size_t i = i0; i < n; i += st) {
      const uint32_t j = idx[i];
      if (CX) {
        xp[2 * i] = xr[2 * j];
        xp[2 * i + 1] = xr[2 * j + 1];
      } else {
        xp[i] = xr[j];
      }
    }
    for (size_t i = i0; i < nyp; i += st) v.yp[r * v.syp + i] = 0.0;
    for (size_t i = i0; i < nxt; i += st) v.xt[r * v.sxt + i] = 0.0;
    for (size_t i = i0; i < nyt; i += st) v.yt[r * v.syt + i] = 0.0;
  }
}

// y[idx[i]] += alpha * yp[i] per column
template <bool CX>
__global__ void scatter_multi_kernel(MvmVecs v, const uint32_t *__restrict__ idx,
                                     double *__restrict__ y, size_t ldy, uint32_t n, double ar,
                                     double ai) {
  for (uint32_t r = 0; r < v.nrhs; r++) {
    const double *yp = v.yp + r * v.syp;
    double *yr = y + r * ldy;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      const uint32_t j = idx[i];
      if (CX) {
        const double re = yp[2 * i], im = yp[2 * i + 1];
        yr[2 * j] += ar * re - ai * im;
        yr[2 * j + 1] += ar * im + ai * re;
      } else {
        yr[j] += ar * yp[i];
      }
    }
  }
}

// One launch of the item kernel.
struct MvLaunch {
  const MvItem *items;
  uint32_t n;
  const void *A[4];        // panel array per kind: W_c^T, N, S, W_r^T (N, S complex when CX)
  const double *X[4];      // x work vector per kind
  double *Y[4];            // y work vector per kind
  size_t sx[4], sy[4];     // column strides (doubles)
  uint32_t first;          // the launch's items: first .. first + n - 1 of the list
  uint32_t nrhs, nseg;
  const uint32_t *mask;
  int *err;
  uint32_t stage_bytes;    // bytes per stage (multiple of 128)
  uint32_t panel_bytes;    // panel region of a stage; the x slices of every column follow
  uint32_t xcol_bytes;     // bytes per x slice of one column (multiple of 16, with slack)
  uint32_t stages;         // ring stages, a multiple of nw: stage s belongs to consumer warp s % nw
  uint32_t nw;             // consumer warps; warp nw produces
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool bar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t spin = 0; spin < WAIT_LIMIT; spin++)
    if (bar_try(bar, parity)) return true;
  return false;
}

// [lo, lo + bytes): the 16-byte aligned span that covers [addr, addr + n); delta = addr - lo.
// The arrays and work vectors carry at least 16 bytes of slack after their ends.
__device__ __forceinline__ void span16(const void *addr, size_t n, const char *&lo,
                                       uint32_t &delta, uint32_t &bytes) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(addr);
  lo = reinterpret_cast<const char *>(a & ~(uintptr_t) 15);
  delta = (uint32_t) (a & 15u);
  bytes = (uint32_t) ((delta + n + 15) & ~(size_t) 15);
}

// complex panel entries: nearfield and coupling panels of a complex operator
__device__ __forceinline__ bool complex_panel(uint32_t kind) {
  return kind == H2B_MV_NEAR || kind == H2B_MV_COUPLING;
}

template <bool CX, typename T>
__device__ __forceinline__ const char *panel_addr(const MvLaunch &L, const MvItem &m, size_t &n) {
  const uint32_t kind = m.flags & H2B_MV_KIND;
  const size_t esz = sizeof(T) * ((CX && complex_panel(kind)) ? 2 : 1);
  n = (size_t) m.rows * m.cols * esz;
  return reinterpret_cast<const char *>(L.A[kind]) + m.p * esz;
}

// entry e of a panel (complex entries as one vector load: a complex panel starts on a multiple of
// its entry size, so the stage copy keeps that alignment)
template <bool PCX, typename T>
__device__ __forceinline__ void entry(const T *P, size_t e, double &re, double &im) {
  if constexpr (PCX) {
    using V2 = typename std::conditional<std::is_same<T, float>::value, float2, double2>::type;
    const V2 v = reinterpret_cast<const V2 *>(P)[e];
    re = (double) v.x;
    im = (double) v.y;
  } else {
    re = (double) P[e];
    im = 0.0;
  }
}

// y[0, R) += P x[0, C) by one warp: lanes take rows (SL slots of 32), the warp runs over the
// columns; one atomic addition per row.
template <bool CX, bool PCX, typename T, int SL>
__device__ __forceinline__ void warp_gemv_n(const T *__restrict__ P, uint32_t R, uint32_t C,
                                            const double *__restrict__ xs, double *y,
                                            uint32_t lane) {
  constexpr int W = CX ? 2 : 1;
  double sr[SL], si[SL];
  bool on[SL];
#pragma unroll
  for (int j = 0; j < SL; j++) {
    sr[j] = si[j] = 0.0;
    on[j] = lane + 32u * j < R;
  }
#pragma unroll 4
  for (uint32_t c = 0; c < C; c++) {
    const double xr = xs[W * c], xi = CX ? xs[W * c + 1] : 0.0;
    const T *col = P + (size_t) (PCX ? 2 : 1) * c * R;
#pragma unroll
    for (int j = 0; j < SL; j++) {
      if (on[j]) {
        double pr, pi;
        entry<PCX>(col, lane + 32u * j, pr, pi);
        if (PCX) {
          sr[j] = fma(pr, xr, fma(-pi, xi, sr[j]));
          si[j] = fma(pr, xi, fma(pi, xr, si[j]));
        } else {
          sr[j] = fma(pr, xr, sr[j]);
          if (CX) si[j] = fma(pr, xi, si[j]);
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < SL; j++) {
    if (on[j]) {
      const uint32_t r = lane + 32u * j;
      atomicAdd(y + W * r, sr[j]);
      if (CX) atomicAdd(y + W * r + 1, si[j]);
    }
  }
}

// y[0, C) += P^T x[0, R) by one warp for a real panel: lanes take columns (SL slots of 32) and
// run over the rows from a lane-dependent start, row (it + lane) mod R at step it, so that the
// warp's reads of the column-major panel fall in distinct banks.
template <bool CX, typename T, int SL>
__device__ __forceinline__ void warp_gemv_t(const T *__restrict__ P, uint32_t R, uint32_t C,
                                            const double *__restrict__ xs, double *y,
                                            uint32_t lane) {
  constexpr int W = CX ? 2 : 1;
  double sr[SL], si[SL];
  bool on[SL];
#pragma unroll
  for (int j = 0; j < SL; j++) {
    sr[j] = si[j] = 0.0;
    on[j] = lane + 32u * j < C;
  }
  uint32_t r = lane % R;
#pragma unroll 4
  for (uint32_t it = 0; it < R; it++) {
    const double xr = xs[W * r], xi = CX ? xs[W * r + 1] : 0.0;
#pragma unroll
    for (int j = 0; j < SL; j++) {
      if (on[j]) {
        const double p = (double) P[r + (size_t) (lane + 32u * j) * R];
        sr[j] = fma(p, xr, sr[j]);
        if (CX) si[j] = fma(p, xi, si[j]);
      }
    }
    r = r + 1 == R ? 0u : r + 1;
  }
#pragma unroll
  for (int j = 0; j < SL; j++) {
    if (on[j]) {
      const uint32_t c = lane + 32u * j;
      atomicAdd(y + W * c, sr[j]);
      if (CX) atomicAdd(y + W * c + 1, si[j]);
    }
  }
}

template <bool CX, bool PCX, typename T>
__device__ __forceinline__ void gemv_n_any(const T *P, uint32_t R, uint32_t C, const double *xs,
                                           double *y, uint32_t lane) {
  switch ((R + 31) >> 5) {
    case 1: warp_gemv_n<CX, PCX, T, 1>(P, R, C, xs, y, lane); break;
    case 2: warp_gemv_n<CX, PCX, T, 2>(P, R, C, xs, y, lane); break;
    case 3: warp_gemv_n<CX, PCX, T, 3>(P, R, C, xs, y, lane); break;
    default: warp_gemv_n<CX, PCX, T, 4>(P, R, C, xs, y, lane); break;
  }
}

template <bool CX, typename T>
__device__ __forceinline__ void gemv_t_any(const T *P, uint32_t R, uint32_t C, const double *xs,
                                           double *y, uint32_t lane) {
  switch ((C + 31) >> 5) {
    case 1: warp_gemv_t<CX, T, 1>(P, R, C, xs, y, lane); break;
    case 2: warp_gemv_t<CX, T, 2>(P, R, C, xs, y, lane); break;
    case 3: warp_gemv_t<CX, T, 3>(P, R, C, xs, y, lane); break;
    default: warp_gemv_t<CX, T, 4>(P, R, C, xs, y, lane); break;
  }
}

// Warp nw produces: for each of the CTA's items i (list entry first + blockIdx.x + i gridDim.x)
// it copies the panel and the x slice of every right-hand side into stage i % S (one bulk copy
// each, completion on full[s]) once the stage's previous item has been released (empty[s]), and
// puts the descriptor in the stage's slot.
// Consumer warp w multiplies the items i = w, w + nw, ... alone: S is a multiple of nw, so stage
// i % S always belongs to the same warp, and no barrier joins the consumer warps.  Every wait is
// bounded; a warp whose wait runs out sets the error flag and leaves, and the others' bounded
// waits end the CTA.
template <bool CX, typename T>
__global__ void __launch_bounds__(MAXTHREADS) mv_items_kernel(MvLaunch L) {
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr int W = CX ? 2 : 1;
  const uint32_t S = L.stages;
  unsigned char *stage0 = smem;
  MvItem *slot = reinterpret_cast<MvItem *>(smem + (size_t) S * L.stage_bytes);
  uint64_t *full = reinterpret_cast<uint64_t *>(slot + S);
  uint64_t *empty = full + S;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t mine = L.n > blockIdx.x ? (L.n - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < S; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&full[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&empty[s])));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (warp == L.nw) {
    // ---- producer (one lane): the next descriptor is fetched while the current copies run
    if (lane != 0 || mine == 0) return;
    MvItem m = L.items[L.first + blockIdx.x];
    uint32_t i = 0;
    bool ok = true;
    for (; i < mine; i++) {
      const uint32_t s = i % S;
      if (i >= S && !(ok = bar_wait(smem_addr(&empty[s]), ((i / S) - 1) & 1u))) break;
      const uint32_t bar = smem_addr(&full[s]);
      slot[s] = m;
      size_t n;
      const char *pa = panel_addr<CX, T>(L, m, n), *lo;
      uint32_t delta, bytes;
      span16(pa, n, lo, delta, bytes);
      const int t = m.flags & H2B_MV_KIND;
      const size_t xn = (size_t) W * sizeof(double) * ((m.flags & H2B_MV_TRANS) ? m.rows : m.cols);
      // only the columns whose system is still running are copied; an item with none (its
      // surface's systems have all stopped) loads nothing and its stage completes at once
      uint32_t total = 0;
      bool any = false;
      for (uint32_t q = 0; q < L.nrhs; q++) {
        if (!col_on(L.mask, L.nseg, m.seg, q)) continue;
        const char *xl;
        uint32_t xd, xb;
        span16(L.X[t] + q * L.sx[t] + (size_t) W * m.xo, xn, xl, xd, xb);
        total += xb;
        any = true;
      }
      if (!any) {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
      } else {
        total += bytes;
        const uint32_t dst = smem_addr(stage0 + (size_t) s * L.stage_bytes);
        // the generic-proxy reads of the stage's previous contents are ordered before these
        // copies
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"(total)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(dst), "l"(lo), "r"(bytes), "r"(bar)
            : "memory");
        for (uint32_t q = 0; q < L.nrhs; q++) {
          if (!col_on(L.mask, L.nseg, m.seg, q)) continue;
          const char *xl;
          uint32_t xd, xb;
          span16(L.X[t] + q * L.sx[t] + (size_t) W * m.xo, xn, xl, xd, xb);
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
              "[%3];" ::"r"(dst + L.panel_bytes + q * L.xcol_bytes), "l"(xl), "r"(xb), "r"(bar)
              : "memory");
        }
      }
      if (i + 1 < mine) m = L.items[L.first + blockIdx.x + (i + 1) * gridDim.x];
    }
    if (!ok) {
      // a wait ran out: flag it and wait (bounded) for the copies this warp issued before it
      // leaves the CTA's shared memory (the consumers give up at their next stage)
      atomicExch(L.err, 1);
      for (uint32_t j = i > S ? i - S : 0; j < i; j++)
        bar_wait(smem_addr(&full[j % S]), (j / S) & 1u);
    }
    return;
  }
  if (warp > L.nw) return;

  // ---- consumers
  for (uint32_t i = warp; i < mine; i += L.nw) {
    const uint32_t s = i % S;
    if (!bar_wait(smem_addr(&full[s]), (i / S) & 1u)) {
      if (lane == 0) atomicExch(L.err, 1);
      return;
    }
    const MvItem m = slot[s];
    const unsigned char *stage = stage0 + (size_t) s * L.stage_bytes;
    size_t n;
    const char *pa = panel_addr<CX, T>(L, m, n), *lo;
    uint32_t delta, bytes;
    span16(pa, n, lo, delta, bytes);
    const T *P = reinterpret_cast<const T *>(stage + delta);
    const int t = m.flags & H2B_MV_KIND;
    const bool trans = (m.flags & H2B_MV_TRANS) != 0;
    const size_t xn = (size_t) W * sizeof(double) * (trans ? m.rows : m.cols);
    for (uint32_t q = 0; q < L.nrhs; q++) {
      if (!col_on(L.mask, L.nseg, m.seg, q)) continue;  // the column's system is done
      const char *xl;
      uint32_t xd, xb;
      span16(L.X[t] + q * L.sx[t] + (size_t) W * m.xo, xn, xl, xd, xb);
      const double *xs =
          reinterpret_cast<const double *>(stage + L.panel_bytes + q * L.xcol_bytes + xd);
      double *y = L.Y[t] + q * L.sy[t] + (size_t) W * m.yo;
      if (trans) gemv_t_any<CX, T>(P, m.rows, m.cols, xs, y, lane);
      else if (CX && complex_panel(t)) gemv_n_any<CX, CX, T>(P, m.rows, m.cols, xs, y, lane);
      else gemv_n_any<CX, false, T>(P, m.rows, m.cols, xs, y, lane);
    }
    __syncwarp();
    if (lane == 0)
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&empty[s]))
                   : "memory");
  }
}

// Stage layout: the panel (FP64 panel bytes scaled to the storage type, plus 32 bytes for the
// alignment and rounding slack) and the x slices of nrhs columns.
template <typename T>
uint32_t panel_region(const MvItems &ph) {
  const size_t b = (size_t) ph.max_bytes * sizeof(T) / sizeof(double) + 32;
  return (uint32_t) ((b + 127) & ~(size_t) 127);
}

template <bool CX>
uint32_t xcol_region(const MvItems &ph) {
  return (uint32_t) ((sizeof(double) * (CX ? 2 : 1) * ph.max_x + 32 + 15) & ~(size_t) 15);
}

template <bool CX, typename T>
uint32_t stage_of(const MvItems &ph, uint32_t nrhs) {
  const size_t b = panel_region<T>(ph) + (size_t) nrhs * xcol_region<CX>(ph);
  return (uint32_t) ((b + 127) & ~(size_t) 127);
}

template <bool CX, typename T>
size_t smem_of(const MvItems &ph, uint32_t stages, uint32_t nrhs) {
  return (size_t) stages * (stage_of<CX, T>(ph, nrhs) + sizeof(MvItem) + 16);
}

// consumer warps and ring stages of a launch shape (stages per consumer warp 1..4)
void ring_shape(const MvmPlan *p, uint32_t &nw, uint32_t &stages) {
  nw = (uint32_t) std::max(1, std::min(MAXTHREADS / 32 - 1, p->warps));
  stages = nw * (uint32_t) std::max(1, std::min(4, p->stages));
}

template <bool CX, typename T>
int launch_range(const MvmPlan *p, const MvItems &ph, const MvLaunch &base, uint32_t first,
                 uint32_t last, cudaStream_t st) {
  if (last <= first) return H2B_OK;
  MvLaunch L = base;
  L.items = ph.items;
  L.first = first;
  L.n = last - first;
  ring_shape(p, L.nw, L.stages);
  L.panel_bytes = panel_region<T>(ph);
  L.xcol_bytes = xcol_region<CX>(ph);
  L.stage_bytes = stage_of<CX, T>(ph, L.nrhs);
  const size_t smem = smem_of<CX, T>(ph, L.stages, L.nrhs);
  if (smem > H2B_MAX_DYN_SMEM || ph.max_rows > MAXROWS || ph.max_cols_t > MAXROWS ||
      ph.max_x > 65536) {
    h2b_set_error("matvec: item panel of %u bytes / %u rows / %u transposed columns / %u "
                  "right-hand sides exceeds the kernel's limits (%zu bytes of shared memory)",
                  ph.max_bytes, ph.max_rows, ph.max_cols_t, L.nrhs, smem);
    return H2B_ERR_ARG;
  }
  const int threads = (int) (L.nw + 1) * 32;
  H2B_CUDA_TRY((h2b_allow_smem<mv_items_kernel<CX, T>>()));
  int occ = 0;
  H2B_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mv_items_kernel<CX, T>,
                                                             threads, smem));
  if (occ < 1) {
    h2b_set_error("matvec: the item kernel does not fit an SM (%zu bytes of shared memory)", smem);
    return H2B_ERR_ARG;
  }
  const int sms = p->num_sms > 0 ? p->num_sms : 148;
  const int per_sm = std::min(occ, std::max(1, p->ctas_per_sm));
  const uint32_t grid = std::min<uint32_t>(L.n, (uint32_t) (per_sm * sms));
  mv_items_kernel<CX, T><<<grid, threads, smem, st>>>(L);
  h2b_note_launch();
  return H2B_OK;
}

template <bool CX, bool SINGLE>
int launch_all(const MvmPlan *p, const double *x, size_t ldx, double *y, size_t ldy, double ar,
               double ai, const MvmVecs &v, cudaStream_t st) {
  using T = typename std::conditional<SINGLE, float, double>::type;
  const size_t W = CX ? 2 : 1;
  const int sms = p->num_sms > 0 ? p->num_sms : 148;
  const uint32_t zn = p->nrow > p->ncol ? p->nrow : p->ncol;
  const uint32_t gz = std::min<uint32_t>((zn + 255) / 256 + 1, (uint32_t) (4 * sms));
  const size_t nyp = W * p->nrow, nxt = W * (size_t) p->k * p->ncol_clusters,
               nyt = W * (size_t) p->k * p->nrow_clusters;
  gather_zero_kernel<CX><<<gz, 256, 0, st>>>(x, ldx, p->cidx, p->ncol, v, nyp, nxt, nyt);
  h2b_note_launch();
  MvLaunch L{};
  L.nrhs = v.nrhs;
  L.nseg = v.nseg;
  L.mask = v.mask;
  L.err = p->err;
  L.A[H2B_MV_FORWARD] = SINGLE ? (const void *) p->fWc : (const void *) p->Wc;
  L.A[H2B_MV_NEAR] = SINGLE ? (const void *) p->fN : (const void *) p->N;
  L.A[H2B_MV_COUPLING] = SINGLE ? (const void *) p->fS : (const void *) p->S;
  L.A[H2B_MV_BACKWARD] = SINGLE ? (const void *) p->fWr : (const void *) p->Wr;
  L.X[H2B_MV_FORWARD] = v.xp, L.Y[H2B_MV_FORWARD] = v.xt;
  L.sx[H2B_MV_FORWARD] = v.sxp, L.sy[H2B_MV_FORWARD] = v.sxt;
  L.X[H2B_MV_NEAR] = v.xp, L.Y[H2B_MV_NEAR] = v.yp;
  L.sx[H2B_MV_NEAR] = v.sxp, L.sy[H2B_MV_NEAR] = v.syp;
  L.X[H2B_MV_COUPLING] = v.xt, L.Y[H2B_MV_COUPLING] = v.yt;
  L.sx[H2B_MV_COUPLING] = v.sxt, L.sy[H2B_MV_COUPLING] = v.syt;
  L.X[H2B_MV_BACKWARD] = v.yt, L.Y[H2B_MV_BACKWARD] = v.yp;
  L.sx[H2B_MV_BACKWARD] = v.syt, L.sy[H2B_MV_BACKWARD] = v.syp;
  const MvItems &it = SINGLE ? p->items_single : p->items;
  // forward + nearfield, coupling (reads xt), backward (reads yt)
  int rc = launch_range<CX, T>(p, it, L, 0, it.start[H2B_MV_COUPLING], st);
  if (rc == H2B_OK)
    rc = launch_range<CX, T>(p, it, L, it.start[H2B_MV_COUPLING], it.start[H2B_MV_BACKWARD], st);
  if (rc == H2B_OK) rc = launch_range<CX, T>(p, it, L, it.start[H2B_MV_BACKWARD], it.n, st);
  if (rc != H2B_OK) return rc;
  scatter_multi_kernel<CX><<<gz, 256, 0, st>>>(v, p->ridx, y, ldy, p->nrow, ar, ai);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

// The plan's own work vectors (one column, no mask).
MvmVecs plan_vecs(const MvmPlan *p) {
  MvmVecs v;
  v.xp = p->xp;
  v.yp = p->yp;
  v.xt = p->xt;
  v.yt = p->yt;
  v.sxp = v.syp = v.sxt = v.syt = 0;
  v.nrhs = 1;
  v.nseg = 1;
  v.mask = nullptr;
  return v;
}

bool has_single(const MvmPlan *p) { return p->fWc && p->fWr && p->fN && p->fS; }

// xs = b xp and xp = a xp, n entries (complex: interleaved pairs).
template <bool CX>
__global__ void scale_copy_kernel(double *__restrict__ xp, double *__restrict__ xs, uint32_t n,
                                  double ar, double ai, double br, double bi) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (CX) {
      const double re = xp[2 * i], im = xp[2 * i + 1];
      xs[2 * i] = br * re - bi * im;
      xs[2 * i + 1] = br * im + bi * re;
      xp[2 * i] = ar * re - ai * im;
      xp[2 * i + 1] = ar * im + ai * re;
    } else {
      const double v = xp[i];
      xs[i] = br * v;
      xp[i] = ar * v;
    }
  }
}

// y += a A x + b B x for two matrices on one structure whose coupling matrices and row bases
// are equal (the caller checks): the forward transforms and nearfield blocks of both run on
// their own scaled copies of x into p's accumulators, then p's coupling matrices and row basis
// are applied once.
template <bool CX, bool SINGLE>
int launch_pair(const MvmPlan *p, const MvmPlan *q, const double *x, double *y, double ar,
                double ai, double br, double bi, const MvmVecs &v, double *xq, cudaStream_t st) {
  using T = typename std::conditional<SINGLE, float, double>::type;
  const size_t W = CX ? 2 : 1;
  const int sms = p->num_sms > 0 ? p->num_sms : 148;
  const uint32_t zn = p->nrow > p->ncol ? p->nrow : p->ncol;
  const uint32_t gz = std::min<uint32_t>((zn + 255) / 256 + 1, (uint32_t) (4 * sms));
  const size_t nyp = W * p->nrow, nxt = W * (size_t) p->k * p->ncol_clusters,
               nyt = W * (size_t) p->k * p->nrow_clusters;
  gather_zero_kernel<CX><<<gz, 256, 0, st>>>(x, 0, p->cidx, p->ncol, v, nyp, nxt, nyt);
  h2b_note_launch();
  scale_copy_kernel<CX><<<gz, 256, 0, st>>>(v.xp, xq, p->ncol, ar, ai, br, bi);
  h2b_note_launch();
  MvLaunch L{};
  L.nrhs = 1;
  L.nseg = 1;
  L.mask = nullptr;
  L.err = p->err;
  L.A[H2B_MV_FORWARD] = SINGLE ? (const void *) p->fWc : (const void *) p->Wc;
  L.A[H2B_MV_NEAR] = SINGLE ? (const void *) p->fN : (const void *) p->N;
  L.A[H2B_MV_COUPLING] = SINGLE ? (const void *) p->fS : (const void *) p->S;
  L.A[H2B_MV_BACKWARD] = SINGLE ? (const void *) p->fWr : (const void *) p->Wr;
  L.X[H2B_MV_FORWARD] = v.xp, L.Y[H2B_MV_FORWARD] = v.xt;
  L.X[H2B_MV_NEAR] = v.xp, L.Y[H2B_MV_NEAR] = v.yp;
  L.X[H2B_MV_COUPLING] = v.xt, L.Y[H2B_MV_COUPLING] = v.yt;
  L.X[H2B_MV_BACKWARD] = v.yt, L.Y[H2B_MV_BACKWARD] = v.yp;
  MvLaunch Lq = L;
  Lq.A[H2B_MV_FORWARD] = SINGLE ? (const void *) q->fWc : (const void *) q->Wc;
  Lq.A[H2B_MV_NEAR] = SINGLE ? (const void *) q->fN : (const void *) q->N;
  Lq.X[H2B_MV_FORWARD] = xq;
  Lq.X[H2B_MV_NEAR] = xq;
  const MvItems &it = SINGLE ? p->items_single : p->items;
  const MvItems &iq = SINGLE ? q->items_single : q->items;
  int rc = launch_range<CX, T>(p, it, L, 0, it.start[H2B_MV_COUPLING], st);
  if (rc == H2B_OK) rc = launch_range<CX, T>(p, iq, Lq, 0, iq.start[H2B_MV_COUPLING], st);
  if (rc == H2B_OK)
    rc = launch_range<CX, T>(p, it, L, it.start[H2B_MV_COUPLING], it.start[H2B_MV_BACKWARD], st);
  if (rc == H2B_OK) rc = launch_range<CX, T>(p, it, L, it.start[H2B_MV_BACKWARD], it.n, st);
  if (rc != H2B_OK) return rc;
  scatter_multi_kernel<CX><<<gz, 256, 0, st>>>(v, p->ridx, y, 0, p->nrow, 1.0, 0.0);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}


}  // namespace

extern "C" int h2b_mvm_prepare(void) {
  H2B_CUDA_TRY((h2b_allow_smem<mv_items_kernel<false, double>>()));
  H2B_CUDA_TRY((h2b_allow_smem<mv_items_kernel<true, double>>()));
  H2B_CUDA_TRY((h2b_allow_smem<mv_items_kernel<false, float>>()));
  H2B_CUDA_TRY((h2b_allow_smem<mv_items_kernel<true, float>>()));
  return H2B_OK;
}

extern "C" size_t h2b_mvm_smem_bytes(const MvmPlan *p, int single) {
  const MvItems &ph = single ? p->items_single : p->items;
  uint32_t nw, stages;
  ring_shape(p, nw, stages);
  if (p->cx)
    return single ? smem_of<true, float>(ph, stages, 1) : smem_of<true, double>(ph, stages, 1);
  return single ? smem_of<false, float>(ph, stages, 1) : smem_of<false, double>(ph, stages, 1);
}

extern "C" int h2b_mvm_launch_single(const MvmPlan *p, const double *x, double *y, double ar,
                                     double ai, cudaStream_t st) {
  if (!has_single(p)) {
    h2b_set_error("matvec: no FP32 copy of the H2 matrix (h2b_h2matrix_make_single)");
    return H2B_ERR_ARG;
  }
  const MvmVecs v = plan_vecs(p);
  return p->cx ? launch_all<true, true>(p, x, 0, y, 0, ar, ai, v, st)
               : launch_all<false, true>(p, x, 0, y, 0, ar, ai, v, st);
}

extern "C" int h2b_mvm_launch(const MvmPlan *p, const double *x, double *y, double ar, double ai,
                              cudaStream_t st) {
  const MvmVecs v = plan_vecs(p);
  return p->cx ? launch_all<true, false>(p, x, 0, y, 0, ar, ai, v, st)
               : launch_all<false, false>(p, x, 0, y, 0, ar, ai, v, st);
}

extern "C" size_t h2b_mvm_pair_work_doubles(const MvmPlan *p) {
  // one column of p's vectors, then the second scaled copy of x with its own slack
  return h2b_mvm_work_doubles(p, 1) + (size_t) (p->cx ? 2 : 1) * p->ncol + 8;
}

extern "C" int h2b_mvm_launch_pair(const MvmPlan *p, const MvmPlan *q, int single,
                                   const double *x, double *y, double ar, double ai, double br,
                                   double bi, double *work, cudaStream_t st) {
  if (single && (!has_single(p) || !has_single(q))) {
    h2b_set_error("matvec: no FP32 copy of the H2 matrix (h2b_h2matrix_make_single)");
    return H2B_ERR_ARG;
  }
  MvmVecs v = plan_vecs(p);
  double *xq = q->xp;
  if (work) {
    const size_t W = p->cx ? 2 : 1;
    v.xp = work;
    v.yp = v.xp + W * p->ncol;
    v.xt = v.yp + W * p->nrow;
    v.yt = v.xt + W * (size_t) p->k * p->ncol_clusters;
    xq = work + h2b_mvm_work_doubles(p, 1);
  }
  if (p->cx)
    return single ? launch_pair<true, true>(p, q, x, y, ar, ai, br, bi, v, xq, st)
                  : launch_pair<true, false>(p, q, x, y, ar, ai, br, bi, v, xq, st);
  return single ? launch_pair<false, true>(p, q, x, y, ar, ai, br, bi, v, xq, st)
                : launch_pair<false, false>(p, q, x, y, ar, ai, br, bi, v, xq, st);
}

extern "C" size_t h2b_mvm_work_doubles(const MvmPlan *p, uint32_t nrhs) {
  const size_t W = p->cx ? 2 : 1;
  // the vectors and 8 doubles of slack after the last one (x slices are copied in 16-byte
  // aligned spans)
  return nrhs * W * ((size_t) p->ncol + p->nrow +
                     (size_t) p->k * (p->ncol_clusters + p->nrow_clusters)) + 8;
}

extern "C" int h2b_mvm_launch_batch(const MvmPlan *p, int single, uint32_t nrhs, const double *x,
                                    size_t ldx, double *y, size_t ldy, double ar, double ai,
                                    double *work, const uint32_t *mask, uint32_t nseg,
                                    cudaStream_t st) {
  if (single && !has_single(p)) {
    h2b_set_error("batched matvec: needs the FP32 copies (h2b_h2matrix_make_single)");
    return H2B_ERR_ARG;
  }
  if (nrhs == 0) {
    h2b_set_error("batched matvec: no columns");
    return H2B_ERR_ARG;
  }
  const size_t W = p->cx ? 2 : 1;
  MvmVecs v;
  v.sxp = W * p->ncol;
  v.syp = W * p->nrow;
  v.sxt = W * (size_t) p->k * p->ncol_clusters;
  v.syt = W * (size_t) p->k * p->nrow_clusters;
  v.xp = work;
  v.yp = v.xp + nrhs * v.sxp;
  v.xt = v.yp + nrhs * v.syp;
  v.yt = v.xt + nrhs * v.sxt;
  v.nrhs = nrhs;
  v.nseg = nseg;
  v.mask = mask;
  if (p->cx)
    return single ? launch_all<true, true>(p, x, ldx, y, ldy, ar, ai, v, st)
                  : launch_all<true, false>(p, x, ldx, y, ldy, ar, ai, v, st);
  return single ? launch_all<false, true>(p, x, ldx, y, ldy, ar, ai, v, st)
                : launch_all<false, false>(p, x, ldx, y, ldy, ar, ai, v, st);
}
