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
// Every product is a list of small dense GEMV work items (h2mvm.h: MvItem) in three launches:
//   1. forward + nearfield: xt_t += (W_t^T slice) x_slice, and y_r += N_b x_c;
//   2. coupling: yt_r += S_b xt_c;
//   3. backward: y_slice += (W_t^T slice)^T yt_t;
// between a gather (xp = x[idx], accumulators cleared) and a scatter (y[idx] += alpha yp).
// Vectors are kept in cluster order, so every item's x and y are contiguous slices.
//
// The item kernel is persistent (a few CTAs per SM, items taken round-robin) and streams each
// item's panel — a contiguous column-major block of N, S or W^T — into a ring of shared-memory
// stages with one bulk asynchronous copy (cp.async.bulk global -> shared, completion counted on
// an mbarrier per stage), so that several panels per SM are in flight while the GEMV of an
// earlier one runs from shared memory.  The copies are local to this GPU and have no cluster
// multicast.  Every wait on a stage is bounded: on time-out the kernel sets the plan's error
// flag, waits (bounded) for its copies in flight and returns.  Partial sums reach their outputs
// with FP64 atomics (an output row is shared by several items).
// CX: complex coefficients (Helmholtz) — S, N, x, y complex (interleaved); W real.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <type_traits>

#include "device_common.cuh"
#include "h2mvm.h"

namespace {

constexpr int TPB = 256;
constexpr int NWARP = TPB / 32;
constexpr int MAXROWS = 128;                 // rows of an untransposed item (k <= 125, 64-row tiles)
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
  const void *A[2];        // panel arrays: A[0] real; A[1] complex pairs when CX
  const double *X[2];      // x work vectors of the two triples
  double *Y[2];            // y work vectors
  size_t sx[2], sy[2];     // column strides (doubles)
  uint32_t nrhs, nseg;
  const uint32_t *mask;
  int *err;
  uint32_t stage_bytes;    // bytes per stage (multiple of 128)
  uint32_t stages;
  uint32_t red_doubles;    // cross-warp reduction buffer
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

// Panel of item m: first byte (16-byte aligned, at or before the panel) and byte count (a
// multiple of 16 that covers the panel).  The arrays carry 64 bytes of slack at their end.
template <bool CX, typename T>
__device__ __forceinline__ void panel_span(const MvLaunch &L, const MvItem &m, const char *&src,
                                           uint32_t &delta, uint32_t &bytes) {
  const int s = m.flags & H2B_MV_SRC1;
  const size_t esz = sizeof(T) * ((CX && s) ? 2 : 1);
  const char *addr = reinterpret_cast<const char *>(L.A[s]) + m.p * esz;
  src = reinterpret_cast<const char *>(reinterpret_cast<uintptr_t>(addr) & ~(uintptr_t) 15);
  delta = (uint32_t) (addr - src);
  bytes = (uint32_t) ((delta + (size_t) m.rows * m.cols * esz + 15) & ~(size_t) 15);
}

template <bool PCX, typename T>
__device__ __forceinline__ void entry(const T *P, size_t e, double &re, double &im) {
  if constexpr (PCX) {
    re = (double) P[2 * e];
    im = (double) P[2 * e + 1];
  } else {
    re = (double) P[e];
    im = 0.0;
  }
}

// y[0, R) += P x[0, C) from the panel in shared memory: warps take columns, lanes rows; the
// warps' partial sums meet in `red` and reach y with one atomic addition per row.
template <bool CX, bool PCX, typename T>
__device__ __forceinline__ void gemv_n(const T *P, uint32_t R, uint32_t C, const double *x,
                                       double *y, double *red) {
  constexpr int W = CX ? 2 : 1;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  double sr[MAXROWS / 32], si[MAXROWS / 32];
#pragma unroll
  for (int j = 0; j < MAXROWS / 32; j++) sr[j] = si[j] = 0.0;
#pragma unroll 2
  for (uint32_t c = warp; c < C; c += NWARP) {
    const double xr = __ldg(x + W * c), xi = CX ? __ldg(x + W * c + 1) : 0.0;
#pragma unroll
    for (int j = 0; j < MAXROWS / 32; j++) {
      const uint32_t r = lane + 32u * j;
      if (r < R) {
        double pr, pi;
        entry<PCX>(P, r + (size_t) c * R, pr, pi);
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
  for (int j = 0; j < MAXROWS / 32; j++) {
    const uint32_t r = lane + 32u * j;
    if (r < R) {
      red[W * (warp * R + r)] = sr[j];
      if (CX) red[W * (warp * R + r) + 1] = si[j];
    }
  }
  __syncthreads();
  for (uint32_t r = threadIdx.x; r < R; r += blockDim.x) {
    double ar = 0.0, ai = 0.0;
#pragma unroll
    for (int w = 0; w < NWARP; w++) {
      ar += red[W * (w * R + r)];
      if (CX) ai += red[W * (w * R + r) + 1];
    }
    atomicAdd(y + W * r, ar);
    if (CX) atomicAdd(y + W * r + 1, ai);
  }
  __syncthreads();  // red is reused
}

// y[0, C) += P^T x[0, R) for a real panel: a warp per column, lanes over the rows, shuffle sums.
template <bool CX, typename T>
__device__ __forceinline__ void gemv_t(const T *P, uint32_t R, uint32_t C, const double *x,
                                       double *y) {
  constexpr int W = CX ? 2 : 1;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  double xr[MAXROWS / 32], xi[MAXROWS / 32];
#pragma unroll
  for (int j = 0; j < MAXROWS / 32; j++) {
    const uint32_t r = lane + 32u * j;
    xr[j] = r < R ? __ldg(x + W * r) : 0.0;
    xi[j] = (CX && r < R) ? __ldg(x + W * r + 1) : 0.0;
  }
  for (uint32_t c = warp; c < C; c += NWARP) {
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int j = 0; j < MAXROWS / 32; j++) {
      const uint32_t r = lane + 32u * j;
      if (r < R) {
        const double p = (double) P[r + (size_t) c * R];
        sr = fma(p, xr[j], sr);
        if (CX) si = fma(p, xi[j], si);
      }
    }
    sr = warp_sum(sr);
    if (CX) si = warp_sum(si);
    if (lane == 0) {
      atomicAdd(y + W * c, sr);
      if (CX) atomicAdd(y + W * c + 1, si);
    }
  }
}

template <bool CX, typename T>
__global__ void __launch_bounds__(TPB) mv_items_kernel(MvLaunch L) {
  extern __shared__ __align__(128) unsigned char smem[];
  const uint32_t S = L.stages;
  unsigned char *stage0 = smem;
  double *red = reinterpret_cast<double *>(smem + (size_t) S * L.stage_bytes);
  uint64_t *bars = reinterpret_cast<uint64_t *>(red + L.red_doubles);
  // items of this CTA: blockIdx.x + i gridDim.x
  const uint32_t mine = L.n > blockIdx.x ? (L.n - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < S; s++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[s])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](uint32_t i) {  // thread 0: the copy of this CTA's i-th item into stage i % S
    const MvItem m = L.items[blockIdx.x + i * gridDim.x];
    const char *src;
    uint32_t delta, bytes;
    panel_span<CX, T>(L, m, src, delta, bytes);
    const uint32_t bar = smem_addr(&bars[i % S]);
    const uint32_t dst = smem_addr(stage0 + (size_t) (i % S) * L.stage_bytes);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
        : "memory");
  };
  if (threadIdx.x == 0)
    for (uint32_t i = 0; i < S && i < mine; i++) issue(i);

  for (uint32_t i = 0; i < mine; i++) {
    const uint32_t s = i % S;
    const bool ok = bar_wait(smem_addr(&bars[s]), (i / S) & 1u);
    if (__syncthreads_or(!ok)) {
      // a copy did not complete: flag it, wait (bounded) for the copies still in flight, stop
      if (threadIdx.x == 0) {
        atomicExch(L.err, 1);
        for (uint32_t j = i; j < i + S && j < mine; j++)
          bar_wait(smem_addr(&bars[j % S]), (j / S) & 1u);
      }
      return;
    }
    const MvItem m = L.items[blockIdx.x + i * gridDim.x];
    const char *src;
    uint32_t delta, bytes;
    panel_span<CX, T>(L, m, src, delta, bytes);
    const unsigned char *panel = stage0 + (size_t) s * L.stage_bytes + delta;
    const int t = m.flags & H2B_MV_SRC1;
    for (uint32_t q = 0; q < L.nrhs; q++) {
      if (!col_on(L.mask, L.nseg, m.seg, q)) continue;
      const double *x = L.X[t] + q * L.sx[t] + (size_t) (CX ? 2 : 1) * m.xo;
      double *y = L.Y[t] + q * L.sy[t] + (size_t) (CX ? 2 : 1) * m.yo;
      if (m.flags & H2B_MV_TRANS) {
        gemv_t<CX>(reinterpret_cast<const T *>(panel), m.rows, m.cols, x, y);
      } else if (CX && t) {
        gemv_n<CX, CX>(reinterpret_cast<const T *>(panel), m.rows, m.cols, x, y, red);
      } else {
        gemv_n<CX, false>(reinterpret_cast<const T *>(panel), m.rows, m.cols, x, y, red);
      }
    }
    __syncthreads();  // every thread is done with stage s
    if (threadIdx.x == 0 && i + S < mine) {
      // the generic-proxy reads of stage s are ordered before the async-proxy copy into it
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(i + S);
    }
  }
}

template <typename T>
uint32_t stage_bytes_of(const MvPhase &ph) {
  // the FP64 panel bytes scaled to the storage type, plus the alignment and rounding slack
  const size_t b = (size_t) ph.max_bytes * sizeof(T) / sizeof(double) + 32;
  return (uint32_t) ((b + 127) & ~(size_t) 127);
}

template <bool CX, typename T>
size_t smem_of(const MvPhase &ph, uint32_t stages) {
  const size_t red = (size_t) NWARP * std::max<uint32_t>(ph.max_rows, 1) * (CX ? 2 : 1);
  return (size_t) stages * stage_bytes_of<T>(ph) + sizeof(double) * red + 8 * stages;
}

template <bool CX, typename T>
int launch_phase(const MvmPlan *p, int phase, const MvLaunch &base, cudaStream_t st) {
  const MvPhase &ph = p->ph[phase];
  if (ph.n == 0) return H2B_OK;
  MvLaunch L = base;
  L.items = ph.items;
  L.n = ph.n;
  L.stages = (uint32_t) std::max(2, std::min(8, p->stages));
  L.stage_bytes = stage_bytes_of<T>(ph);
  L.red_doubles = (uint32_t) ((size_t) NWARP * std::max<uint32_t>(ph.max_rows, 1) * (CX ? 2 : 1));
  const size_t smem = smem_of<CX, T>(ph, L.stages);
  if (smem > H2B_MAX_DYN_SMEM || ph.max_rows > MAXROWS) {
    h2b_set_error("matvec: item panel of %u bytes / %u rows exceeds the kernel's limits",
                  ph.max_bytes, ph.max_rows);
    return H2B_ERR_ARG;
  }
  H2B_CUDA_TRY((h2b_allow_smem<mv_items_kernel<CX, T>>()));
  const int sms = p->num_sms > 0 ? p->num_sms : 148;
  const uint32_t grid = std::min<uint32_t>(ph.n, (uint32_t) (std::max(1, p->ctas_per_sm) * sms));
  mv_items_kernel<CX, T><<<grid, TPB, smem, st>>>(L);
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
  const void *Wc = SINGLE ? (const void *) p->fWc : (const void *) p->Wc;
  const void *Wr = SINGLE ? (const void *) p->fWr : (const void *) p->Wr;
  const void *N = SINGLE ? (const void *) p->fN : (const void *) p->N;
  const void *S = SINGLE ? (const void *) p->fS : (const void *) p->S;
  // 1: forward slices (W_c^T, xp -> xt) and nearfield blocks (N, xp -> yp)
  L.A[0] = Wc, L.X[0] = v.xp, L.Y[0] = v.xt, L.sx[0] = v.sxp, L.sy[0] = v.sxt;
  L.A[1] = N, L.X[1] = v.xp, L.Y[1] = v.yp, L.sx[1] = v.sxp, L.sy[1] = v.syp;
  int rc = launch_phase<CX, T>(p, 0, L, st);
  // 2: coupling blocks (S, xt -> yt)
  L.A[0] = nullptr, L.X[0] = nullptr, L.Y[0] = nullptr;
  L.A[1] = S, L.X[1] = v.xt, L.Y[1] = v.yt, L.sx[1] = v.sxt, L.sy[1] = v.syt;
  if (rc == H2B_OK) rc = launch_phase<CX, T>(p, 1, L, st);
  // 3: backward slices (W_r^T transposed, yt -> yp)
  L.A[0] = Wr, L.X[0] = v.yt, L.Y[0] = v.yp, L.sx[0] = v.syt, L.sy[0] = v.syp;
  L.A[1] = nullptr, L.X[1] = nullptr, L.Y[1] = nullptr;
  if (rc == H2B_OK) rc = launch_phase<CX, T>(p, 2, L, st);
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

}  // namespace

extern "C" int h2b_mvm_prepare(void) {
  H2B_CUDA_TRY((h2b_allow_smem<mv_items_kernel<false, double>>()));
  H2B_CUDA_TRY((h2b_allow_smem<mv_items_kernel<true, double>>()));
  H2B_CUDA_TRY((h2b_allow_smem<mv_items_kernel<false, float>>()));
  H2B_CUDA_TRY((h2b_allow_smem<mv_items_kernel<true, float>>()));
  return H2B_OK;
}

extern "C" size_t h2b_mvm_smem_bytes(const MvmPlan *p, int phase, int single, int stages) {
  const MvPhase &ph = p->ph[phase];
  if (p->cx)
    return single ? smem_of<true, float>(ph, stages) : smem_of<true, double>(ph, stages);
  return single ? smem_of<false, float>(ph, stages) : smem_of<false, double>(ph, stages);
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

extern "C" size_t h2b_mvm_work_doubles(const MvmPlan *p, uint32_t nrhs) {
  const size_t W = p->cx ? 2 : 1;
  return nrhs * W * ((size_t) p->ncol + p->nrow +
                     (size_t) p->k * (p->ncol_clusters + p->nrow_clusters));
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
