// H2 matrix-vector product y += alpha A x on the device (sm_100a).
//
// Follows addeval_h2matrix_avector (Library/h2matrix.c:1269):
//   forward transform   xt_t = V_t^T x_t (leaves), xt_t = sum_s E_s^T xt_s (Library/clusterbasis.c:524)
//   coupling / near     yt_t += S_b xt_s,  y_t += N_b x_s      (fastaddeval, Library/h2matrix.c:1211)
//   backward transform  yt_s += E_s yt_t,  y_t += V_t yt_t     (Library/clusterbasis.c:749)
// The nested transforms are multiplied out once after assembly (flatbasis.cu): for every cluster
// t of an admissible block, W_t = V_t (leaf) or [W_s E_s] over the sons s, the |t| x k basis on
// t's own indices.  The forward transform is then xt_t = W_t^T x_t and the backward transform
// y_t += W_t yt_t for every such cluster independently, with no dependence between levels.
// Vectors are kept in cluster order (xp[i] = x[idx[i]]) so that every cluster's entries are
// contiguous.  A product is five launches:
//   gather_zero   xp = x[idx], accumulators cleared;
//   forward+near  CTAs [0, items): xt_t += W_t[rows]^T x[rows] for one slice of rows of t;
//                 the other CTAs: y_r += N_b x_c for one nearfield block (independent of xt);
//   coupling      yt_r += S_b xt_c per admissible block;
//   backward      y[rows] += W_t[rows] yt_t per slice;
//   scatter       y[idx] += alpha yp.
// Partial sums reach their outputs with FP64 atomics.  The column side W^T is stored k x |t|
// (column-major), so the forward GEMVs read consecutive addresses with consecutive threads.
// CX: complex coefficients (Helmholtz) — S, N, x, y complex (interleaved); W real.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "device_common.cuh"
#include "h2mvm.h"

namespace {

constexpr int TPB = 256;
constexpr int KMAXW = 2 * 128;  // k <= 128 complex coefficients
// independent matrix loads in flight per thread in the GEMV loops
#ifndef H2B_MVM_UNROLL
#define H2B_MVM_UNROLL 8
#endif
constexpr int MVM_UNROLL = H2B_MVM_UNROLL;

// out[r] = sum_{c < ncols} P[r + c*ld] * v[c] for r < nrows (P column-major, real), v complex if
// CX.  Threads: r = t % nrows, group g = t / nrows takes the columns c = g mod G.  The result is
// written to `out` (shared or global) by the group-0 threads; `red` holds G * nrows * W doubles.
// All threads of the CTA must call it (it synchronises).  With VGLOBAL, `v` is a global array
// read through L2 (it may have been written by another CTA of the same launch); otherwise `v`
// is in shared memory.
template <bool CX, bool VGLOBAL, typename TP = double>
__device__ __forceinline__ void gemv_split(const TP *__restrict__ P, uint32_t ld,
                                           uint32_t nrows, uint32_t ncols,
                                           const double *__restrict__ v, double *red,
                                           double *out) {
  constexpr int W = CX ? 2 : 1;
  const uint32_t G = blockDim.x / nrows;
  const uint32_t t = threadIdx.x, r = t % nrows, g = t / nrows;
  double sr = 0.0, si = 0.0;
  if (g < G) {
#pragma unroll MVM_UNROLL
    for (uint32_t c = g; c < ncols; c += G) {
      const double p = (double) P[r + (size_t) c * ld];
      const double vr = VGLOBAL ? __ldcg(v + W * c) : v[W * c];
      sr = fma(p, vr, sr);
      if (CX) si = fma(p, VGLOBAL ? __ldcg(v + W * c + 1) : v[W * c + 1], si);
    }
    red[W * (g * nrows + r)] = sr;
    if (CX) red[W * (g * nrows + r) + 1] = si;
  }
  __syncthreads();
  if (t < nrows) {
    double ar = 0.0, ai = 0.0;
    for (uint32_t h = 0; h < G; h++) {
      ar += red[W * (h * nrows + t)];
      if (CX) ai += red[W * (h * nrows + t) + 1];
    }
    out[W * t] = ar;
    if (CX) out[W * t + 1] = ai;
  }
  __syncthreads();
}

// y_rows += M x_cols for a column-major rows x cols panel M (ld = rows, complex if CX).  The
// column groups' partial sums are combined in shared memory (`red`, blockDim * W doubles), so
// each output row receives one atomic addition per block.  All threads must call it.
template <bool CX, typename TM = double>
__device__ __forceinline__ void panel_mv_atomic(const TM *__restrict__ M, uint32_t rows,
                                                uint32_t cols, const double *__restrict__ xv,
                                                double *__restrict__ yv, double *red) {
  constexpr int W = CX ? 2 : 1;
  const uint32_t rb = rows < 64 ? rows : 64;  // rows per pass
  const uint32_t groups = blockDim.x / rb;
  for (uint32_t r0 = 0; r0 < rows; r0 += rb) {
    const uint32_t rl = threadIdx.x % rb, r = r0 + rl, g = threadIdx.x / rb;
    if (g < groups && r < rows) {
      double sr = 0.0, si = 0.0;
#pragma unroll MVM_UNROLL
      for (uint32_t j = g; j < cols; j += groups) {
        const size_t e = (size_t) r + (size_t) j * rows;
        if (CX) {
          const double mr = (double) M[2 * e], mi = (double) M[2 * e + 1], xr = xv[2 * j],
                       xi = xv[2 * j + 1];
          sr = fma(mr, xr, fma(-mi, xi, sr));
          si = fma(mr, xi, fma(mi, xr, si));
        } else {
          sr = fma((double) M[e], xv[j], sr);
        }
      }
      red[W * (g * rb + rl)] = sr;
      if (CX) red[W * (g * rb + rl) + 1] = si;
    }
    __syncthreads();
    if (threadIdx.x < rb && r0 + threadIdx.x < rows) {
      double ar = 0.0, ai = 0.0;
      for (uint32_t h = 0; h < groups; h++) {
        ar += red[W * (h * rb + threadIdx.x)];
        if (CX) ai += red[W * (h * rb + threadIdx.x) + 1];
      }
      atomicAdd(&yv[W * (r0 + threadIdx.x)], ar);
      if (CX) atomicAdd(&yv[W * (r0 + threadIdx.x) + 1], ai);
    }
    __syncthreads();
  }
}

// Flattened-basis path, for nrhs right-hand sides at once.  Every CTA loads its matrix panel
// once per column it multiplies; the columns after the first find the panel in L1/L2, so HBM
// reads the matrix about once per product of all columns.  With a mask (batched solves on a
// forest: mask[surface + r * nseg] for column r) a CTA skips the columns whose system is done.
struct MvmVecs {
  double *xp, *yp, *xt, *yt;      // work vectors, column r at r * stride
  size_t sxp, syp, sxt, syt;
  uint32_t nrhs, nseg;
  const uint32_t *mask;           // NULL: every column
  const uint32_t *rseg, *cseg;    // surface of each row / column cluster
};

__device__ __forceinline__ bool col_on(const MvmVecs &v, uint32_t seg, uint32_t r) {
  return !v.mask || v.mask[seg + r * v.nseg] != 0;
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

// Launch 1 (flat): xt_c += W_c^T x over rows [r0, r0 + nr) of c (CTAs < items; W_c^T is k x |c|,
// ld = k), and the nearfield blocks (the other CTAs).
template <bool CX, bool SINGLE = false>
__global__ void __launch_bounds__(TPB) forward_flat_near_kernel(MvmFlatArgs f, MvmCoupleArgs c,
                                                                MvmVecs v) {
  constexpr int W = CX ? 2 : 1;
  __shared__ double red[TPB * W];
  __shared__ double tmp[KMAXW];
  if (blockIdx.x >= f.nitems) {
    const uint32_t nb = blockIdx.x - f.nitems;
    const uint32_t r = c.near_rc[nb], cc = c.near_cc[nb];
    const uint32_t seg = v.rseg ? v.rseg[r] : 0;
    for (uint32_t q = 0; q < v.nrhs; q++) {
      if (!col_on(v, seg, q)) continue;
      const double *xp = v.xp + q * v.sxp + (size_t) W * c.coff[cc];
      double *yp = v.yp + q * v.syp + (size_t) W * c.roff[r];
      if (SINGLE)
        panel_mv_atomic<CX>(c.Ns + (size_t) W * c.near_off[nb], c.rsize[r], c.csize[cc], xp, yp,
                            red);
      else
        panel_mv_atomic<CX>(c.N + (size_t) W * c.near_off[nb], c.rsize[r], c.csize[cc], xp, yp,
                            red);
    }
    return;
  }
  const uint32_t *it = f.items + 3 * (size_t) blockIdx.x;
  const uint32_t cl = it[0], r0 = it[1], nr = it[2];
  const uint32_t k = (uint32_t) f.k;
  const uint32_t seg = v.cseg ? v.cseg[cl] : 0;
  for (uint32_t q = 0; q < v.nrhs; q++) {
    if (!col_on(v, seg, q)) continue;
    const double *xp = v.xp + q * v.sxp + (size_t) W * (f.off[cl] + r0);
    if (SINGLE)
      gemv_split<CX, false>(f.Ws + f.woff[cl] + (size_t) r0 * k, k, k, nr, xp, red, tmp);
    else
      gemv_split<CX, false>(f.W + f.woff[cl] + (size_t) r0 * k, k, k, nr, xp, red, tmp);
    double *xt = v.xt + q * v.sxt + (size_t) W * k * cl;
    for (uint32_t e = threadIdx.x; e < W * k; e += blockDim.x) atomicAdd(&xt[e], tmp[e]);
    __syncthreads();  // tmp is reused by the next column
  }
}

// Launch 2 (flat): coupling blocks yt_r += S_b xt_c per column.
template <bool CX, bool SINGLE>
__global__ void __launch_bounds__(TPB) coupling_flat_kernel(MvmCoupleArgs a, MvmVecs v) {
  constexpr int W = CX ? 2 : 1;
  __shared__ double red[TPB * W];
  const uint32_t b = blockIdx.x;
  const uint32_t k = (uint32_t) a.k;
  const uint32_t seg = v.rseg ? v.rseg[a.adm_rc[b]] : 0;
  for (uint32_t q = 0; q < v.nrhs; q++) {
    if (!col_on(v, seg, q)) continue;
    const double *xt = v.xt + q * v.sxt + (size_t) W * k * a.adm_cc[b];
    double *yt = v.yt + q * v.syt + (size_t) W * k * a.adm_rc[b];
    if (SINGLE)
      panel_mv_atomic<CX>(a.Ss + (size_t) W * k * k * b, k, k, xt, yt, red);
    else
      panel_mv_atomic<CX>(a.S + (size_t) W * k * k * b, k, k, xt, yt, red);
  }
}

// Launch 3 (flat): yp[rows r0 .. r0 + nr of c] += W_c[r0:, :] yt_c (W_c is |c| x k, ld = |c|).
template <bool CX, bool SINGLE = false>
__global__ void __launch_bounds__(TPB) backward_flat_kernel(MvmFlatArgs f, MvmVecs v) {
  constexpr int W = CX ? 2 : 1;
  __shared__ double red[TPB * W];
  __shared__ double tmp[H2B_MVM_FLAT_ROWS * W];
  const uint32_t *it = f.items + 3 * (size_t) blockIdx.x;
  const uint32_t cl = it[0], r0 = it[1], nr = it[2];
  const uint32_t k = (uint32_t) f.k;
  const uint32_t seg = v.rseg ? v.rseg[cl] : 0;
  for (uint32_t q = 0; q < v.nrhs; q++) {
    if (!col_on(v, seg, q)) continue;
    const double *yt = v.yt + q * v.syt + (size_t) W * k * cl;
    if (SINGLE)
      gemv_split<CX, false>(f.Ws + f.woff[cl] + r0, f.size[cl], nr, k, yt, red, tmp);
    else
      gemv_split<CX, false>(f.W + f.woff[cl] + r0, f.size[cl], nr, k, yt, red, tmp);
    double *y = v.yp + q * v.syp + (size_t) W * (f.off[cl] + r0);
    for (uint32_t e = threadIdx.x; e < W * nr; e += blockDim.x) atomicAdd(&y[e], tmp[e]);
    __syncthreads();  // tmp is reused by the next column
  }
}

// ------------------------------------------------------------------------------------------
// Warp-per-item variant of the three flattened-path launches (used for the FP32 copies).  Every
// work item is a small dense GEMV y_rows += P x_cols (a coupling block, a nearfield block, or a
// slice of a flattened basis) and one warp does it alone: lane l owns rows l, l + 32, ... (WG_R
// per pass) and walks the columns with WG_U columns' loads in flight; each row's sum reaches its
// output with one atomic addition.  No shared memory and no barriers, and a panel serves up to
// WG_Q right-hand sides per read (the others are re-read from L2).
// ------------------------------------------------------------------------------------------
#ifndef H2B_MVM_WARP
#define H2B_MVM_WARP 1
#endif
// resident CTAs per SM the warp kernels are compiled for (register budget 65536 / (256 * this))
#ifndef H2B_MVM_WARP_MINB
#define H2B_MVM_WARP_MINB 1
#endif
constexpr int WG_R = 4;  // rows per lane per pass (128 rows)
constexpr int WG_U = 4;  // columns unrolled (loads in flight per row)
constexpr int WG_Q = 4;  // right-hand sides per pass

// One matrix entry, widened to FP64: (re, im) of P[e] (complex P interleaved).
template <bool PCX, typename TP>
__device__ __forceinline__ void load_entry(const TP *__restrict__ P, size_t e, double &re,
                                           double &im) {
  if constexpr (PCX) {
    if constexpr (sizeof(TP) == 8) {
      const double2 t = __ldg(reinterpret_cast<const double2 *>(P) + e);
      re = t.x;
      im = t.y;
    } else {
      const float2 t = __ldg(reinterpret_cast<const float2 *>(P) + e);
      re = (double) t.x;
      im = (double) t.y;
    }
  } else {
    re = (double) __ldg(P + e);
    im = 0.0;
  }
}

// y_q[rows] += P x_q for the nq (<= NQ) right-hand sides given, P column-major (ld), real or
// complex (PCX); x, y complex when CX.  Called by all lanes of one warp.
template <bool CX, bool PCX, int NQ, typename TP>
__device__ __forceinline__ void warp_gemv(const TP *__restrict__ P, uint32_t ld, uint32_t nrows,
                                          uint32_t ncols, const double *const (&xq)[NQ],
                                          double *const (&yq)[NQ], int nq) {
  constexpr int WV = CX ? 2 : 1;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t r0 = 0; r0 < nrows; r0 += 32 * WG_R) {
    double sr[NQ][WG_R], si[NQ][WG_R];
#pragma unroll
    for (int q = 0; q < NQ; q++)
#pragma unroll
      for (int i = 0; i < WG_R; i++) sr[q][i] = si[q][i] = 0.0;
#pragma unroll WG_U
    for (uint32_t c = 0; c < ncols; c++) {
      double xr[NQ], xi[NQ];
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        xr[q] = q < nq ? __ldg(xq[q] + WV * c) : 0.0;
        xi[q] = (CX && q < nq) ? __ldg(xq[q] + WV * c + 1) : 0.0;
      }
#pragma unroll
      for (int i = 0; i < WG_R; i++) {
        const uint32_t r = r0 + lane + 32u * i;
        if (r < nrows) {
          double pr, pi;
          load_entry<PCX>(P, (size_t) r + (size_t) c * ld, pr, pi);
#pragma unroll
          for (int q = 0; q < NQ; q++) {
            if (PCX) {
              sr[q][i] = fma(pr, xr[q], fma(-pi, xi[q], sr[q][i]));
              si[q][i] = fma(pr, xi[q], fma(pi, xr[q], si[q][i]));
            } else {
              sr[q][i] = fma(pr, xr[q], sr[q][i]);
              if (CX) si[q][i] = fma(pr, xi[q], si[q][i]);
            }
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < WG_R; i++) {
      const uint32_t r = r0 + lane + 32u * i;
      if (r < nrows) {
#pragma unroll
        for (int q = 0; q < NQ; q++) {
          if (q < nq) {
            atomicAdd(yq[q] + WV * r, sr[q][i]);
            if (CX) atomicAdd(yq[q] + WV * r + 1, si[q][i]);
          }
        }
      }
    }
  }
}

// The item's work, applied to the unmasked right-hand sides in groups of NQ.  off_x / off_y:
// offsets (in doubles) of the item's vector slices inside one column of the x / y work vector.
template <bool CX, bool PCX, int NQ, typename TP>
__device__ __forceinline__ void warp_item(const TP *__restrict__ P, uint32_t ld, uint32_t nrows,
                                          uint32_t ncols, const MvmVecs &v, uint32_t seg,
                                          const double *x0, size_t sx, double *y0, size_t sy) {
  for (uint32_t q0 = 0; q0 < v.nrhs; q0 += NQ) {
    const double *xq[NQ];
    double *yq[NQ];
    int nq = 0;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      xq[q] = x0;
      yq[q] = y0;
    }
    for (uint32_t q = q0; q < v.nrhs && q < q0 + NQ; q++)
      if (col_on(v, seg, q)) {
        // (nq < NQ: at most NQ columns per group)
#pragma unroll
        for (int s = 0; s < NQ; s++)
          if (s == nq) {
            xq[s] = x0 + q * sx;
            yq[s] = y0 + q * sy;
          }
        nq++;
      }
    if (nq > 0) warp_gemv<CX, PCX, NQ>(P, ld, nrows, ncols, xq, yq, nq);
  }
}

// Launch 1: forward items xt_c += W_c^T x[rows r0 .. r0 + nr of c] (W_c^T: k x |c|, ld k) and
// the nearfield blocks yp_r += N_b xp_c, one warp each.
template <bool CX, bool SINGLE, int NQ>
__global__ void __launch_bounds__(TPB, H2B_MVM_WARP_MINB) forward_near_warp_kernel(MvmFlatArgs f, MvmCoupleArgs c,
                                                                MvmVecs v) {
  constexpr int W = CX ? 2 : 1;
  const uint32_t item = blockIdx.x * (TPB / 32) + (threadIdx.x >> 5);
  if (item < f.nitems) {
    const uint32_t *it = f.items + 3 * (size_t) item;
    const uint32_t cl = it[0], r0 = it[1], nr = it[2];
    const uint32_t k = (uint32_t) f.k;
    const uint32_t seg = v.cseg ? v.cseg[cl] : 0;
    const double *x0 = v.xp + (size_t) W * (f.off[cl] + r0);
    double *y0 = v.xt + (size_t) W * k * cl;
    if (SINGLE)
      warp_item<CX, false, NQ>(f.Ws + f.woff[cl] + (size_t) r0 * k, k, k, nr, v, seg, x0, v.sxp,
                               y0, v.sxt);
    else
      warp_item<CX, false, NQ>(f.W + f.woff[cl] + (size_t) r0 * k, k, k, nr, v, seg, x0, v.sxp,
                               y0, v.sxt);
  } else if (item < f.nitems + c.nnear) {
    const uint32_t nb = item - f.nitems;
    const uint32_t r = c.near_rc[nb], cc = c.near_cc[nb];
    const uint32_t seg = v.rseg ? v.rseg[r] : 0;
    const uint32_t rows = c.rsize[r];
    const double *x0 = v.xp + (size_t) W * c.coff[cc];
    double *y0 = v.yp + (size_t) W * c.roff[r];
    if (SINGLE)
      warp_item<CX, CX, NQ>(c.Ns + (size_t) W * c.near_off[nb], rows, rows, c.csize[cc], v, seg,
                            x0, v.sxp, y0, v.syp);
    else
      warp_item<CX, CX, NQ>(c.N + (size_t) W * c.near_off[nb], rows, rows, c.csize[cc], v, seg,
                            x0, v.sxp, y0, v.syp);
  }
}

// Launch 2: coupling blocks yt_r += S_b xt_c, one warp each.
template <bool CX, bool SINGLE, int NQ>
__global__ void __launch_bounds__(TPB, H2B_MVM_WARP_MINB) coupling_warp_kernel(MvmCoupleArgs a, MvmVecs v) {
  constexpr int W = CX ? 2 : 1;
  const uint32_t b = blockIdx.x * (TPB / 32) + (threadIdx.x >> 5);
  if (b >= a.nadm) return;
  const uint32_t k = (uint32_t) a.k;
  const uint32_t seg = v.rseg ? v.rseg[a.adm_rc[b]] : 0;
  const double *x0 = v.xt + (size_t) W * k * a.adm_cc[b];
  double *y0 = v.yt + (size_t) W * k * a.adm_rc[b];
  if (SINGLE)
    warp_item<CX, CX, NQ>(a.Ss + (size_t) W * k * k * b, k, k, k, v, seg, x0, v.sxt, y0, v.syt);
  else
    warp_item<CX, CX, NQ>(a.S + (size_t) W * k * k * b, k, k, k, v, seg, x0, v.sxt, y0, v.syt);
}

// Launch 3: backward items yp[rows r0 .. r0 + nr of c] += W_c[r0:, :] yt_c (W_c: |c| x k,
// ld |c|), one warp each.
template <bool CX, bool SINGLE, int NQ>
__global__ void __launch_bounds__(TPB, H2B_MVM_WARP_MINB) backward_warp_kernel(MvmFlatArgs f, MvmVecs v) {
  constexpr int W = CX ? 2 : 1;
  const uint32_t item = blockIdx.x * (TPB / 32) + (threadIdx.x >> 5);
  if (item >= f.nitems) return;
  const uint32_t *it = f.items + 3 * (size_t) item;
  const uint32_t cl = it[0], r0 = it[1], nr = it[2];
  const uint32_t k = (uint32_t) f.k;
  const uint32_t seg = v.rseg ? v.rseg[cl] : 0;
  const double *x0 = v.yt + (size_t) W * k * cl;
  double *y0 = v.yp + (size_t) W * (f.off[cl] + r0);
  if (SINGLE)
    warp_item<CX, false, NQ>(f.Ws + f.woff[cl] + r0, f.size[cl], nr, k, v, seg, x0, v.syt, y0,
                             v.syp);
  else
    warp_item<CX, false, NQ>(f.W + f.woff[cl] + r0, f.size[cl], nr, k, v, seg, x0, v.syt, y0,
                             v.syp);
}

template <bool CX, bool SINGLE, int NQ>
void launch_warp_items(const MvmPlan *p, const MvmVecs &v, cudaStream_t st) {
  constexpr uint32_t WPB = TPB / 32;
  const MvmCoupleArgs &ca = p->cpl;
  const uint32_t n1 = p->ffwd.nitems + ca.nnear;
  if (n1) {
    forward_near_warp_kernel<CX, SINGLE, NQ><<<(n1 + WPB - 1) / WPB, TPB, 0, st>>>(p->ffwd, ca, v);
    h2b_note_launch();
  }
  if (ca.nadm) {
    coupling_warp_kernel<CX, SINGLE, NQ><<<(ca.nadm + WPB - 1) / WPB, TPB, 0, st>>>(ca, v);
    h2b_note_launch();
  }
  if (p->fbwd.nitems) {
    backward_warp_kernel<CX, SINGLE, NQ><<<(p->fbwd.nitems + WPB - 1) / WPB, TPB, 0, st>>>(p->fbwd, v);
    h2b_note_launch();
  }
}

template <bool CX, bool SINGLE>
int launch_flat(const MvmPlan *p, const double *x, size_t ldx, double *y, size_t ldy, double ar,
                double ai, const MvmVecs &v, cudaStream_t st) {
  const size_t W = CX ? 2 : 1;
  const int sms = p->num_sms > 0 ? p->num_sms : 148;
  const MvmCoupleArgs &ca = p->cpl;
  const uint32_t zn = p->nrow > p->ncol ? p->nrow : p->ncol;
  const uint32_t gz = std::min<uint32_t>((zn + 255) / 256 + 1, (uint32_t) (4 * sms));
  const size_t nyp = W * p->nrow, nxt = W * (size_t) p->k * p->ncol_clusters,
               nyt = W * (size_t) p->k * p->nrow_clusters;
  gather_zero_kernel<CX><<<gz, 256, 0, st>>>(x, ldx, p->cidx, p->ncol, v, nyp, nxt, nyt);
  h2b_note_launch();
  // FP32-stored products run one warp per item (measured faster); FP64 ones one CTA per item
  // (measured faster: the warp form's registers halve its occupancy for 8-byte entries)
  if (H2B_MVM_WARP && SINGLE) {
    if (v.nrhs == 1)
      launch_warp_items<CX, SINGLE, 1>(p, v, st);
    else
      launch_warp_items<CX, SINGLE, WG_Q>(p, v, st);
  } else {
    if (p->ffwd.nitems + ca.nnear) {
      forward_flat_near_kernel<CX, SINGLE><<<p->ffwd.nitems + ca.nnear, TPB, 0, st>>>(p->ffwd,
                                                                                       ca, v);
      h2b_note_launch();
    }
    if (ca.nadm) {
      coupling_flat_kernel<CX, SINGLE><<<ca.nadm, TPB, 0, st>>>(ca, v);
      h2b_note_launch();
    }
    if (p->fbwd.nitems) {
      backward_flat_kernel<CX, SINGLE><<<p->fbwd.nitems, TPB, 0, st>>>(p->fbwd, v);
      h2b_note_launch();
    }
  }
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
  v.rseg = v.cseg = nullptr;
  return v;
}

}  // namespace

extern "C" int h2b_mvm_launch_single(const MvmPlan *p, const double *x, double *y, double ar,
                                     double ai, cudaStream_t st) {
  if (!p->cpl.Ss || !p->cpl.Ns || !p->ffwd.Ws || !p->fbwd.Ws) {
    h2b_set_error("matvec: no FP32 copy of the H2 matrix (h2b_h2matrix_make_single)");
    return H2B_ERR_ARG;
  }
  if (p->k > 128) {
    h2b_set_error("matvec: rank %d > 128", p->k);
    return H2B_ERR_ARG;
  }
  const MvmVecs v = plan_vecs(p);
  return p->cx ? launch_flat<true, true>(p, x, 0, y, 0, ar, ai, v, st)
               : launch_flat<false, true>(p, x, 0, y, 0, ar, ai, v, st);
}

extern "C" int h2b_mvm_launch(const MvmPlan *p, const double *x, double *y, double ar, double ai,
                              cudaStream_t st) {
  if (p->k > 128) {
    h2b_set_error("matvec: rank %d > 128", p->k);
    return H2B_ERR_ARG;
  }
  const MvmVecs v = plan_vecs(p);
  return p->cx ? launch_flat<true, false>(p, x, 0, y, 0, ar, ai, v, st)
               : launch_flat<false, false>(p, x, 0, y, 0, ar, ai, v, st);
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
  if (single && (!p->cpl.Ss || !p->cpl.Ns || !p->ffwd.Ws || !p->fbwd.Ws)) {
    h2b_set_error("batched matvec: needs the FP32 copies (h2b_h2matrix_make_single)");
    return H2B_ERR_ARG;
  }
  if (p->k > 128 || nrhs == 0) {
    h2b_set_error("batched matvec: rank %d > 128 or no columns", p->k);
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
  v.rseg = mask ? p->rseg : nullptr;
  v.cseg = mask ? p->cseg : nullptr;
  if (mask && (!p->rseg || !p->cseg)) {
    h2b_set_error("batched matvec: masking needs the surface of every cluster");
    return H2B_ERR_ARG;
  }
  if (p->cx)
    return single ? launch_flat<true, true>(p, x, ldx, y, ldy, ar, ai, v, st)
                  : launch_flat<true, false>(p, x, ldx, y, ldy, ar, ai, v, st);
  return single ? launch_flat<false, true>(p, x, ldx, y, ldy, ar, ai, v, st)
                : launch_flat<false, false>(p, x, ldx, y, ldy, ar, ai, v, st);
}
