// H2 matrix-vector product y += alpha A x on the device (sm_100a).
//
// Follows addeval_h2matrix_avector (Library/h2matrix.c:1269):
//   forward transform   xt_t = V_t^T x_t (leaves), xt_t = sum_s E_s^T xt_s (Library/clusterbasis.c:524)
//   coupling / near     yt_t += S_b xt_s,  y_t += N_b x_s      (fastaddeval, Library/h2matrix.c:1211)
//   backward transform  yt_s += E_s yt_t,  y_t += V_t yt_t     (Library/clusterbasis.c:749)
// Vectors are kept in cluster order (xp[i] = x[idx[i]]) so that every cluster's entries are
// contiguous.  The forward transform is one launch: a CTA per leaf, and the CTA that finishes
// the last son of a cluster continues with the father (an atomic arrival counter per cluster,
// reset by that CTA), so no CTA ever waits for another.  Coupling and nearfield blocks share one
// launch (a CTA per block, results added with FP64 atomics).  The backward transform runs level
// by level from the root; the leaf level adds V_t yt_t.  All kernels are memory-bound GEMVs:
// column-major panels are read with consecutive threads on consecutive rows.
// CX: complex coefficients (Helmholtz) — S, N, x, y complex (interleaved); V, E real.
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "h2mvm.h"

namespace {

template <bool CX> struct Val;
template <> struct Val<false> {
  double v;
  __device__ static Val zero() { return Val{0.0}; }
};
template <> struct Val<true> {
  double re, im;
  __device__ static Val zero() { return Val{0.0, 0.0}; }
};

__device__ __forceinline__ void vadd_atomic(double *p, const Val<false> &v) { atomicAdd(p, v.v); }
__device__ __forceinline__ void vadd_atomic(double *p, const Val<true> &v) {
  atomicAdd(p, v.re);
  atomicAdd(p + 1, v.im);
}

// xp = x[idx] (cluster order); clears nothing else
template <bool CX>
__global__ void gather_kernel(const double *__restrict__ x, const uint32_t *__restrict__ idx,
                              double *__restrict__ xp, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t j = idx[i];
    if (CX) {
      xp[2 * i] = x[2 * j];
      xp[2 * i + 1] = x[2 * j + 1];
    } else {
      xp[i] = x[j];
    }
  }
}

// y[idx[i]] += alpha * yp[i]
template <bool CX>
__global__ void scatter_kernel(const double *__restrict__ yp, const uint32_t *__restrict__ idx,
                               double *__restrict__ y, uint32_t n, double ar, double ai) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t j = idx[i];
    if (CX) {
      const double re = yp[2 * i], im = yp[2 * i + 1];
      y[2 * j] += ar * re - ai * im;
      y[2 * j + 1] += ar * im + ai * re;
    } else {
      y[j] += ar * yp[i];
    }
  }
}

// out[nu] = sum_i P[i + nu*rows] * v[i] for nu < k: warp per column, lanes over rows.
template <bool CX>
__device__ __forceinline__ void panel_tmv(const double *__restrict__ P, uint32_t rows, int k,
                                          const double *__restrict__ v, double *__restrict__ out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int nu = warp; nu < k; nu += nw) {
    const double *col = P + (size_t) nu * rows;
    double sr = 0.0, si = 0.0;
    for (uint32_t i = lane; i < rows; i += 32) {
      const double p = col[i];
      // v may have been written by another CTA of this launch: read through L2
      if (CX) {
        sr = fma(p, __ldcg(v + 2 * i), sr);
        si = fma(p, __ldcg(v + 2 * i + 1), si);
      } else {
        sr = fma(p, __ldcg(v + i), sr);
      }
    }
    sr = warp_sum(sr);
    if (CX) si = warp_sum(si);
    if (lane == 0) {
      if (CX) {
        out[2 * nu] = sr;
        out[2 * nu + 1] = si;
      } else {
        out[nu] = sr;
      }
    }
  }
}

template <bool CX>
__global__ void __launch_bounds__(256) forward_kernel(MvmForwardArgs a) {
  const int k = a.k;
  constexpr int W = CX ? 2 : 1;
  __shared__ double tmp[2 * 2 * 128];  // two sons' contributions (k <= 128, complex)
  __shared__ int last;
  uint32_t c = a.leaves[blockIdx.x];
  // leaf: xt_c = V_c^T xp[off .. off + size)
  panel_tmv<CX>(a.V + a.voff[c], a.size[c], k, a.xp + (size_t) W * a.off[c],
                a.xt + (size_t) W * k * c);
  // climb while this CTA completes the last son of the father
  while (true) {
    __syncthreads();
    const uint32_t f = a.father[c];
    if (f == UINT32_MAX) return;
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned old = atomicAdd(&a.counter[f], 1u);
      last = (old == 1u);
      if (last) a.counter[f] = 0u;  // reset for the next product
      __threadfence();
    }
    __syncthreads();
    if (!last) return;
    // xt_f = E_s0^T xt_s0 + E_s1^T xt_s1 (k x k transfers, column-major, rows = son points)
    const uint32_t s0 = a.son0[f], s1 = a.son1[f];
    panel_tmv<CX>(a.E + (size_t) (s0 - 1) * k * k, (uint32_t) k, k,
                  a.xt + (size_t) W * k * s0, tmp);
    panel_tmv<CX>(a.E + (size_t) (s1 - 1) * k * k, (uint32_t) k, k,
                  a.xt + (size_t) W * k * s1, tmp + W * k);
    __syncthreads();
    for (int e = threadIdx.x; e < W * k; e += blockDim.x)
      a.xt[(size_t) W * k * f + e] = tmp[e] + tmp[W * k + e];
    c = f;
  }
}

// y_rows += M x_cols for a column-major rows x cols panel M (ld = rows); atomics on the output.
template <bool CX>
__device__ __forceinline__ void panel_mv_atomic(const double *__restrict__ M, uint32_t rows,
                                                uint32_t cols, const double *__restrict__ xv,
                                                double *__restrict__ yv) {
  constexpr int W = CX ? 2 : 1;
  // threads: row r = t % rows_per, column group g = t / rows_per
  const uint32_t rb = rows < 64 ? rows : 64;   // rows per pass
  const uint32_t groups = blockDim.x / rb;
  for (uint32_t r0 = 0; r0 < rows; r0 += rb) {
    const uint32_t r = r0 + threadIdx.x % rb, g = threadIdx.x / rb;
    if (g < groups && r < rows) {
      double sr = 0.0, si = 0.0;
      for (uint32_t j = g; j < cols; j += groups) {
        const size_t e = (size_t) r + (size_t) j * rows;
        if (CX) {
          const double mr = M[2 * e], mi = M[2 * e + 1], xr = xv[2 * j], xi = xv[2 * j + 1];
          sr = fma(mr, xr, fma(-mi, xi, sr));
          si = fma(mr, xi, fma(mi, xr, si));
        } else {
          sr = fma(M[e], xv[j], sr);
        }
      }
      atomicAdd(&yv[W * r], sr);
      if (CX) atomicAdd(&yv[W * r + 1], si);
    }
  }
}

template <bool CX>
__global__ void __launch_bounds__(256) couple_near_kernel(MvmCoupleArgs a) {
  constexpr int W = CX ? 2 : 1;
  const uint32_t b = blockIdx.x;
  const uint32_t k = (uint32_t) a.k;
  if (b < a.nadm) {
    panel_mv_atomic<CX>(a.S + (size_t) W * k * k * b, k, k, a.xt + (size_t) W * k * a.adm_cc[b],
                        a.yt + (size_t) W * k * a.adm_rc[b]);
  } else {
    const uint32_t nb = b - a.nadm;
    const uint32_t r = a.near_rc[nb], c = a.near_cc[nb];
    panel_mv_atomic<CX>(a.N + (size_t) W * a.near_off[nb], a.rsize[r], a.csize[c],
                        a.xp + (size_t) W * a.coff[c], a.yp + (size_t) W * a.roff[r]);
  }
}

// yt_c += E_c yt_father(c) for the clusters of one level (E_c: k x k, rows = c's points).
template <bool CX>
__global__ void __launch_bounds__(256) downsweep_kernel(MvmDownArgs a) {
  constexpr int W = CX ? 2 : 1;
  const uint32_t c = a.clusters[blockIdx.x];
  const uint32_t f = a.father[c];
  const int k = a.k;
  __shared__ double yf[2 * 128];
  for (int e = threadIdx.x; e < W * k; e += blockDim.x) yf[e] = a.yt[(size_t) W * k * f + e];
  __syncthreads();
  const double *E = a.E + (size_t) (c - 1) * k * k;
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    double sr = 0.0, si = 0.0;
    for (int j = 0; j < k; j++) {
      const double e = E[i + (size_t) j * k];
      sr = fma(e, yf[W * j], sr);
      if (CX) si = fma(e, yf[W * j + 1], si);
    }
    a.yt[(size_t) W * k * c + W * i] += sr;
    if (CX) a.yt[(size_t) W * k * c + W * i + 1] += si;
  }
}

// yp[off + i] += sum_nu V_c[i, nu] yt_c[nu] for every row leaf.
template <bool CX>
__global__ void __launch_bounds__(256) backward_leaf_kernel(MvmBackArgs a) {
  constexpr int W = CX ? 2 : 1;
  const uint32_t c = a.leaves[blockIdx.x];
  const int k = a.k;
  const uint32_t rows = a.size[c];
  __shared__ double yc[2 * 128];
  for (int e = threadIdx.x; e < W * k; e += blockDim.x) yc[e] = a.yt[(size_t) W * k * c + e];
  __syncthreads();
  const double *V = a.V + a.voff[c];
  double *yp = a.yp + (size_t) W * a.off[c];
  for (uint32_t i = threadIdx.x; i < rows; i += blockDim.x) {
    double sr = 0.0, si = 0.0;
    for (int nu = 0; nu < k; nu++) {
      const double v = V[i + (size_t) nu * rows];
      sr = fma(v, yc[W * nu], sr);
      if (CX) si = fma(v, yc[W * nu + 1], si);
    }
    yp[W * i] += sr;
    if (CX) yp[W * i + 1] += si;
  }
}

}  // namespace

extern "C" int h2b_mvm_launch(const MvmPlan *p, const double *x, double *y, double ar, double ai,
                              cudaStream_t st) {
  const int cx = p->cx;
  const size_t W = cx ? 2 : 1;
  const int sms = p->num_sms > 0 ? p->num_sms : 148;
  H2B_CUDA_TRY(cudaMemsetAsync(p->yp, 0, sizeof(double) * W * p->nrow, st));
  H2B_CUDA_TRY(cudaMemsetAsync(p->yt, 0, sizeof(double) * W * p->k * p->nrow_clusters, st));
  const uint32_t gg = (p->ncol + 255) / 256 < (uint32_t) (4 * sms) ? (p->ncol + 255) / 256
                                                                   : (uint32_t) (4 * sms);
  MvmForwardArgs fa = p->fwd;
  MvmCoupleArgs ca = p->cpl;
  MvmBackArgs ba = p->bwd;
  if (cx) {
    gather_kernel<true><<<gg, 256, 0, st>>>(x, p->cidx, p->xp, p->ncol);
    forward_kernel<true><<<fa.nleaves, 256, 0, st>>>(fa);
    couple_near_kernel<true><<<ca.nadm + ca.nnear, 256, 0, st>>>(ca);
    for (uint32_t l = 1; l < p->rdepth; l++) {
      MvmDownArgs da = p->down;
      da.clusters = p->level_list + p->level_start[l];
      const uint32_t n = p->level_start[l + 1] - p->level_start[l];
      if (n) downsweep_kernel<true><<<n, 128, 0, st>>>(da);
    }
    backward_leaf_kernel<true><<<ba.nleaves, 128, 0, st>>>(ba);
    scatter_kernel<true><<<gg, 256, 0, st>>>(p->yp, p->ridx, y, p->nrow, ar, ai);
  } else {
    gather_kernel<false><<<gg, 256, 0, st>>>(x, p->cidx, p->xp, p->ncol);
    forward_kernel<false><<<fa.nleaves, 256, 0, st>>>(fa);
    couple_near_kernel<false><<<ca.nadm + ca.nnear, 256, 0, st>>>(ca);
    for (uint32_t l = 1; l < p->rdepth; l++) {
      MvmDownArgs da = p->down;
      da.clusters = p->level_list + p->level_start[l];
      const uint32_t n = p->level_start[l + 1] - p->level_start[l];
      if (n) downsweep_kernel<false><<<n, 128, 0, st>>>(da);
    }
    backward_leaf_kernel<false><<<ba.nleaves, 128, 0, st>>>(ba);
    scatter_kernel<false><<<gg, 256, 0, st>>>(p->yp, p->ridx, y, p->nrow, ar, ai);
  }
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}
