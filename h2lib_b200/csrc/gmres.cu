// Restarted GMRES with Householder QR on the device (sm_100a).
//
// Algorithm of init_gmres / step_gmres / finish_gmres (Library/krylov.c:612/659/725) and the
// driver solve_gmres_avector (Library/krylovsolvers.c:183): the Krylov basis is orthogonalised by
// Householder reflectors H_j = I - tau_j v_j v_j^H stored below the diagonal of the n x kmax
// matrix qr (v_j[j] = 1 implicit), the Hessenberg columns are reduced by Givens rotations and the
// transformed residual rhat gives the residual estimate |rhat_k|.
// The products of reflectors are applied in compact-WY form Q = H_0 ... H_j = I - V T V^H (T upper
// triangular, built column by column as in LAPACK's forward dlarft), so each application is two
// GEMV passes over V instead of j dependent dot/axpy pairs.  This is the same operator as the
// reference's sequential application; only the rounding order differs.
//
// All state (k, tau, T, rhat, scalars) lives on the device; kernels read the current dimension k
// from device memory, so the kernel sequence of one step is identical for every step and is
// captured once into a CUDA graph.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "device_common.cuh"
#include "gmres.h"

namespace {

constexpr int TPB = 256;

struct cd {
  double re, im;
};
__device__ __forceinline__ cd cmul(cd a, cd b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cd cconj(cd a) { return {a.re, -a.im}; }
__device__ __forceinline__ cd cadd(cd a, cd b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cd csub(cd a, cd b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ double cabs2(cd a) { return a.re * a.re + a.im * a.im; }
__device__ __forceinline__ cd cdivr(cd a, double r) { return {a.re / r, a.im / r}; }
__device__ __forceinline__ cd cdiv(cd a, cd b) {
  const double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}

template <bool CX> __device__ __forceinline__ cd ld(const double *p, size_t i) {
  return CX ? cd{p[2 * i], p[2 * i + 1]} : cd{p[i], 0.0};
}
template <bool CX> __device__ __forceinline__ void st(double *p, size_t i, cd v) {
  if (CX) {
    p[2 * i] = v.re;
    p[2 * i + 1] = v.im;
  } else {
    p[i] = v.re;
  }
}

__device__ __forceinline__ double block_sum(double v, double *red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    s = warp_sum(s);
  }
  return s;  // valid in warp 0
}

// element (i, j) of the reflector matrix V (unit lower trapezoidal)
template <bool CX>
__device__ __forceinline__ cd vij(const GmresDev &g, uint32_t i, uint32_t j) {
  if (i < j) return {0.0, 0.0};
  if (i == j) return {1.0, 0.0};
  return ld<CX>(g.qr, (size_t) i + (size_t) j * g.n);
}

// The new Krylov vector a = A q (in g.abuf) is moved into column k+1 of qr, and the partial sums
// part[b][j] = sum_{i in chunk b} conj(V[i,j]) a[i] (j <= k) of w = V_{0..k}^H a are formed.
template <bool CX>
__global__ void __launch_bounds__(TPB) vth_kernel(GmresDev g) {
  __shared__ double red[2][TPB / 32];
  const uint32_t k = g.state->k;
  const uint32_t ncols = k + 1;
  double *col = g.qr + (size_t) (CX ? 2 : 1) * (k + 1) * g.n;
  const uint32_t i = blockIdx.x * TPB + threadIdx.x;
  const bool in = i < g.n;
  const cd x = in ? ld<CX>(g.abuf, i) : cd{0.0, 0.0};
  if (in) st<CX>(col, i, x);
  for (uint32_t j = 0; j < ncols; j++) {
    cd p = {0.0, 0.0};
    if (in) p = cmul(cconj(vij<CX>(g, i, j)), x);
    const double sr = block_sum(p.re, red[0]);
    double si = 0.0;
    if (CX) si = block_sum(p.im, red[1]);
    if (threadIdx.x == 0) {
      g.part[(size_t) blockIdx.x * g.ldpart * 2 + 2 * j] = sr;
      g.part[(size_t) blockIdx.x * g.ldpart * 2 + 2 * j + 1] = si;
    }
  }
}

// a -= V u over rows (columns 0..k), then partial norm^2 of a[k+1..n)
template <bool CX>
__global__ void __launch_bounds__(TPB) apply_v_norm_kernel(GmresDev g) {
  __shared__ double red[TPB / 32];
  __shared__ double us[2 * GMRES_KMAX];
  const uint32_t k = g.state->k;
  for (uint32_t j = threadIdx.x; j <= k; j += TPB) {
    us[2 * j] = g.u[2 * j];
    us[2 * j + 1] = g.u[2 * j + 1];
  }
  __syncthreads();
  double *a = g.qr + (size_t) (CX ? 2 : 1) * (k + 1) * g.n;
  const uint32_t i = blockIdx.x * TPB + threadIdx.x;
  double nrm = 0.0;
  if (i < g.n) {
    cd ai = ld<CX>(a, i);
    const uint32_t jmax = i < k ? i : k;  // V[i, j] = 0 for j > i
    for (uint32_t j = 0; j <= jmax; j++)
      ai = csub(ai, cmul(vij<CX>(g, i, j), cd{us[2 * j], us[2 * j + 1]}));
    st<CX>(a, i, ai);
    if (i >= k + 1) nrm = cabs2(ai);
  }
  const double s = block_sum(nrm, red);
  if (threadIdx.x == 0) g.part[(size_t) blockIdx.x * g.ldpart * 2] = s;
}

// scale a[i > k+1] *= gamma, a[k+1] = alpha; partial z_j = sum_{i>k+1} conj(V[i,j]) a[i]
template <bool CX>
__global__ void __launch_bounds__(TPB) scale_vth_kernel(GmresDev g) {
  __shared__ double red[2][TPB / 32];
  const uint32_t k = g.state->k;
  const cd gamma = {g.state->gamma_re, g.state->gamma_im};
  double *a = g.qr + (size_t) (CX ? 2 : 1) * (k + 1) * g.n;
  const uint32_t i = blockIdx.x * TPB + threadIdx.x;
  cd x = {0.0, 0.0};
  if (i < g.n && i > k + 1) {
    x = cmul(ld<CX>(a, i), gamma);
    st<CX>(a, i, x);
  }
  if (i == k + 1) st<CX>(a, i, cd{g.state->alpha_re, g.state->alpha_im});
  for (uint32_t j = 0; j <= k; j++) {
    cd p = {0.0, 0.0};
    if (i < g.n && i > k + 1) p = cmul(cconj(vij<CX>(g, i, j)), x);
    const double sr = block_sum(p.re, red[0]);
    double si = 0.0;
    if (CX) si = block_sum(p.im, red[1]);
    if (threadIdx.x == 0) {
      g.part[(size_t) blockIdx.x * g.ldpart * 2 + 2 * j] = sr;
      g.part[(size_t) blockIdx.x * g.ldpart * 2 + 2 * j + 1] = si;
    }
  }
}

// q = e_{k} - V_{0..k} u  (k = current dimension after the step)
template <bool CX>
__global__ void __launch_bounds__(TPB) make_q_kernel(GmresDev g) {
  __shared__ double us[2 * GMRES_KMAX];
  const uint32_t k = g.state->k;
  for (uint32_t j = threadIdx.x; j <= k; j += TPB) {
    us[2 * j] = g.u[2 * j];
    us[2 * j + 1] = g.u[2 * j + 1];
  }
  __syncthreads();
  const uint32_t i = blockIdx.x * TPB + threadIdx.x;
  if (i >= g.n) return;
  cd q = {i == k ? 1.0 : 0.0, 0.0};
  const uint32_t jmax = i < k ? i : k;
  for (uint32_t j = 0; j <= jmax; j++) q = csub(q, cmul(vij<CX>(g, i, j), cd{us[2 * j], us[2 * j + 1]}));
  st<CX>(g.q, i, q);
}

__device__ cd sum_parts(const GmresDev &g, uint32_t j, uint32_t nb) {
  cd s = {0.0, 0.0};
  for (uint32_t b = 0; b < nb; b++) {
    s.re += g.part[(size_t) b * g.ldpart * 2 + 2 * j];
    s.im += g.part[(size_t) b * g.ldpart * 2 + 2 * j + 1];
  }
  return s;
}

__device__ __forceinline__ cd Tij(const GmresDev &g, uint32_t i, uint32_t j) {
  return {g.T[2 * ((size_t) i + (size_t) j * g.kmax)], g.T[2 * ((size_t) i + (size_t) j * g.kmax) + 1]};
}
__device__ __forceinline__ void setT(const GmresDev &g, uint32_t i, uint32_t j, cd v) {
  g.T[2 * ((size_t) i + (size_t) j * g.kmax)] = v.re;
  g.T[2 * ((size_t) i + (size_t) j * g.kmax) + 1] = v.im;
}

// Householder scalars of a column with entries diag (first) and squared norm norm2
// (qrdecomp_amatrix, Library/factorizations.c:2179).
__device__ void householder(cd diag, double norm2, GmresState *s, uint32_t col, const GmresDev &g) {
  const double norm = sqrt(norm2);
  if (norm2 <= 1e-300) {
    s->gamma_re = 1.0;
    s->gamma_im = 0.0;
    s->alpha_re = diag.re;
    s->alpha_im = diag.im;
    g.tau[2 * col] = 0.0;
    g.tau[2 * col + 1] = 0.0;
    return;
  }
  const double ad = sqrt(cabs2(diag));
  const cd sgn = ad == 0.0 ? cd{1.0, 0.0} : cdivr(diag, ad);
  const double adiag = ad + norm;
  double beta = 1.0 / (norm2 + ad * norm);
  beta *= adiag * adiag;
  const cd gamma = cdivr(cconj(sgn), adiag);
  s->gamma_re = gamma.re;
  s->gamma_im = gamma.im;
  s->alpha_re = -sgn.re * norm;
  s->alpha_im = -sgn.im * norm;
  g.tau[2 * col] = beta;
  g.tau[2 * col + 1] = 0.0;
}

// Givens rotations of Library/krylov.c:551 / :587 (complex form as in the reference).
__device__ cd findapply_givens(cd *a, cd *b) {
  const cd aa = *a, bb = *b;
  cd s, c, rho;
  if (cabs2(bb) < cabs2(aa)) {
    const cd t = cdiv(bb, aa);
    c = {1.0 / sqrt(cabs2(t) + 1.0), 0.0};
    s = cmul(t, c);
    rho = s;
  } else if (cabs2(aa) < cabs2(bb)) {
    const cd t = cdiv(aa, bb);
    s = {1.0 / sqrt(cabs2(t) + 1.0), 0.0};
    c = cmul(t, s);
    rho = cdiv(cd{1.0, 0.0}, c);
  } else {
    c = {1.0, 0.0};
    s = {0.0, 0.0};
    rho = {1.0, 0.0};
  }
  *a = cadd(cmul(c, aa), cmul(s, bb));
  *b = {0.0, 0.0};
  return rho;
}

__device__ void apply_givens(cd rho, cd *a, cd *b) {
  const cd aa = *a, bb = *b;
  cd s, c;
  if (cabs2(rho) < 1.0) {
    s = rho;
    c = {sqrt(1.0 - cabs2(s)), 0.0};
  } else if (cabs2(rho) > 1.0) {
    c = cdiv(cd{1.0, 0.0}, rho);
    s = {sqrt(1.0 - cabs2(c)), 0.0};
  } else {
    c = {1.0, 0.0};
    s = {0.0, 0.0};
  }
  *a = cadd(cmul(c, aa), cmul(s, bb));
  *b = csub(cmul(c, bb), cmul(s, aa));
}

// Bookkeeping kernels: one CTA of SMALL_THREADS threads (>= kmax); O(k) work per thread for the
// triangular products, sequential only where the algorithm is (Givens, triangular solve).
constexpr int SMALL_THREADS = GMRES_KMAX;

__device__ double block_sum_small(double v, double *red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < SMALL_THREADS / 32; w++) s += red[w];
  return s;  // valid in every thread
}

template <bool CX>
__global__ void __launch_bounds__(SMALL_THREADS) small_kernel(GmresDev g, int phase) {
  __shared__ double zr[GMRES_KMAX], zi[GMRES_KMAX], red[SMALL_THREADS / 32];
  GmresState *s = g.state;
  const uint32_t k = s->k;
  const uint32_t nb = g.nblocks;
  const uint32_t t = threadIdx.x;
  __syncthreads();  // every thread has read k before anyone may change it
  if (phase == 0) {
    // after vth: w = V^H a; u = T^H w
    if (t <= k) {
      cd w = sum_parts(g, t, nb);
      zr[t] = w.re;
      zi[t] = w.im;
      g.w[2 * t] = w.re;
      g.w[2 * t + 1] = w.im;
    }
    __syncthreads();
    if (t <= k) {
      cd u = {0.0, 0.0};
      for (uint32_t i = 0; i <= t; i++) u = cadd(u, cmul(cconj(Tij(g, i, t)), cd{zr[i], zi[i]}));
      g.u[2 * t] = u.re;
      g.u[2 * t + 1] = u.im;
    }
  } else if (phase == 1) {
    // after apply_v_norm: Householder scalars of column k+1, rows >= k+1
    double part = 0.0;
    for (uint32_t b = t; b < nb; b += SMALL_THREADS) part += g.part[(size_t) b * g.ldpart * 2];
    const double norm2 = block_sum_small(part, red);
    if (t == 0) {
      const double *a = g.qr + (size_t) (CX ? 2 : 1) * (k + 1) * g.n;
      householder(ld<CX>(a, k + 1), norm2, s, k + 1, g);
    }
  } else if (phase == 2) {
    // after scale_vth: T column k+1; u for q; Givens; k += 1
    const cd tau = {g.tau[2 * (k + 1)], g.tau[2 * (k + 1) + 1]};
    if (t <= k) {
      const cd z = cadd(sum_parts(g, t, nb), cconj(vij<CX>(g, k + 1, t)));  // + conj(v_t[k+1])
      zr[t] = z.re;
      zi[t] = z.im;
    }
    __syncthreads();
    if (t <= k) {
      cd acc = {0.0, 0.0};
      for (uint32_t j = t; j <= k; j++) acc = cadd(acc, cmul(Tij(g, t, j), cd{zr[j], zi[j]}));
      setT(g, t, k + 1, cmul(cd{-tau.re, -tau.im}, acc));
    }
    if (t == 0) setT(g, k + 1, k + 1, tau);
    __syncthreads();
    // u = T y, y_j = conj(V[k+1, j]) (j <= k), y_{k+1} = 1
    if (t <= k + 1) {
      cd acc = {0.0, 0.0};
      for (uint32_t j = t; j <= k + 1; j++) {
        const cd y = j == k + 1 ? cd{1.0, 0.0} : cconj(vij<CX>(g, k + 1, j));
        acc = cadd(acc, cmul(Tij(g, t, j), y));
      }
      g.u[2 * t] = acc.re;
      g.u[2 * t + 1] = acc.im;
    }
    if (t != 0) return;
    // Givens rotations on the new Hessenberg column (rows 0..k+1 of column k+1)
    double *col = g.qr + (size_t) (CX ? 2 : 1) * (k + 1) * g.n;
    for (uint32_t i = 0; i < k; i++) {
      const cd rho = ld<CX>(g.qr + (size_t) (CX ? 2 : 1) * (i + 1) * g.n, i + 1);
      cd a = ld<CX>(col, i), b = ld<CX>(col, i + 1);
      apply_givens(rho, &a, &b);
      st<CX>(col, i, a);
      st<CX>(col, i + 1, b);
    }
    cd a = ld<CX>(col, k), b = ld<CX>(col, k + 1);
    const cd rho = findapply_givens(&a, &b);
    st<CX>(col, k, a);
    st<CX>(col, k + 1, rho);
    cd r0 = {g.rhat[2 * k], g.rhat[2 * k + 1]}, r1 = {g.rhat[2 * (k + 1)], g.rhat[2 * (k + 1) + 1]};
    apply_givens(rho, &r0, &r1);
    g.rhat[2 * k] = r0.re;
    g.rhat[2 * k + 1] = r0.im;
    g.rhat[2 * (k + 1)] = r1.re;
    g.rhat[2 * (k + 1) + 1] = r1.im;
    s->k = k + 1;
    s->err = sqrt(cabs2(r1));
  } else if (phase == 3) {
    // finish: rhat_k = R^{-1} rhat_k (back substitution, row by row); z = V_k^H rhat;
    // u = T_k z
    if (t < k) {
      zr[t] = g.rhat[2 * t];
      zi[t] = g.rhat[2 * t + 1];
    }
    __syncthreads();
    for (uint32_t jj = k; jj-- > 0;) {
      if (t == 0) {
        const cd r = cdiv(cd{zr[jj], zi[jj]}, ld<CX>(g.qr + (size_t) (CX ? 2 : 1) * (jj + 1) * g.n, jj));
        zr[jj] = r.re;
        zi[jj] = r.im;
      }
      __syncthreads();
      // eliminate the solved unknown from the rows above (column jj+1 of R)
      if (t < jj) {
        const cd v = cmul(ld<CX>(g.qr + (size_t) (CX ? 2 : 1) * (jj + 1) * g.n, t), cd{zr[jj], zi[jj]});
        zr[t] -= v.re;
        zi[t] -= v.im;
      }
      __syncthreads();
    }
    if (t < k) {
      g.rhat[2 * t] = zr[t];
      g.rhat[2 * t + 1] = zi[t];
    }
    __shared__ double wr[GMRES_KMAX], wi[GMRES_KMAX];
    if (t < k) {
      cd acc = {zr[t], zi[t]};
      for (uint32_t i = t + 1; i < k; i++) acc = cadd(acc, cmul(cconj(vij<CX>(g, i, t)), cd{zr[i], zi[i]}));
      wr[t] = acc.re;
      wi[t] = acc.im;
    }
    __syncthreads();
    if (t < k) {
      cd acc = {0.0, 0.0};
      for (uint32_t j = t; j < k; j++) acc = cadd(acc, cmul(Tij(g, t, j), cd{wr[j], wi[j]}));
      g.u[2 * t] = acc.re;
      g.u[2 * t + 1] = acc.im;
    }
  } else if (phase == 4 || phase == 6) {
    // ||r||^2 (init, Householder of column 0) or ||b||^2, from part[b][0]
    double part = 0.0;
    for (uint32_t b = t; b < nb; b += SMALL_THREADS) part += g.part[(size_t) b * g.ldpart * 2];
    const double norm2 = block_sum_small(part, red);
    if (t == 0) {
      if (phase == 4)
        householder(ld<CX>(g.qr, 0), norm2, s, 0, g);
      else
        s->bnorm = sqrt(norm2);
    }
  } else if (phase == 5) {
    // init, after scaling column 0: T, rhat, k, err
    for (uint32_t i = t; i < 2 * (g.kmax + 1); i += SMALL_THREADS) g.rhat[i] = 0.0;
    __syncthreads();
    if (t == 0) {
      g.rhat[0] = s->alpha_re;
      g.rhat[1] = s->alpha_im;
      setT(g, 0, 0, cd{g.tau[0], g.tau[1]});
      s->k = 0;
      s->err = sqrt(s->alpha_re * s->alpha_re + s->alpha_im * s->alpha_im);
    }
  }
}

// x += rhat_(k) - V_k u (finish); vector kernels
template <bool CX>
__global__ void __launch_bounds__(TPB) update_x_kernel(GmresDev g, double *x) {
  __shared__ double us[2 * GMRES_KMAX];
  const uint32_t k = g.state->k;
  for (uint32_t j = threadIdx.x; j < k; j += TPB) {
    us[2 * j] = g.u[2 * j];
    us[2 * j + 1] = g.u[2 * j + 1];
  }
  __syncthreads();
  const uint32_t i = blockIdx.x * TPB + threadIdx.x;
  if (i >= g.n || k == 0) return;
  cd d = i < k ? cd{g.rhat[2 * i], g.rhat[2 * i + 1]} : cd{0.0, 0.0};
  const uint32_t jmax = i < k - 1 ? i : k - 1;
  for (uint32_t j = 0; j <= jmax; j++) d = csub(d, cmul(vij<CX>(g, i, j), cd{us[2 * j], us[2 * j + 1]}));
  st<CX>(x, i, cadd(ld<CX>(x, i), d));
}

// qr[:,0] = b; also partial ||b||^2 (for phase 6)
template <bool CX>
__global__ void __launch_bounds__(TPB) copy_b_kernel(GmresDev g, const double *b) {
  __shared__ double red[TPB / 32];
  const uint32_t i = blockIdx.x * TPB + threadIdx.x;
  double v = 0.0;
  if (i < g.n) {
    const cd bi = ld<CX>(b, i);
    st<CX>(g.qr, i, bi);
    v = cabs2(bi);
  }
  const double s = block_sum(v, red);
  if (threadIdx.x == 0) g.part[(size_t) blockIdx.x * g.ldpart * 2] = s;
}

// partial ||qr[:,0]||^2
template <bool CX>
__global__ void __launch_bounds__(TPB) norm0_kernel(GmresDev g) {
  __shared__ double red[TPB / 32];
  const uint32_t i = blockIdx.x * TPB + threadIdx.x;
  const double v = i < g.n ? cabs2(ld<CX>(g.qr, i)) : 0.0;
  const double s = block_sum(v, red);
  if (threadIdx.x == 0) g.part[(size_t) blockIdx.x * g.ldpart * 2] = s;
}

// column 0: scale rows > 0 by gamma, row 0 = alpha; q = H_0 e_0 = e_0 - tau_0 v_0
template <bool CX>
__global__ void __launch_bounds__(TPB) scale0_kernel(GmresDev g) {
  const uint32_t i = blockIdx.x * TPB + threadIdx.x;
  if (i >= g.n) return;
  const cd gamma = {g.state->gamma_re, g.state->gamma_im};
  const cd tau = {g.tau[0], g.tau[1]};
  if (i == 0) {
    st<CX>(g.qr, 0, cd{g.state->alpha_re, g.state->alpha_im});
    st<CX>(g.q, 0, csub(cd{1.0, 0.0}, tau));
  } else {
    const cd v = cmul(ld<CX>(g.qr, i), gamma);
    st<CX>(g.qr, i, v);
    st<CX>(g.q, i, cmul(cd{-tau.re, -tau.im}, v));
  }
}

template <bool CX>
int step_impl(const GmresDev &g, const GmresOp &op, cudaStream_t st) {
  const uint32_t nb = g.nblocks;
  // a = A q into the staging vector, then into column k+1 of qr (k is read on the device)
  H2B_CUDA_TRY(cudaMemsetAsync(g.abuf, 0, sizeof(double) * (CX ? 2 : 1) * g.n, st));
  int rc = op.apply(op.ctx, g.q, g.abuf, 1.0, 0.0, st);
  if (rc != H2B_OK) return rc;
  vth_kernel<CX><<<nb, TPB, 0, st>>>(g);
  small_kernel<CX><<<1, SMALL_THREADS, 0, st>>>(g, 0);
  apply_v_norm_kernel<CX><<<nb, TPB, 0, st>>>(g);
  small_kernel<CX><<<1, SMALL_THREADS, 0, st>>>(g, 1);
  scale_vth_kernel<CX><<<nb, TPB, 0, st>>>(g);
  small_kernel<CX><<<1, SMALL_THREADS, 0, st>>>(g, 2);
  make_q_kernel<CX><<<nb, TPB, 0, st>>>(g);
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

template <bool CX>
int init_impl(const GmresDev &g, const GmresOp &op, const double *b, double *x, cudaStream_t st) {
  const uint32_t nb = g.nblocks;
  copy_b_kernel<CX><<<nb, TPB, 0, st>>>(g, b);
  // qr[:,0] = b - A x
  int rc = op.apply(op.ctx, x, g.qr, -1.0, 0.0, st);
  if (rc != H2B_OK) return rc;
  norm0_kernel<CX><<<nb, TPB, 0, st>>>(g);
  small_kernel<CX><<<1, SMALL_THREADS, 0, st>>>(g, 4);
  scale0_kernel<CX><<<nb, TPB, 0, st>>>(g);
  small_kernel<CX><<<1, SMALL_THREADS, 0, st>>>(g, 5);
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

template <bool CX>
int finish_impl(const GmresDev &g, const GmresOp &op, const double *b, double *x,
                cudaStream_t st) {
  const uint32_t nb = g.nblocks;
  small_kernel<CX><<<1, SMALL_THREADS, 0, st>>>(g, 3);
  update_x_kernel<CX><<<nb, TPB, 0, st>>>(g, x);
  H2B_CUDA_TRY(cudaGetLastError());
  return init_impl<CX>(g, op, b, x, st);
}

template <bool CX>
int bnorm_impl(const GmresDev &g, const double *b, cudaStream_t st) {
  copy_b_kernel<CX><<<g.nblocks, TPB, 0, st>>>(g, b);
  small_kernel<CX><<<1, SMALL_THREADS, 0, st>>>(g, 6);
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

// Loop control of the graph-resident iteration (one thread each).
__global__ void precheck_kernel(GmresDev g, cudaGraphConditionalHandle hw) {
  const GmresState *s = g.state;
  const bool go = s->err > s->tol && (s->maxiter == 0 || s->iter + 1 != s->maxiter) &&
                  s->budget > 0 && !s->nan;
  cudaGraphSetConditional(hw, go ? 1u : 0u);
}

__global__ void decide_kernel(GmresDev g, cudaGraphConditionalHandle hi) {
  cudaGraphSetConditional(hi, g.state->k + 1 >= g.kmax ? 1u : 0u);
}

__global__ void control_kernel(GmresDev g, cudaGraphConditionalHandle hw) {
  GmresState *s = g.state;
  s->iter++;
  s->budget--;
  if (!(s->err == s->err)) s->nan = 1;
  const bool go = s->err > s->tol && (s->maxiter == 0 || s->iter + 1 != s->maxiter) &&
                  s->budget > 0 && !s->nan;
  cudaGraphSetConditional(hw, go ? 1u : 0u);
}

}  // namespace

extern "C" int h2b_gmres_loop_graph(const GmresDev *g, const GmresOp *op, const double *b,
                                    double *x, cudaStream_t st, cudaGraphExec_t *exec) {
  cudaGraph_t top = nullptr;
  *exec = nullptr;
  H2B_CUDA_TRY(cudaGraphCreate(&top, 0));
  struct GraphFree {
    cudaGraph_t gr;
    ~GraphFree() { cudaGraphDestroy(gr); }
  } gf{top};
  cudaGraphConditionalHandle hw, hi;
  H2B_CUDA_TRY(cudaGraphConditionalHandleCreate(&hw, top, 0, 0));
  GmresDev gv = *g;
  // top: precheck -> WHILE
  cudaGraphNode_t pre, wnode, dec, inode;
  {
    void *args[] = {&gv, &hw};
    cudaKernelNodeParams kp = {};
    kp.func = (void *) precheck_kernel;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = args;
    H2B_CUDA_TRY(cudaGraphAddKernelNode(&pre, top, nullptr, 0, &kp));
  }
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = hw;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  H2B_CUDA_TRY(cudaGraphAddNode(&wnode, top, &pre, 1, &wp));
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  // body: decide -> IF(restart) -> step -> control
  H2B_CUDA_TRY(cudaGraphConditionalHandleCreate(&hi, body, 0, 0));
  {
    void *args[] = {&gv, &hi};
    cudaKernelNodeParams kp = {};
    kp.func = (void *) decide_kernel;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = args;
    H2B_CUDA_TRY(cudaGraphAddKernelNode(&dec, body, nullptr, 0, &kp));
  }
  cudaGraphNodeParams ip = {};
  ip.type = cudaGraphNodeTypeConditional;
  ip.conditional.handle = hi;
  ip.conditional.type = cudaGraphCondTypeIf;
  ip.conditional.size = 1;
  H2B_CUDA_TRY(cudaGraphAddNode(&inode, body, &dec, 1, &ip));
  cudaGraph_t ifbody = ip.conditional.phGraph_out[0];
  int rc;
  H2B_CUDA_TRY(cudaStreamBeginCaptureToGraph(st, ifbody, nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal));
  rc = g->cx ? finish_impl<true>(*g, *op, b, x, st) : finish_impl<false>(*g, *op, b, x, st);
  cudaGraph_t captured = nullptr;
  cudaError_t ce = cudaStreamEndCapture(st, &captured);
  if (rc != H2B_OK) return rc;
  H2B_CUDA_TRY(ce);
  H2B_CUDA_TRY(cudaStreamBeginCaptureToGraph(st, body, &inode, nullptr, 1,
                                             cudaStreamCaptureModeThreadLocal));
  rc = g->cx ? step_impl<true>(*g, *op, st) : step_impl<false>(*g, *op, st);
  if (rc == H2B_OK) {
    control_kernel<<<1, 1, 0, st>>>(gv, hw);
    if (cudaGetLastError() != cudaSuccess) rc = H2B_ERR_CUDA;
  }
  ce = cudaStreamEndCapture(st, &captured);
  if (rc != H2B_OK) return rc;
  H2B_CUDA_TRY(ce);
  H2B_CUDA_TRY(cudaGraphInstantiate(exec, top, 0));
  return H2B_OK;
}

extern "C" int h2b_gmres_step(const GmresDev *g, const GmresOp *op, cudaStream_t st) {
  return g->cx ? step_impl<true>(*g, *op, st) : step_impl<false>(*g, *op, st);
}
extern "C" int h2b_gmres_init(const GmresDev *g, const GmresOp *op, const double *b, double *x,
                              cudaStream_t st) {
  return g->cx ? init_impl<true>(*g, *op, b, x, st) : init_impl<false>(*g, *op, b, x, st);
}
extern "C" int h2b_gmres_finish(const GmresDev *g, const GmresOp *op, const double *b, double *x,
                                cudaStream_t st) {
  return g->cx ? finish_impl<true>(*g, *op, b, x, st) : finish_impl<false>(*g, *op, b, x, st);
}
extern "C" int h2b_gmres_bnorm(const GmresDev *g, const double *b, cudaStream_t st) {
  return g->cx ? bnorm_impl<true>(*g, b, st) : bnorm_impl<false>(*g, b, st);
}
