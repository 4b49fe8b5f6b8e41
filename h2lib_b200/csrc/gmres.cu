// Restarted GMRES with Householder QR on the device (sm_100a), for one system or a batch of
// independent systems.
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
// A batch holds nsys systems on disjoint row ranges of the global vectors (the block-diagonal
// operator of a forest H2 matrix, or one system per right-hand side): each system has its own
// qr, reflectors, Hessenberg data, residual estimate, restart and stopping decision, exactly as
// if it were solved alone; only the operator application is shared.  Vector kernels run one CTA
// per block of GMRES_TPB rows of one system; the bookkeeping kernel runs one CTA per system.
// All state lives on the device and kernels read it there, so the kernel sequence of one step
// is the same for every step and the whole iteration is one CUDA graph (h2b_gmres_loop_graph).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "device_common.cuh"
#include "gmres.h"

namespace {

constexpr int TPB = GMRES_TPB;

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

// The arrays of one system.
struct Sys {
  uint32_t n, nblk, s;
  double *qr, *tau, *T, *rhat, *w, *u, *q, *abuf, *part;
  GmresState *state;
};

template <bool CX>
__device__ __forceinline__ Sys sys_view(const GmresDev &g, uint32_t s) {
  constexpr size_t W = CX ? 2 : 1;
  const GmresSys y = g.sys[s];
  Sys v;
  v.n = y.n;
  v.nblk = y.nblk;
  v.s = s;
  v.qr = g.qr + W * y.qoff;
  v.tau = g.tau + 2 * (size_t) s * g.kmax;
  v.T = g.T + 2 * (size_t) s * g.kmax * g.kmax;
  v.rhat = g.rhat + 2 * (size_t) s * (g.kmax + 1);
  v.w = g.w + 2 * (size_t) s * (g.kmax + 1);
  v.u = g.u + 2 * (size_t) s * (g.kmax + 1);
  v.q = g.q + W * y.row0;
  v.abuf = g.abuf + W * y.row0;
  v.part = g.part + 2 * (size_t) y.blk0 * g.ldpart;
  v.state = g.state + s;
  return v;
}

__device__ __forceinline__ bool selected(const GmresState *s, int sel) {
  return sel == GMRES_SEL_ALL || (sel == GMRES_SEL_ACTIVE ? s->active != 0 : s->restart != 0);
}

// Vector kernels: CTA -> (system, local row i).  Returns false (uniformly per CTA) when the
// system is not selected.
template <bool CX>
__device__ __forceinline__ bool vec_view(const GmresDev &g, int sel, Sys &v, uint32_t &i,
                                         uint32_t &lb) {
  const uint32_t s = g.blk[blockIdx.x];
  v = sys_view<CX>(g, s);
  lb = blockIdx.x - g.sys[s].blk0;
  i = lb * TPB + threadIdx.x;
  return selected(v.state, sel);
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
__device__ __forceinline__ cd vij(const Sys &v, uint32_t i, uint32_t j) {
  if (i < j) return {0.0, 0.0};
  if (i == j) return {1.0, 0.0};
  return ld<CX>(v.qr, (size_t) i + (size_t) j * v.n);
}

__device__ __forceinline__ void put_part(const GmresDev &g, const Sys &v, uint32_t lb, uint32_t j,
                                         double re, double im) {
  v.part[(size_t) lb * g.ldpart * 2 + 2 * j] = re;
  v.part[(size_t) lb * g.ldpart * 2 + 2 * j + 1] = im;
}

// part[lb][j] = sum over this CTA's rows of pj(j), for j = 0..k: one warp reduction per j into
// shared memory and a single barrier, instead of a block-wide reduction (two barriers) per j.
template <bool CX, typename F>
__device__ __forceinline__ void block_dots(const GmresDev &g, const Sys &v, uint32_t lb,
                                           uint32_t k, F pj) {
  __shared__ double ws[2][TPB / 32][GMRES_KMAX + 1];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  // eight columns at a time: their loads are issued together and their eight shuffle trees
  // interleave, instead of one load and one dependent tree per column (each column's sum is
  // the same tree either way)
  constexpr uint32_t CH = 8;
  for (uint32_t j0 = 0; j0 <= k; j0 += CH) {
    cd p[CH];
#pragma unroll
    for (uint32_t u = 0; u < CH; u++) p[u] = j0 + u <= k ? pj(j0 + u) : cd{0.0, 0.0};
#pragma unroll
    for (uint32_t u = 0; u < CH; u++) {
      const double sr = warp_sum(p[u].re);
      const double si = CX ? warp_sum(p[u].im) : 0.0;
      if (lane == 0 && j0 + u <= k) {
        ws[0][w][j0 + u] = sr;
        ws[1][w][j0 + u] = si;
      }
    }
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j <= k; j += blockDim.x) {
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int q = 0; q < TPB / 32; q++) {
      sr += ws[0][q][j];
      si += ws[1][q][j];
    }
    put_part(g, v, lb, j, sr, si);
  }
}

// The new Krylov vector a = A q (in abuf) is moved into column k+1 of qr, and the partial sums
// part[b][j] = sum_{i in block b} conj(V[i,j]) a[i] (j <= k) of w = V_{0..k}^H a are formed.
template <bool CX>
__global__ void __launch_bounds__(TPB) vth_kernel(GmresDev g) {
  Sys v;
  uint32_t i, lb;
  if (!vec_view<CX>(g, GMRES_SEL_ACTIVE, v, i, lb)) return;
  const uint32_t k = v.state->k;
  double *col = v.qr + (size_t) (CX ? 2 : 1) * (k + 1) * v.n;
  const bool in = i < v.n;
  const cd x = in ? ld<CX>(v.abuf, i) : cd{0.0, 0.0};
  if (in) st<CX>(col, i, x);
  block_dots<CX>(g, v, lb, k, [&](uint32_t j) {
    return in ? cmul(cconj(vij<CX>(v, i, j)), x) : cd{0.0, 0.0};
  });
}

// a -= V u over rows (columns 0..k), then the partial sums of the next bookkeeping phase, in
// slots 0..k+1 of part: [0] ||a[k+1..n)||^2, [1 + j] sum_{i > k+1} conj(V[i,j]) a[i] (j <= k).  The
// second are the products of the previous reflectors with the next one (a below row k+1, scaled
// by the Householder factor gamma), taken before the scaling: gamma is a common factor of them,
// applied once the bookkeeping has computed it.
template <bool CX>
__global__ void __launch_bounds__(TPB) apply_v_dots_kernel(GmresDev g) {
  __shared__ double us[2 * GMRES_KMAX];
  Sys v;
  uint32_t i, lb;
  if (!vec_view<CX>(g, GMRES_SEL_ACTIVE, v, i, lb)) return;
  const uint32_t k = v.state->k;
  for (uint32_t j = threadIdx.x; j <= k; j += TPB) {
    us[2 * j] = v.u[2 * j];
    us[2 * j + 1] = v.u[2 * j + 1];
  }
  __syncthreads();
  double *a = v.qr + (size_t) (CX ? 2 : 1) * (k + 1) * v.n;
  cd ai = {0.0, 0.0};
  if (i < v.n) {
    ai = ld<CX>(a, i);
    const uint32_t jmax = i < k ? i : k;  // V[i, j] = 0 for j > i
    for (uint32_t j = 0; j <= jmax; j++)
      ai = csub(ai, cmul(vij<CX>(v, i, j), cd{us[2 * j], us[2 * j + 1]}));
    st<CX>(a, i, ai);
  }
  const bool below = i < v.n && i > k + 1;
  block_dots<CX>(g, v, lb, k + 1, [&](uint32_t j) {
    if (j == 0) return cd{(i < v.n && i >= k + 1) ? cabs2(ai) : 0.0, 0.0};
    return below ? cmul(cconj(vij<CX>(v, i, j - 1)), ai) : cd{0.0, 0.0};
  });
}

// After the bookkeeping of a step (k is the new dimension): the new reflector's rows below k are
// scaled by gamma (column k of qr; its row k holds the stored rotation), then q = e_k - V_{0..k} u.
// Each thread scales its own row before it reads it.
template <bool CX>
__global__ void __launch_bounds__(TPB) scale_make_q_kernel(GmresDev g) {
  __shared__ double us[2 * GMRES_KMAX];
  Sys v;
  uint32_t i, lb;
  if (!vec_view<CX>(g, GMRES_SEL_ACTIVE, v, i, lb)) return;
  const uint32_t k = v.state->k;
  const cd gamma = {v.state->gamma_re, v.state->gamma_im};
  for (uint32_t j = threadIdx.x; j <= k; j += TPB) {
    us[2 * j] = v.u[2 * j];
    us[2 * j + 1] = v.u[2 * j + 1];
  }
  __syncthreads();
  if (i >= v.n) return;
  if (i > k) {
    double *col = v.qr + (size_t) (CX ? 2 : 1) * k * v.n;
    st<CX>(col, i, cmul(ld<CX>(col, i), gamma));
  }
  cd q = {i == k ? 1.0 : 0.0, 0.0};
  const uint32_t jmax = i < k ? i : k;
  for (uint32_t j = 0; j <= jmax; j++) q = csub(q, cmul(vij<CX>(v, i, j), cd{us[2 * j], us[2 * j + 1]}));
  st<CX>(v.q, i, q);
}

// z[j] = sum over the system's blocks of part[b][j], j <= k.  Lanes take consecutive columns
// (coalesced reads of a block's partial sums), warps take interleaved blocks, so every thread has
// all its loads in flight at once; the warps' sums are combined in shared memory.  The caller
// synchronises before reading z.
__device__ void sum_parts_all(const GmresDev &g, const Sys &v, uint32_t k, double *zr,
                              double *zi, uint32_t j0 = 0) {
  constexpr int NW = GMRES_KMAX / 32;  // warps of the bookkeeping CTA (GMRES_KMAX threads)
  __shared__ double wsr[NW][GMRES_KMAX], wsi[NW][GMRES_KMAX];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint32_t j = lane; j <= k; j += 32) {
    double sr = 0.0, si = 0.0;
#pragma unroll 8
    for (uint32_t b = w; b < v.nblk; b += NW) {
      sr += v.part[(size_t) b * g.ldpart * 2 + 2 * (j0 + j)];
      si += v.part[(size_t) b * g.ldpart * 2 + 2 * (j0 + j) + 1];
    }
    wsr[w][j] = sr;
    wsi[w][j] = si;
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j <= k; j += blockDim.x) {
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int q = 0; q < NW; q++) {
      sr += wsr[q][j];
      si += wsi[q][j];
    }
    zr[j] = sr;
    zi[j] = si;
  }
}

__device__ __forceinline__ cd Tij(const GmresDev &g, const Sys &v, uint32_t i, uint32_t j) {
  return {v.T[2 * ((size_t) i + (size_t) j * g.kmax)], v.T[2 * ((size_t) i + (size_t) j * g.kmax) + 1]};
}
__device__ __forceinline__ void setT(const GmresDev &g, const Sys &v, uint32_t i, uint32_t j, cd x) {
  v.T[2 * ((size_t) i + (size_t) j * g.kmax)] = x.re;
  v.T[2 * ((size_t) i + (size_t) j * g.kmax) + 1] = x.im;
}

// Householder scalars of a column with entries diag (first) and squared norm norm2
// (qrdecomp_amatrix, Library/factorizations.c:2179).
__device__ void householder(cd diag, double norm2, GmresState *s, uint32_t col, const Sys &v) {
  const double norm = sqrt(norm2);
  if (norm2 <= 1e-300) {
    s->gamma_re = 1.0;
    s->gamma_im = 0.0;
    s->alpha_re = diag.re;
    s->alpha_im = diag.im;
    v.tau[2 * col] = 0.0;
    v.tau[2 * col + 1] = 0.0;
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
  v.tau[2 * col] = beta;
  v.tau[2 * col + 1] = 0.0;
}

// Givens rotations of Library/krylov.c:551 / :587.  A rotation is stored as one number rho:
// |rho| < 1: s = rho, c = sqrt(1 - |s|^2) real; |rho| > 1: c = 1 / rho, s = sqrt(1 - |c|^2) real.
// unitary = false is the reference's complex form, (a, b) -> (c a + s b, c b - s a) with
// s = c b / a (or c = s a / b): for complex entries that matrix is not unitary, so |rhat_k| is no
// longer the residual norm (for real entries both forms coincide).  unitary = true uses
// s = c conj(b / a) (or c = s conj(a / b)) and (a, b) -> (c a + s b, conj(c) b - conj(s) a),
// a unitary matrix that eliminates b the same way, so |rhat_k| stays the residual norm.
__device__ cd findapply_givens(cd *a, cd *b, bool unitary) {
  const cd aa = *a, bb = *b;
  cd s, c, rho;
  const double a2 = cabs2(aa), b2 = cabs2(bb);
  if (b2 < a2 || (unitary && b2 == a2 && a2 > 0.0)) {
    const cd t = cdiv(bb, aa);
    c = {1.0 / sqrt(cabs2(t) + 1.0), 0.0};
    s = cmul(unitary ? cconj(t) : t, c);
    rho = s;
  } else if (a2 < b2) {
    const cd t = cdiv(aa, bb);
    s = {1.0 / sqrt(cabs2(t) + 1.0), 0.0};
    c = cmul(unitary ? cconj(t) : t, s);
    rho = cdiv(cd{1.0, 0.0}, c);
  } else {
    c = {1.0, 0.0};
    s = {0.0, 0.0};
    rho = unitary ? cd{0.0, 0.0} : cd{1.0, 0.0};
  }
  *a = cadd(cmul(c, aa), cmul(s, bb));
  *b = {0.0, 0.0};
  return rho;
}

__device__ void apply_givens(cd rho, cd *a, cd *b, bool unitary) {
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
  *b = unitary ? csub(cmul(cconj(c), bb), cmul(cconj(s), aa)) : csub(cmul(c, bb), cmul(s, aa));
}

// Bookkeeping kernels: one CTA of SMALL_THREADS threads (>= kmax) per system; O(k) work per
// thread for the triangular products, sequential only where the algorithm is (Givens, triangular
// solve).
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
__global__ void __launch_bounds__(SMALL_THREADS) small_kernel(GmresDev g, int phase, int sel) {
  __shared__ double zr[GMRES_KMAX], zi[GMRES_KMAX], red[SMALL_THREADS / 32];
  __shared__ double wr[GMRES_KMAX], wi[GMRES_KMAX];
  __shared__ double hs[4];  // phase 1: gamma, alpha
  __shared__ double yr[GMRES_KMAX], yi[GMRES_KMAX];  // phase 1: conj(V[k+1, j])
  const Sys v = sys_view<CX>(g, blockIdx.x);
  GmresState *s = v.state;
  if (!selected(s, sel)) return;
  const uint32_t k = s->k;
  const uint32_t t = threadIdx.x;
  __syncthreads();  // every thread has read k before anyone may change it
  if (phase == 0) {
    // after vth: w = V^H a; u = T^H w
    sum_parts_all(g, v, k, zr, zi);
    __syncthreads();
    if (t <= k) {
      v.w[2 * t] = zr[t];
      v.w[2 * t + 1] = zi[t];
    }
    if (t <= k) {
      cd u = {0.0, 0.0};
      for (uint32_t i = 0; i <= t; i++) u = cadd(u, cmul(cconj(Tij(g, v, i, t)), cd{zr[i], zi[i]}));
      v.u[2 * t] = u.re;
      v.u[2 * t + 1] = u.im;
    }
  } else if (phase == 1) {
    // after apply_v_dots: the Householder scalars of column k+1 from ||a[k+1..n)||^2 (part slot
    // 0); the T column k+1 from the reflector products (part slots 1..k+1, times gamma); u for q;
    // the Givens rotations of the new Hessenberg column (entry k+1 = alpha); k += 1.
    {
      // y_j = conj(V[k+1, j]) (j <= k), read before anything waits on the Householder scalars
      if (t <= k) {
        const cd y = cconj(vij<CX>(v, k + 1, t));
        yr[t] = y.re;
        yi[t] = y.im;
      }
      double part = 0.0;
      for (uint32_t b = t; b < v.nblk; b += SMALL_THREADS)
        part += v.part[(size_t) b * g.ldpart * 2];
      const double norm2 = block_sum_small(part, red);
      if (t == 0) {
        const double *a = v.qr + (size_t) (CX ? 2 : 1) * (k + 1) * v.n;
        householder(k + 1 < v.n ? ld<CX>(a, k + 1) : cd{0.0, 0.0}, norm2, s, k + 1, v);
        hs[0] = s->gamma_re;
        hs[1] = s->gamma_im;
        hs[2] = s->alpha_re;
        hs[3] = s->alpha_im;
      }
      __syncthreads();
    }
    const cd tau = {v.tau[2 * (k + 1)], v.tau[2 * (k + 1) + 1]};
    sum_parts_all(g, v, k, zr, zi, 1u);
    __syncthreads();
    if (t <= k) {  // gamma z + conj(v_t[k+1])
      cd z = cmul(cd{zr[t], zi[t]}, cd{hs[0], hs[1]});
      z = cadd(z, cd{yr[t], yi[t]});
      zr[t] = z.re;
      zi[t] = z.im;
    }
    __syncthreads();
    // T column k+1: T[t, k+1] = -tau sum_{j=t..k} T[t, j] z_j, T[k+1, k+1] = tau; and
    // u = T y with y_{k+1} = 1: both sums run over row t of T in one pass
    if (t <= k) {
      cd acc = {0.0, 0.0}, uy = {0.0, 0.0};
#pragma unroll 4
      for (uint32_t j = t; j <= k; j++) {
        const cd tv = Tij(g, v, t, j);
        acc = cadd(acc, cmul(tv, cd{zr[j], zi[j]}));
        uy = cadd(uy, cmul(tv, cd{yr[j], yi[j]}));
      }
      const cd tn = cmul(cd{-tau.re, -tau.im}, acc);
      setT(g, v, t, k + 1, tn);
      uy = cadd(uy, tn);
      v.u[2 * t] = uy.re;
      v.u[2 * t + 1] = uy.im;
    } else if (t == k + 1) {
      setT(g, v, k + 1, k + 1, tau);
      v.u[2 * t] = tau.re;
      v.u[2 * t + 1] = tau.im;
    }
    // Givens rotations on the new Hessenberg column (rows 0..k+1 of column k+1): the column and
    // the stored rotations (diagonal of the previous columns) are staged in shared memory, so the
    // sequential sweep by one thread never waits on global memory.
    double *col = v.qr + (size_t) (CX ? 2 : 1) * (k + 1) * v.n;
    __syncthreads();  // zr / zi (read by the T loop above) are reused below
    if (t <= k + 1) {
      const cd c = t == k + 1 ? cd{hs[2], hs[3]} : ld<CX>(col, t);
      wr[t] = c.re;
      wi[t] = c.im;
    }
    if (t < k) {
      const cd r = ld<CX>(v.qr + (size_t) (CX ? 2 : 1) * (t + 1) * v.n, t + 1);
      zr[t] = r.re;
      zi[t] = r.im;
    }
    __syncthreads();
    if (t == 0) {
      for (uint32_t i = 0; i < k; i++) {
        cd a = {wr[i], wi[i]}, b = {wr[i + 1], wi[i + 1]};
        apply_givens(cd{zr[i], zi[i]}, &a, &b, g.unitary != 0);
        wr[i] = a.re;
        wi[i] = a.im;
        wr[i + 1] = b.re;
        wi[i + 1] = b.im;
      }
      cd a = {wr[k], wi[k]}, b = {wr[k + 1], wi[k + 1]};
      const cd rho = findapply_givens(&a, &b, g.unitary != 0);
      wr[k] = a.re;
      wi[k] = a.im;
      wr[k + 1] = rho.re;  // the rotation is stored below the diagonal
      wi[k + 1] = rho.im;
      cd r0 = {v.rhat[2 * k], v.rhat[2 * k + 1]},
         r1 = {v.rhat[2 * (k + 1)], v.rhat[2 * (k + 1) + 1]};
      apply_givens(rho, &r0, &r1, g.unitary != 0);
      v.rhat[2 * k] = r0.re;
      v.rhat[2 * k + 1] = r0.im;
      v.rhat[2 * (k + 1)] = r1.re;
      v.rhat[2 * (k + 1) + 1] = r1.im;
      s->k = k + 1;
      s->err = sqrt(cabs2(r1));
    }
    __syncthreads();
    if (t <= k + 1) st<CX>(col, t, cd{wr[t], wi[t]});
  } else if (phase == 3) {
    // finish: rhat_k = R^{-1} rhat_k (back substitution, row by row); z = V_k^H rhat;
    // u = T_k z
    if (t < k) {
      zr[t] = v.rhat[2 * t];
      zi[t] = v.rhat[2 * t + 1];
    }
    __syncthreads();
    for (uint32_t jj = k; jj-- > 0;) {
      if (t == 0) {
        const cd r = cdiv(cd{zr[jj], zi[jj]}, ld<CX>(v.qr + (size_t) (CX ? 2 : 1) * (jj + 1) * v.n, jj));
        zr[jj] = r.re;
        zi[jj] = r.im;
      }
      __syncthreads();
      // eliminate the solved unknown from the rows above (column jj+1 of R)
      if (t < jj) {
        const cd x = cmul(ld<CX>(v.qr + (size_t) (CX ? 2 : 1) * (jj + 1) * v.n, t), cd{zr[jj], zi[jj]});
        zr[t] -= x.re;
        zi[t] -= x.im;
      }
      __syncthreads();
    }
    if (t < k) {
      v.rhat[2 * t] = zr[t];
      v.rhat[2 * t + 1] = zi[t];
    }
    if (t < k) {
      cd acc = {zr[t], zi[t]};
      for (uint32_t i = t + 1; i < k; i++) acc = cadd(acc, cmul(cconj(vij<CX>(v, i, t)), cd{zr[i], zi[i]}));
      wr[t] = acc.re;
      wi[t] = acc.im;
    }
    __syncthreads();
    if (t < k) {
      cd acc = {0.0, 0.0};
      for (uint32_t j = t; j < k; j++) acc = cadd(acc, cmul(Tij(g, v, t, j), cd{wr[j], wi[j]}));
      v.u[2 * t] = acc.re;
      v.u[2 * t + 1] = acc.im;
    }
  } else if (phase == 4 || phase == 6) {
    // ||r||^2 (init, Householder of column 0) or ||b||^2, from part[b][0]
    double part = 0.0;
    for (uint32_t b = t; b < v.nblk; b += SMALL_THREADS) part += v.part[(size_t) b * g.ldpart * 2];
    const double norm2 = block_sum_small(part, red);
    if (t == 0) {
      if (phase == 4) {
        householder(ld<CX>(v.qr, 0), norm2, s, 0, v);
      } else {
        s->bnorm = sqrt(norm2);
        s->tol = g.eps * s->bnorm;
      }
    }
  } else if (phase == 5) {
    // init, after scaling column 0: T, rhat, k, err
    for (uint32_t i = t; i < 2 * (g.kmax + 1); i += SMALL_THREADS) v.rhat[i] = 0.0;
    __syncthreads();
    if (t == 0) {
      v.rhat[0] = s->alpha_re;
      v.rhat[1] = s->alpha_im;
      setT(g, v, 0, 0, cd{v.tau[0], v.tau[1]});
      s->k = 0;
      s->err = sqrt(s->alpha_re * s->alpha_re + s->alpha_im * s->alpha_im);
      // FP64: the reference steps after every restart.  Mixed: err is the FP64 residual of the
      // new start, an exact stopping test.
      s->active = g.mixed ? (s->err > s->tol ? 1u : 0u) : 1u;
      s->verify = 0;
    }
  }
}

// x += rhat_(k) - V_k u (finish); vector kernels
template <bool CX>
__global__ void __launch_bounds__(TPB) update_x_kernel(GmresDev g, double *x, int sel) {
  __shared__ double us[2 * GMRES_KMAX];
  Sys v;
  uint32_t i, lb;
  if (!vec_view<CX>(g, sel, v, i, lb)) return;
  const uint32_t k = v.state->k;
  for (uint32_t j = threadIdx.x; j < k; j += TPB) {
    us[2 * j] = v.u[2 * j];
    us[2 * j + 1] = v.u[2 * j + 1];
  }
  __syncthreads();
  if (i >= v.n || k == 0) return;
  double *xs = x + (size_t) (CX ? 2 : 1) * g.sys[v.s].row0;
  cd d = i < k ? cd{v.rhat[2 * i], v.rhat[2 * i + 1]} : cd{0.0, 0.0};
  const uint32_t jmax = i < k - 1 ? i : k - 1;
  for (uint32_t j = 0; j <= jmax; j++) d = csub(d, cmul(vij<CX>(v, i, j), cd{us[2 * j], us[2 * j + 1]}));
  st<CX>(xs, i, cadd(ld<CX>(xs, i), d));
}

// abuf = 0 over the whole vector
template <bool CX>
__global__ void __launch_bounds__(TPB) zero_abuf_kernel(GmresDev g) {
  const size_t n = (size_t) (CX ? 2 : 1) * g.n;
  for (size_t i = blockIdx.x * (size_t) TPB + threadIdx.x; i < n; i += (size_t) gridDim.x * TPB)
    g.abuf[i] = 0.0;
}

// partial ||b||^2 (for phase 6)
template <bool CX>
__global__ void __launch_bounds__(TPB) bnorm_kernel(GmresDev g, const double *b) {
  __shared__ double red[TPB / 32];
  Sys v;
  uint32_t i, lb;
  vec_view<CX>(g, GMRES_SEL_ALL, v, i, lb);
  const double *bs = b + (size_t) (CX ? 2 : 1) * g.sys[v.s].row0;
  const double x = i < v.n ? cabs2(ld<CX>(bs, i)) : 0.0;
  const double s = block_sum(x, red);
  if (threadIdx.x == 0) put_part(g, v, lb, 0, s, 0.0);
}

// qr[:,0] = b - A x (A x in abuf) and its partial norm^2
template <bool CX>
__global__ void __launch_bounds__(TPB) init0_kernel(GmresDev g, const double *b, int sel) {
  __shared__ double red[TPB / 32];
  Sys v;
  uint32_t i, lb;
  if (!vec_view<CX>(g, sel, v, i, lb)) return;
  const double *bs = b + (size_t) (CX ? 2 : 1) * g.sys[v.s].row0;
  double x = 0.0;
  if (i < v.n) {
    const cd r = csub(ld<CX>(bs, i), ld<CX>(v.abuf, i));
    st<CX>(v.qr, i, r);
    x = cabs2(r);
  }
  const double s = block_sum(x, red);
  if (threadIdx.x == 0) put_part(g, v, lb, 0, s, 0.0);
}

// column 0: scale rows > 0 by gamma, row 0 = alpha; q = H_0 e_0 = e_0 - tau_0 v_0
template <bool CX>
__global__ void __launch_bounds__(TPB) scale0_kernel(GmresDev g, int sel) {
  Sys v;
  uint32_t i, lb;
  if (!vec_view<CX>(g, sel, v, i, lb)) return;
  if (i >= v.n) return;
  const cd gamma = {v.state->gamma_re, v.state->gamma_im};
  const cd tau = {v.tau[0], v.tau[1]};
  if (i == 0) {
    st<CX>(v.qr, 0, cd{v.state->alpha_re, v.state->alpha_im});
    st<CX>(v.q, 0, csub(cd{1.0, 0.0}, tau));
  } else {
    const cd x = cmul(ld<CX>(v.qr, i), gamma);
    st<CX>(v.qr, i, x);
    st<CX>(v.q, i, cmul(cd{-tau.re, -tau.im}, x));
  }
}

template <bool CX>
int step_impl(const GmresDev &g, const GmresOp &op, cudaStream_t st) {
  const uint32_t nb = g.nblocks;
  // a = A q into the staging vector, then into column k+1 of qr (k is read on the device)
  zero_abuf_kernel<CX><<<nb, TPB, 0, st>>>(g);
  int rc = (op.apply_lo ? op.apply_lo : op.apply)(op.ctx, g.q, g.abuf, 1.0, 0.0, st);
  if (rc != H2B_OK) return rc;
  // w = V^H a; u = T^H w; a -= V u with the next column's norm and dot products; Householder
  // scalars, T column, Givens (k += 1); scaled reflector and q
  vth_kernel<CX><<<nb, TPB, 0, st>>>(g);
  small_kernel<CX><<<g.nsys, SMALL_THREADS, 0, st>>>(g, 0, GMRES_SEL_ACTIVE);
  apply_v_dots_kernel<CX><<<nb, TPB, 0, st>>>(g);
  small_kernel<CX><<<g.nsys, SMALL_THREADS, 0, st>>>(g, 1, GMRES_SEL_ACTIVE);
  scale_make_q_kernel<CX><<<nb, TPB, 0, st>>>(g);
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

template <bool CX>
int init_impl(const GmresDev &g, const GmresOp &op, const double *b, double *x, int sel,
              cudaStream_t st) {
  const uint32_t nb = g.nblocks;
  // qr[:,0] = b - A x
  zero_abuf_kernel<CX><<<nb, TPB, 0, st>>>(g);
  int rc = op.apply(op.ctx, x, g.abuf, 1.0, 0.0, st);
  if (rc != H2B_OK) return rc;
  init0_kernel<CX><<<nb, TPB, 0, st>>>(g, b, sel);
  small_kernel<CX><<<g.nsys, SMALL_THREADS, 0, st>>>(g, 4, sel);
  scale0_kernel<CX><<<nb, TPB, 0, st>>>(g, sel);
  small_kernel<CX><<<g.nsys, SMALL_THREADS, 0, st>>>(g, 5, sel);
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

template <bool CX>
int finish_only(const GmresDev &g, double *x, int sel, cudaStream_t st) {
  small_kernel<CX><<<g.nsys, SMALL_THREADS, 0, st>>>(g, 3, sel);
  update_x_kernel<CX><<<g.nblocks, TPB, 0, st>>>(g, x, sel);
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

template <bool CX>
int finish_impl(const GmresDev &g, const GmresOp &op, const double *b, double *x, int sel,
                cudaStream_t st) {
  int rc = finish_only<CX>(g, x, sel, st);
  if (rc != H2B_OK) return rc;
  return init_impl<CX>(g, op, b, x, sel, st);
}

template <bool CX>
int bnorm_impl(const GmresDev &g, const double *b, cudaStream_t st) {
  bnorm_kernel<CX><<<g.nblocks, TPB, 0, st>>>(g, b);
  small_kernel<CX><<<g.nsys, SMALL_THREADS, 0, st>>>(g, 6, GMRES_SEL_ALL);
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

// Loop control of the graph-resident iteration (one CTA each, threads stride over the systems).
__device__ __forceinline__ bool keeps_going(const GmresState *s, uint32_t maxiter) {
  return s->err > s->tol && (maxiter == 0 || s->iter + 1 != maxiter) && !s->nan;
}

__global__ void precheck_kernel(GmresDev g, cudaGraphConditionalHandle hw) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (uint32_t s = threadIdx.x; s < g.nsys; s += blockDim.x) {
    GmresState *y = g.state + s;
    y->active = keeps_going(y, g.ctl->maxiter) ? 1u : 0u;
    y->restart = 0;
    if (g.mask) g.mask[s] = y->active;
    if (y->active) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    g.ctl->any_active = any;
    cudaGraphSetConditional(hw, (any && g.ctl->budget > 0) ? 1u : 0u);
  }
}

__global__ void decide_kernel(GmresDev g, cudaGraphConditionalHandle hi) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (uint32_t s = threadIdx.x; s < g.nsys; s += blockDim.x) {
    GmresState *y = g.state + s;
    y->restart = (y->active && (y->k + 1 >= g.kmax || y->verify)) ? 1u : 0u;
    if (y->restart) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    g.ctl->any_restart = any;
    cudaGraphSetConditional(hi, any ? 1u : 0u);
  }
}

__global__ void control_kernel(GmresDev g, cudaGraphConditionalHandle hw) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (uint32_t s = threadIdx.x; s < g.nsys; s += blockDim.x) {
    GmresState *y = g.state + s;
    y->restart = 0;
    if (!y->active) {  // stopped earlier, or by the FP64 residual of a restart in this step
      if (g.mask) g.mask[s] = 0;
      continue;
    }
    y->iter++;
    if (!(y->err == y->err)) y->nan = 1;
    y->active = keeps_going(y, g.ctl->maxiter) ? 1u : 0u;
    // mixed precision: an estimate below tol is checked by a restart with the FP64 residual
    if (g.mixed && !y->active && !y->nan && !(y->err > y->tol) &&
        (g.ctl->maxiter == 0 || y->iter + 1 != g.ctl->maxiter)) {
      y->active = 1;
      y->verify = 1;
    }
    if (g.mask) g.mask[s] = y->active;
    if (y->active) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    g.ctl->budget--;
    g.ctl->any_active = any;
    cudaGraphSetConditional(hw, (any && g.ctl->budget > 0) ? 1u : 0u);
  }
}

constexpr int CTL_THREADS = 256;

int add_ctl_node(cudaGraphNode_t *node, cudaGraph_t graph, const cudaGraphNode_t *dep,
                 size_t ndep, void *func, GmresDev *g, cudaGraphConditionalHandle *h) {
  void *args[] = {g, h};
  cudaKernelNodeParams kp = {};
  kp.func = func;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(CTL_THREADS);
  kp.kernelParams = args;
  H2B_CUDA_TRY(cudaGraphAddKernelNode(node, graph, dep, ndep, &kp));
  return H2B_OK;
}

}  // namespace

size_t h2b_gmres_workspace(int cx, uint32_t nsys, const uint32_t *sizes, uint32_t kmax,
                           uint32_t *nblocks) {
  const size_t W = cx ? 2 : 1;
  uint64_t n = 0, nb = 0;
  for (uint32_t s = 0; s < nsys; s++) {
    n += sizes[s];
    nb += (sizes[s] + TPB - 1) / TPB;
  }
  if (nblocks) *nblocks = (uint32_t) nb;
  const size_t ld = kmax + 1;
  return W * n * kmax                       // qr
         + 2 * (size_t) nsys * kmax          // tau
         + 2 * (size_t) nsys * kmax * kmax   // T
         + 3 * 2 * (size_t) nsys * ld        // rhat, w, u
         + 2 * W * n                         // q, abuf
         + 2 * nb * ld                       // part
         + (sizeof(GmresState) * nsys + sizeof(GmresCtl) + sizeof(GmresSys) * nsys +
            sizeof(uint32_t) * (nb + nsys)) / sizeof(double) + 64;
}

void h2b_gmres_layout(GmresDev *g, double *p, int cx, uint32_t nsys, const uint32_t *sizes,
                      uint32_t kmax, GmresSys *sys_host, uint32_t *blk_host) {
  const size_t W = cx ? 2 : 1;
  uint64_t n = 0, q = 0;
  uint32_t nb = 0;
  for (uint32_t s = 0; s < nsys; s++) {
    sys_host[s].n = sizes[s];
    sys_host[s].row0 = (uint32_t) n;
    sys_host[s].qoff = q;
    sys_host[s].blk0 = nb;
    sys_host[s].nblk = (sizes[s] + TPB - 1) / TPB;
    for (uint32_t b = 0; b < sys_host[s].nblk; b++) blk_host[nb + b] = s;
    nb += sys_host[s].nblk;
    n += sizes[s];
    q += (uint64_t) sizes[s] * kmax;
  }
  const size_t ld = kmax + 1;
  g->cx = cx;
  g->nsys = nsys;
  g->n = (uint32_t) n;
  g->kmax = kmax;
  g->nblocks = nb;
  g->ldpart = (uint32_t) ld;
  g->qr = p; p += W * n * kmax;
  g->tau = p; p += 2 * (size_t) nsys * kmax;
  g->T = p; p += 2 * (size_t) nsys * kmax * kmax;
  g->rhat = p; p += 2 * (size_t) nsys * ld;
  g->w = p; p += 2 * (size_t) nsys * ld;
  g->u = p; p += 2 * (size_t) nsys * ld;
  g->q = p; p += W * n;
  g->abuf = p; p += W * n;
  g->part = p; p += 2 * (size_t) nb * ld;
  char *c = (char *) (((uintptr_t) p + 255) & ~(uintptr_t) 255);
  g->state = (GmresState *) c; c += sizeof(GmresState) * nsys;
  g->ctl = (GmresCtl *) c; c += sizeof(GmresCtl);
  c = (char *) (((uintptr_t) c + 15) & ~(uintptr_t) 15);
  g->sys = (const GmresSys *) c; c += sizeof(GmresSys) * nsys;
  g->blk = (const uint32_t *) c;
  g->mask = (uint32_t *) c + nb;
}

extern "C" int h2b_gmres_step(const GmresDev *g, const GmresOp *op, cudaStream_t st) {
  return g->cx ? step_impl<true>(*g, *op, st) : step_impl<false>(*g, *op, st);
}
extern "C" int h2b_gmres_init(const GmresDev *g, const GmresOp *op, const double *b, double *x,
                              int sel, cudaStream_t st) {
  return g->cx ? init_impl<true>(*g, *op, b, x, sel, st) : init_impl<false>(*g, *op, b, x, sel, st);
}
extern "C" int h2b_gmres_finish(const GmresDev *g, const GmresOp *op, const double *b, double *x,
                                int sel, cudaStream_t st) {
  return g->cx ? finish_impl<true>(*g, *op, b, x, sel, st)
               : finish_impl<false>(*g, *op, b, x, sel, st);
}
extern "C" int h2b_gmres_bnorm(const GmresDev *g, const double *b, cudaStream_t st) {
  return g->cx ? bnorm_impl<true>(*g, b, st) : bnorm_impl<false>(*g, b, st);
}

extern "C" int h2b_gmres_update(const GmresDev *g, double *x, int sel, cudaStream_t st) {
  return g->cx ? finish_only<true>(*g, x, sel, st) : finish_only<false>(*g, x, sel, st);
}

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
  int rc;
  // top: precheck -> WHILE
  cudaGraphNode_t pre, wnode, dec, inode;
  if ((rc = add_ctl_node(&pre, top, nullptr, 0, (void *) precheck_kernel, &gv, &hw)) != H2B_OK)
    return rc;
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = hw;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  H2B_CUDA_TRY(cudaGraphAddNode(&wnode, top, &pre, 1, &wp));
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  // body: decide -> IF(restart) -> step -> control
  H2B_CUDA_TRY(cudaGraphConditionalHandleCreate(&hi, body, 0, 0));
  if ((rc = add_ctl_node(&dec, body, nullptr, 0, (void *) decide_kernel, &gv, &hi)) != H2B_OK)
    return rc;
  cudaGraphNodeParams ip = {};
  ip.type = cudaGraphNodeTypeConditional;
  ip.conditional.handle = hi;
  ip.conditional.type = cudaGraphCondTypeIf;
  ip.conditional.size = 1;
  H2B_CUDA_TRY(cudaGraphAddNode(&inode, body, &dec, 1, &ip));
  cudaGraph_t ifbody = ip.conditional.phGraph_out[0];
  H2B_CUDA_TRY(cudaStreamBeginCaptureToGraph(st, ifbody, nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal));
  rc = g->cx ? finish_impl<true>(*g, *op, b, x, GMRES_SEL_RESTART, st)
             : finish_impl<false>(*g, *op, b, x, GMRES_SEL_RESTART, st);
  cudaGraph_t captured = nullptr;
  cudaError_t ce = cudaStreamEndCapture(st, &captured);
  if (rc != H2B_OK) return rc;
  H2B_CUDA_TRY(ce);
  H2B_CUDA_TRY(cudaStreamBeginCaptureToGraph(st, body, &inode, nullptr, 1,
                                             cudaStreamCaptureModeThreadLocal));
  rc = g->cx ? step_impl<true>(*g, *op, st) : step_impl<false>(*g, *op, st);
  if (rc == H2B_OK) {
    control_kernel<<<1, CTL_THREADS, 0, st>>>(gv, hw);
    if (cudaGetLastError() != cudaSuccess) rc = H2B_ERR_CUDA;
  }
  ce = cudaStreamEndCapture(st, &captured);
  if (rc != H2B_OK) return rc;
  H2B_CUDA_TRY(ce);
  H2B_CUDA_TRY(cudaGraphInstantiate(exec, top, 0));
  return H2B_OK;
}

extern "C" int h2b_gmres_run(const GmresDev *g, const GmresOp *op, const double *b, double *x,
                             uint32_t maxiter, cudaStream_t st, GmresState *host_state) {
  constexpr uint32_t kLoopBudget = 512;
  cudaGraphExec_t exec = nullptr;
  int rc = h2b_gmres_loop_graph(g, op, b, x, st, &exec);
  if (rc != H2B_OK) return rc;
  struct ExecFree {
    cudaGraphExec_t e;
    ~ExecFree() {
      if (e) cudaGraphExecDestroy(e);
    }
  } ef{exec};
  H2B_CUDA_TRY(cudaMemsetAsync(g->state, 0, sizeof(GmresState) * g->nsys, st));
  // the first residual needs every system's product
  H2B_CUDA_TRY(cudaMemsetAsync(g->mask, 1, sizeof(uint32_t) * g->nsys, st));
  H2B_CUDA_TRY(cudaMemsetAsync(g->T, 0, sizeof(double) * 2 * (size_t) g->nsys * g->kmax * g->kmax, st));
  if ((rc = h2b_gmres_bnorm(g, b, st)) != H2B_OK) return rc;
  if ((rc = h2b_gmres_init(g, op, b, x, GMRES_SEL_ALL, st)) != H2B_OK) return rc;
  GmresCtl ctl = {maxiter, kLoopBudget, 0, 0};
  while (true) {
    ctl.budget = kLoopBudget;
    H2B_CUDA_TRY(cudaMemcpyAsync(g->ctl, &ctl, sizeof(GmresCtl), cudaMemcpyHostToDevice, st));
    H2B_CUDA_TRY(cudaGraphLaunch(exec, st));
    GmresCtl out;
    H2B_CUDA_TRY(cudaMemcpyAsync(&out, g->ctl, sizeof(GmresCtl), cudaMemcpyDeviceToHost, st));
    H2B_CUDA_TRY(cudaStreamSynchronize(st));
    if (!out.any_active) break;
    if (out.budget != 0) {
      h2b_set_error("GMRES: device loop stopped with active systems and budget %u left",
                    out.budget);
      return H2B_ERR_INTERNAL;
    }
  }
  if ((rc = g->cx ? finish_only<true>(*g, x, GMRES_SEL_ALL, st)
                  : finish_only<false>(*g, x, GMRES_SEL_ALL, st)) != H2B_OK)
    return rc;
  if (host_state) {
    H2B_CUDA_TRY(cudaMemcpyAsync(host_state, g->state, sizeof(GmresState) * g->nsys,
                                 cudaMemcpyDeviceToHost, st));
  }
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  return H2B_OK;
}
