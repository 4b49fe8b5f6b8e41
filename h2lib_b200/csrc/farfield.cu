// Farfield fill kernels of the Chebyshev-interpolation H2 matrix (sm_100a, FP64).
//
//   leaf bases      V_t[i, nu] = int phi_i L_nu   (or the normal derivative d/dn L_nu for the
//                   double-layer column basis), q^2-point rule per triangle:
//                   assemble_bem3d_lagrange_{c,l}_amatrix, Library/bem3d.c:7616/7758 and
//                   assemble_bem3d_dn_lagrange_{c,l}_amatrix, :8024/8200;
//   transfers       E_s[i, nu] = L^father_nu(xi^son_i):  assemble_bem3d_lagrange_amatrix, :8497;
//   coupling        S_b[i, j] = (1/4pi) g(xi^row_i, xi^col_j):  assemble_bem3d_inter_uniform,
//                   :6079 -> fill_bem3d, :3439.
// Interpolation points per cluster are the tensor Chebyshev nodes of its bounding box widened to
// at least 2 * 5e-3 per axis (assemble_interpoints3d_realavector, :5236); the host computes the
// m one-dimensional nodes per axis and cluster (pts[c][axis][mu]).  The multi-index
// nu = (jx * m + jy) * m + jz orders the tensor basis as the reference does.
// The bases are real for both Laplace and (non-directional) Helmholtz; the coupling matrices
// are complex for Helmholtz.  One CTA per leaf / cluster / admissible block.
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "farfield.h"

namespace {

constexpr int MMAX = 8;

// Lagrange polynomial mu of nodes xi[0..m) at x as wbar_mu prod_{l != mu} (x - xi_l), with the
// barycentric weight wbar_mu = 1 / prod_{l != mu} (xi_mu - xi_l) computed once per node set,
// and its derivative wbar_mu sum_{l != mu} prod_{l2 != mu, l} (x - xi_l2): the same polynomials
// as lagrange_1d (and its derivative) without a division per evaluation.
__device__ __forceinline__ double lagr_bar(double x, const double *xi, double wbar, int mu, int m) {
  double v = wbar;
  for (int l = 0; l < m; l++)
    if (l != mu) v *= x - xi[l];
  return v;
}

__device__ __forceinline__ double dlagr_bar(double x, const double *xi, double wbar, int mu,
                                            int m) {
  double s = 0.0;
  for (int l = 0; l < m; l++) {
    if (l == mu) continue;
    double tmp = 1.0;
    for (int l2 = 0; l2 < m; l2++)
      if (l2 != mu && l2 != l) tmp *= x - xi[l2];
    s += tmp;
  }
  return wbar * s;
}

// Leaf bases.  Rows of leaf c: its triangles (constant basis) or vertices (linear basis).  A
// leaf's nu range is split over a.split CTAs (CTA (leaf, part) computes the columns
// [part k / split, ...)), so that the launch has several CTAs per SM.  The CTA's triangle
// list (TriRef, local row indices) is processed in batches of BATCH triangles: first the
// one-dimensional Lagrange values (and derivatives) at every quadrature point of the batch are
// tabulated in shared memory (3 axes x M), then each thread, which owns one nu of the CTA's range
// for the whole launch (its three one-dimensional indices formed once), takes the batch's
// triangles in turn and forms the tensor products from the table.  The interpolation order M is
// a template parameter, so no index arithmetic divides at run time.  The CTA's columns of V
// (rows x its nu) are accumulated in shared memory (atomics for the linear basis, where a vertex
// receives the integrals of all triangles around it) and written once.
constexpr int BATCH = 32;
constexpr int NSMAX = 64;   // single-triangle rule points (q^2, q <= 8)

template <bool LINEAR, bool DN, int M>
__global__ void __launch_bounds__(256) leaf_basis_kernel(FarLeafArgs a) {
  constexpr int K = M * M * M;
  extern __shared__ double smem[];
  __shared__ double wbar[3][M];
  const uint32_t split = (uint32_t) a.split;
  const uint32_t leaf = blockIdx.x / split, part = blockIdx.x % split;
  const uint32_t c = a.leaves[leaf];
  const int nu0 = (int) ((part * (uint32_t) K) / split);
  const int nu1 = (int) (((part + 1) * (uint32_t) K) / split);
  const int kp = nu1 - nu0;
  const uint32_t rows = a.size[c];
  const uint32_t tr0 = a.tr_off[leaf], ntr = a.tr_len[leaf];
  const double *pts = a.pts + (size_t) c * 3 * M;
  const int ns = a.ns;
  const int kpmax = (K + (int) split - 1) / (int) split;
  double *V = smem;                                   // rows * kp (the CTA's columns)
  double *tab = V + (size_t) rows * kpmax;            // BATCH * ns * 3 * M
  double *dtab = tab + (size_t) BATCH * ns * 3 * M;   // same size (derivatives, DN only)
  for (uint32_t e = threadIdx.x; e < rows * (uint32_t) kp; e += blockDim.x) V[e] = 0.0;
  if (threadIdx.x < 3u * M) {
    const int d = (int) threadIdx.x / M, mu = (int) threadIdx.x % M;
    const double *xi = pts + d * M;
    double p = 1.0;
    for (int l = 0; l < M; l++)
      if (l != mu) p *= xi[mu] - xi[l];
    wbar[d][mu] = 1.0 / p;
  }

  // the rule's weights, and per batch the triangles' vertices, normals, Gram determinants and
  // local rows, are staged in shared memory (the loops below then read no global memory)
  __shared__ double sw[4][NSMAX];          // rows 0..2 linear-basis weighted, 3 raw
  __shared__ double sx[NSMAX], sy[NSMAX];
  __shared__ double tv[BATCH][9], tn[BATCH][3], tg[BATCH];
  __shared__ int tl[BATCH][3];
  for (int q = (int) threadIdx.x; q < ns; q += (int) blockDim.x) {
    sx[q] = a.xs[q];
    sy[q] = a.ys[q];
    sw[3][q] = a.ws[q];
    if (LINEAR)
      for (int l = 0; l < 3; l++) sw[l][q] = a.wsl[l * ns + q];
  }
  // this thread's column: lnu = threadIdx.x % kp, triangles threadIdx.x / kp + g * tstep
  const int tstep = (int) blockDim.x / kp;
  const int lnu = (int) threadIdx.x % kp, tfirst = (int) threadIdx.x / kp;
  const bool active = tfirst < tstep;  // threads past the last whole group of kp stay idle
  const int nu = nu0 + lnu;
  const int jx = nu / (M * M), jy = (nu / M) % M, jz = nu % M;
  for (uint32_t b0 = 0; b0 < ntr; b0 += BATCH) {
    const uint32_t nb = ntr - b0 < (uint32_t) BATCH ? ntr - b0 : (uint32_t) BATCH;
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < nb; e += blockDim.x) {
      const TriRef r = a.refs[tr0 + b0 + e];
      const TriRec &T = a.tri[r.t];
      for (int d = 0; d < 3; d++) {
        tv[e][d] = T.a[d];
        tv[e][3 + d] = T.b[d];
        tv[e][6 + d] = T.c[d];
        tn[e][d] = T.n[d];
        tl[e][d] = r.l[d];
      }
      tg[e] = T.g;
    }
    __syncthreads();
    // table: entry ((s * ns + q) * 3 + d) * M + mu; a thread keeps one (d, mu) and steps through
    // the (s, q) points with the rule's point count as a running remainder (no division by ns)
    if (threadIdx.x < (blockDim.x / (3 * M)) * (3 * M)) {
      const int dm = (int) threadIdx.x % (3 * M), d = dm / M, mu = dm % M;
      const uint32_t step = blockDim.x / (3 * M);
      const double *xi = pts + d * M;
      const double wb = wbar[d][mu];
      uint32_t sq = threadIdx.x / (3 * M), s = 0, q = sq;
      while (q >= (uint32_t) ns) {
        q -= ns;
        s++;
      }
      for (; sq < nb * ns; sq += step) {
        const double tx = sx[q], sy_ = sy[q];
        const double x = tv[s][d] * (1.0 - tx) + tv[s][3 + d] * (tx - sy_) + tv[s][6 + d] * sy_;
        const size_t e = (size_t) sq * 3 * M + dm;
        tab[e] = lagr_bar(x, xi, wb, mu, M);
        if (DN) dtab[e] = dlagr_bar(x, xi, wb, mu, M);
        q += step;
        while (q >= (uint32_t) ns) {
          q -= ns;
          s++;
        }
      }
    }
    __syncthreads();
    if (!active) continue;
    for (uint32_t s = tfirst; s < nb; s += tstep) {
      double sum[3] = {0.0, 0.0, 0.0};
      for (int q = 0; q < ns; q++) {
        const double *t3 = tab + ((size_t) s * ns + q) * 3 * M;
        const double lx = t3[jx], ly = t3[M + jy], lz = t3[2 * M + jz];
        double val;
        if (!DN) {
          val = lx * ly * lz;
        } else {
          const double *d3 = dtab + ((size_t) s * ns + q) * 3 * M;
          val = tn[s][0] * (d3[jx] * ly * lz) + tn[s][1] * (lx * d3[M + jy] * lz) +
                tn[s][2] * (lx * ly * d3[2 * M + jz]);
        }
        if (LINEAR) {
#pragma unroll
          for (int l = 0; l < 3; l++) sum[l] += sw[l][q] * val;
        } else {
          sum[0] += sw[3][q] * val;
        }
      }
      if (LINEAR) {
#pragma unroll
        for (int l = 0; l < 3; l++) {
          const int row = tl[s][l];
          if (row >= 0) atomicAdd(&V[row + (uint32_t) lnu * rows], sum[l] * tg[s]);
        }
      } else {
        V[tl[s][0] + (uint32_t) lnu * rows] = tg[s] * sum[0];
      }
    }
  }
  __syncthreads();
  double *out = a.V + a.voff[c];
  if (a.transposed) {
    // V^T, k x rows column-major: consecutive threads write consecutive nu
    for (uint32_t e = threadIdx.x; e < rows * (uint32_t) kp; e += blockDim.x) {
      const uint32_t l2 = e % (uint32_t) kp, i = e / (uint32_t) kp;
      out[(size_t) nu0 + l2 + (size_t) i * K] = V[i + l2 * rows];
    }
  } else {
    double *o = out + (size_t) nu0 * rows;
    for (uint32_t e = threadIdx.x; e < rows * (uint32_t) kp; e += blockDim.x) o[e] = V[e];
  }
}

// Transfer matrix of every non-root cluster: E_c[i, nu] = L^father_nu(xi^c_i), k x k, the
// product Lx[ia][jx] Ly[ib][jy] Lz[ic][jz] of the one-dimensional factors (i = (ia m + ib) m + ic,
// nu = (jx m + jy) m + jz).  CTA per cluster, thread per index of the stored matrix's fast
// dimension (i for E, nu for E^T), looping over the other one: consecutive threads write
// consecutive words.
__global__ void __launch_bounds__(128) transfer_kernel(FarTransferArgs a) {
  const uint32_t c = a.clusters[blockIdx.x];
  const uint32_t f = a.father[c];
  const int m = a.m, k = a.k, mm = m * m;
  const double *fp = a.pts + (size_t) f * 3 * m, *sp = a.pts + (size_t) c * 3 * m;
  __shared__ double L1[3][MMAX][MMAX];  // L1[d][son node][father polynomial]
  for (int e = threadIdx.x; e < 3 * mm; e += blockDim.x) {
    const int d = e / mm, p = (e / m) % m, mu = e % m;
    L1[d][p][mu] = lagrange_1d(sp[d * m + p], fp + d * m, mu, m);
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t >= k) return;
  const int t0 = t / mm, t1 = (t / m) % m, t2 = t % m;
  double *E = a.E + (size_t) (c - 1) * k * k + t;  // clusters 1..n-1 in pre-order
  int o = 0;
  if (!a.transposed) {
    // t = son node i: E[i + nu k] over nu
    for (int jx = 0; jx < m; jx++)
      for (int jy = 0; jy < m; jy++) {
        const double xy = L1[0][t0][jx] * L1[1][t1][jy];
        for (int jz = 0; jz < m; jz++, o += k) E[o] = xy * L1[2][t2][jz];
      }
  } else {
    // t = father polynomial nu: E^T[nu + i k] over i
    for (int ia = 0; ia < m; ia++)
      for (int ib = 0; ib < m; ib++) {
        const double xy = L1[0][ia][t0] * L1[1][ib][t1];
        for (int ic = 0; ic < m; ic++, o += k) E[o] = xy * L1[2][ic][t2];
      }
  }
}

// Coupling matrices: S_b[i, j] = (1/4pi) g(xi^r_i, xi^c_j), i = (ix m + iy) m + iz.  CTA per
// block, thread per row i (k <= 128 rows, the CTA rounded up to whole warps): the thread keeps
// its row point in registers and walks the columns j, whose points the CTA tabulates in shared
// memory first (every thread then reads the same word: a broadcast), so no index arithmetic is
// left in the loop.  Column j of S_b is written by consecutive threads (column-major, ld k):
// 8 or 16 bytes per entry, one store each.
template <bool CX>
__global__ void __launch_bounds__(128) coupling_kernel(FarCouplingArgs a) {
  __shared__ double yc[3][128];
  const uint32_t b = blockIdx.x;
  const uint32_t rc = a.rc[b], cc = a.cc[b];
  const int m = a.m, k = a.k, mm = m * m;
  const double *rp = a.rpts + (size_t) rc * 3 * m, *cp = a.cpts + (size_t) cc * 3 * m;
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    yc[0][j] = cp[j / mm];
    yc[1][j] = cp[m + (j / m) % m];
    yc[2][j] = cp[2 * m + j % m];
  }
  const int i = threadIdx.x;
  double x0 = 0.0, x1 = 0.0, x2 = 0.0;
  if (i < k) {
    x0 = rp[i / mm];
    x1 = rp[m + (i / m) % m];
    x2 = rp[2 * m + i % m];
  }
  __syncthreads();
  if (i >= k) return;
  const double kc = a.kconst, kre = a.k_re, kim = a.k_imn;
  if (!CX) {
    double *S = a.S + (size_t) b * k * k + i;
    for (int j = 0; j < k; j++) {
      const double d0 = x0 - yc[0][j], d1 = x1 - yc[1][j], d2 = x2 - yc[2][j];
      const double r2 = fma(d0, d0, fma(d1, d1, d2 * d2));
      S[(size_t) j * k] = kc * rsqrt_nr(r2);
    }
  } else {
    double2 *S = reinterpret_cast<double2 *>(a.S) + (size_t) b * k * k + i;
    for (int j = 0; j < k; j++) {
      const double d0 = x0 - yc[0][j], d1 = x1 - yc[1][j], d2 = x2 - yc[2][j];
      const double r2 = fma(d0, d0, fma(d1, d1, d2 * d2));
      const double rinv = rsqrt_nr(r2);
      double r = r2 * rinv, rn = rinv, sn, cs;
      if (kim != 0.0) rn *= exp(kim * r);
      sincos(kre * r, &sn, &cs);
      S[(size_t) j * k] = make_double2(kc * (rn * cs), kc * (rn * sn));
    }
  }
}

}  // namespace

template <bool L, bool D, int M>
static int launch_leaf(const FarLeafArgs *a, size_t smem, cudaStream_t st) {
  H2B_CUDA_TRY((h2b_allow_smem<leaf_basis_kernel<L, D, M>>()));
  leaf_basis_kernel<L, D, M><<<a->nleaves * (uint32_t) a->split, 256, smem, st>>>(*a);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

template <bool L, bool D>
static int launch_leaf_m(const FarLeafArgs *a, size_t smem, cudaStream_t st) {
  switch (a->m) {
    case 1: return launch_leaf<L, D, 1>(a, smem, st);
    case 2: return launch_leaf<L, D, 2>(a, smem, st);
    case 3: return launch_leaf<L, D, 3>(a, smem, st);
    case 4: return launch_leaf<L, D, 4>(a, smem, st);
    case 5: return launch_leaf<L, D, 5>(a, smem, st);
    default:
      h2b_set_error("leaf basis: interpolation order %d outside 1..5", a->m);
      return H2B_ERR_ARG;
  }
}

extern "C" int h2b_far_leaf_basis(const FarLeafArgs *a, int linear, int dn, cudaStream_t st) {
  if (a->nleaves == 0) return H2B_OK;
  if (a->split < 1 || a->split > a->k) {
    h2b_set_error("leaf basis: %d CTAs per leaf outside 1..%d", a->split, a->k);
    return H2B_ERR_ARG;
  }
  // the derivative table only for the normal-derivative bases
  const size_t smem = sizeof(double) * ((size_t) a->max_rows * ((a->k + a->split - 1) / a->split) +
                                        (dn ? 2 : 1) * (size_t) BATCH * a->ns * 3 * a->m);
  if (smem > 200u * 1024u || a->ns > NSMAX || (a->k + a->split - 1) / a->split > 256) {
    h2b_set_error("leaf basis block of %u x %d (rule of %d points) exceeds shared memory",
                  a->max_rows, a->k, a->ns);
    return H2B_ERR_ARG;
  }
  if (linear && dn) return launch_leaf_m<true, true>(a, smem, st);
  if (linear) return launch_leaf_m<true, false>(a, smem, st);
  if (dn) return launch_leaf_m<false, true>(a, smem, st);
  return launch_leaf_m<false, false>(a, smem, st);
}

extern "C" int h2b_far_transfer(const FarTransferArgs *a, cudaStream_t st) {
  if (a->n == 0) return H2B_OK;
  if (a->m > MMAX) {
    h2b_set_error("interpolation order %d > %d", a->m, MMAX);
    return H2B_ERR_ARG;
  }
  if (a->k > 128 || a->k != a->m * a->m * a->m) {
    h2b_set_error("transfer: rank %d is not m^3 <= 128", a->k);
    return H2B_ERR_ARG;
  }
  transfer_kernel<<<a->n, 32u * (((unsigned) a->k + 31u) / 32u), 0, st>>>(*a);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

extern "C" int h2b_far_coupling(const FarCouplingArgs *a, int cx, cudaStream_t st) {
  if (a->n == 0) return H2B_OK;
  if (a->k > 128 || a->k != a->m * a->m * a->m) {
    h2b_set_error("coupling: rank %d is not m^3 <= 128", a->k);
    return H2B_ERR_ARG;
  }
  const unsigned threads = 32u * (((unsigned) a->k + 31u) / 32u);
  if (cx)
    coupling_kernel<true><<<a->n, threads, 0, st>>>(*a);
  else
    coupling_kernel<false><<<a->n, threads, 0, st>>>(*a);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}
