// Greenhybrid cluster bases on the device (sm_100a, FP64): one CTA per cluster and one launch per
// tree level, deepest first.  The CTA fills A_t in shared memory, runs the full-pivoting cross
// approximation on it and writes the normalised row factor: a leaf's basis, or its sons'
// transfer matrices.  A second kernel forms the flattened bases W_t = [W_s E_s] level by level.
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "green.h"

namespace {

constexpr int GT = 256;  // threads per CTA

// A pivot candidate: |a|^2 and its position in the reference's scan order (columns outer, rows
// inner); of equal values the first in that order wins (decomp_fullaca_rkmatrix takes a new
// maximum only when it is strictly larger).
struct Best {
  double v;
  uint32_t l;
};

__device__ __forceinline__ Best better(Best a, Best b) {
  return (b.v > a.v || (b.v == a.v && b.l < a.l)) ? b : a;
}

// The CTA's best of every thread's candidate b, the same in every thread.
__device__ Best block_best(Best b, Best *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Best c;
    c.v = __shfl_down_sync(0xFFFFFFFFu, b.v, o);
    c.l = __shfl_down_sync(0xFFFFFFFFu, b.l, o);
    b = better(b, c);
  }
  __syncthreads();  // the previous result in red[] has been read
  if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    Best r = red[0];
    for (uint32_t w = 1; w < blockDim.x / 32; w++) r = better(r, red[w]);
    red[GT / 32] = r;
  }
  __syncthreads();
  return red[GT / 32];
}

// Largest |A(i, j)|^2 over i, j >= k (A column-major, ld = rows), the same in every thread.
__device__ Best block_argmax(const double *A, uint32_t rows, uint32_t cols, uint32_t k,
                             Best *red) {
  Best b{0.0, 0xFFFFFFFFu};
  const uint32_t nr = rows - k, tot = nr * (cols - k);
  for (uint32_t e = threadIdx.x; e < tot; e += blockDim.x) {
    const uint32_t i = k + e % nr, j = k + e / nr;
    const double a = A[i + (size_t) j * rows];
    b = better(b, Best{a * a, j * rows + i});
  }
  return block_best(b, red);
}

// Quadrature points and weighted normals of the widened box surface (build_bem3d_cube_quadpoints,
// Library/bem3d.c:5063): faces z = a - delta, x = b + delta, z = b + delta, x = a - delta,
// y = a - delta, y = b + delta, each with ml x ml points; the normal carries the point's weight.
__device__ void box_quadpoints(const GreenArgs &g, const double *box, double *Z, double *N) {
  const double *a = box, *b = box + 3;
  double diam = 0.0;
  for (int d = 0; d < 3; d++) diam = fmax(diam, b[d] - a[d]);
  const double delta = g.delta * diam;
  const int ml = g.ml, np = 6 * ml * ml;
  const double e0 = b[0] - a[0] + 2.0 * delta, e1 = b[1] - a[1] + 2.0 * delta,
               e2 = b[2] - a[2] + 2.0 * delta;
  const double m0 = 0.5 * (b[0] + a[0]), m1 = 0.5 * (b[1] + a[1]), m2 = 0.5 * (b[2] + a[2]);
  for (int nu = (int) threadIdx.x; nu < np; nu += (int) blockDim.x) {
    const int face = nu / (ml * ml), mu1 = (nu / ml) % ml, mu2 = nu % ml;
    const double u = 0.5 * g.tg[mu1], v = 0.5 * g.tg[mu2];
    double velo, z[3], n[3] = {0.0, 0.0, 0.0};
    switch (face) {
      case 0: velo = e0 * e1 * 0.25; break;
      case 1: velo = e1 * e2 * 0.25; break;
      case 2: velo = e0 * e1 * 0.25; break;
      case 3: velo = e1 * e2 * 0.25; break;
      default: velo = e0 * e2 * 0.25; break;
    }
    const double f = velo * g.wg[mu1] * g.wg[mu2];
    switch (face) {
      case 0: z[0] = m0 + e0 * u; z[1] = m1 + e1 * v; z[2] = a[2] - delta; n[2] = -f; break;
      case 1: z[0] = b[0] + delta; z[1] = m1 + e1 * u; z[2] = m2 + e2 * v; n[0] = f; break;
      case 2: z[0] = m0 + e0 * u; z[1] = m1 + e1 * v; z[2] = b[2] + delta; n[2] = f; break;
      case 3: z[0] = a[0] - delta; z[1] = m1 + e1 * u; z[2] = m2 + e2 * v; n[0] = -f; break;
      case 4: z[0] = m0 + e0 * u; z[1] = a[1] - delta; z[2] = m2 + e2 * v; n[1] = -f; break;
      default: z[0] = m0 + e0 * u; z[1] = b[1] + delta; z[2] = m2 + e2 * v; n[1] = f; break;
    }
    for (int d = 0; d < 3; d++) {
      Z[3 * nu + d] = z[d];
      N[3 * nu + d] = n[d];
    }
  }
}

// A_t(r, j): basis function rowid[r] integrated against the fundamental solution at Z_j
// (columns j < k2) and its derivative in the weighted normal N_j (columns k2 + j), with the
// single-triangle rule: fill_row_{c,l}_bem3d / fill_dnz_row_{c,l}_bem3d (Library/bem3d.c:3542,
// :4020, :4252, :4740) with the Laplace kernels of Library/laplacebem3d.c:36 and :84; on the
// column side of the double layer the kernels differentiate in the triangle's normal too
// (fill_col_l_bem3d / fill_dnz_col_l_bem3d, :4136 / :4857, with dlp_kernel and hs_kernel,
// Library/laplacebem3d.c:84 / :187, arguments (Z_j, x)).
template <bool LINEAR, bool DCOL>
__device__ void fill_matrix(const GreenArgs &g, double *A, uint32_t rows, const uint32_t *rowid,
                            const double *Z, const double *N, int k2, const double *sw,
                            const double *sx, const double *sy) {
  const int ns = g.ns;
  const uint32_t tot = rows * (uint32_t) (2 * k2);
  for (uint32_t e = threadIdx.x; e < tot; e += blockDim.x) {
    const uint32_t r = e % rows, j = e / rows;
    const bool dn = j >= (uint32_t) k2;
    const uint32_t pj = dn ? j - (uint32_t) k2 : j;
    const double z0 = Z[3 * pj], z1 = Z[3 * pj + 1], z2 = Z[3 * pj + 2];
    const double n0 = N[3 * pj], n1 = N[3 * pj + 1], n2 = N[3 * pj + 2];
    const uint32_t bf = rowid[r];
    const uint32_t u0 = LINEAR ? g.vt_off[bf] : 0u, u1 = LINEAR ? g.vt_off[bf + 1] : 1u;
    double acc = 0.0;
    for (uint32_t u = u0; u < u1; u++) {
      const uint32_t t = LINEAR ? g.vt_tri[u] : bf;
      const TriRec &T = g.tri[t];
      const int c = LINEAR ? (T.v[0] == bf ? 0 : (T.v[1] == bf ? 1 : 2)) : 3;
      const double *w = sw + c * ns;
      double sum = 0.0;
      for (int q = 0; q < ns; q++) {
        const double tx = sx[q], s = sy[q];
        const double ax = 1.0 - tx, bx = tx - s, cx = s;
        const double x0 = T.a[0] * ax + T.b[0] * bx + T.c[0] * cx;
        const double x1 = T.a[1] * ax + T.b[1] * bx + T.c[1] * cx;
        const double x2 = T.a[2] * ax + T.b[2] * bx + T.c[2] * cx;
        double f;
        if (!DCOL) {
          const double d0 = x0 - z0, d1 = x1 - z1, d2 = x2 - z2;
          const double ri = rsqrt_nr(d0 * d0 + d1 * d1 + d2 * d2);
          f = dn ? (d0 * n0 + d1 * n1 + d2 * n2) * (ri * ri * ri) : ri;
        } else {
          const double d0 = z0 - x0, d1 = z1 - x1, d2 = z2 - x2;
          const double r2 = d0 * d0 + d1 * d1 + d2 * d2, ri = rsqrt_nr(r2);
          const double dt = d0 * T.n[0] + d1 * T.n[1] + d2 * T.n[2];
          if (!dn) {
            f = dt * (ri * ri * ri);
          } else {
            const double r5 = (ri * ri) * (ri * ri) * ri;
            const double dz = d0 * n0 + d1 * n1 + d2 * n2;
            const double nn = n0 * T.n[0] + n1 * T.n[1] + n2 * T.n[2];
            f = r5 * (-3.0 * (dz * dt) + r2 * nn);
          }
        }
        sum += w[q] * f;
      }
      acc += sum * (T.g * g.kconst);
    }
    A[r + (size_t) j * rows] = acc;
  }
}

template <bool LINEAR, bool DCOL>
__global__ void __launch_bounds__(GT) green_basis_kernel(GreenArgs g) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int K = g.K, k2 = K / 2, ns = g.ns;
  const uint32_t c = g.clusters[blockIdx.x];
  double *A = reinterpret_cast<double *>(smem);
  double *Z = A + (size_t) g.max_rows * K;
  double *N = Z + 3 * k2;
  double *sw = N + 3 * k2;  // 4 x ns: corner-weighted (linear basis) and raw weights
  double *sx = sw + 4 * ns;
  double *sy = sx + ns;
  Best *red = reinterpret_cast<Best *>(sy + ns);
  uint32_t *rowid = reinterpret_cast<uint32_t *>(red + GT / 32 + 1);
  uint32_t *rpiv = rowid + g.max_rows;
  uint32_t *cpiv = rpiv + g.max_rows;

  // the rows: a leaf's own basis functions, else the pivot rows of its sons in son order
  const uint32_t s0 = g.son0[c], s1 = g.son1[c];
  const bool leaf = s0 == UINT32_MAX;
  const uint32_t k0 = leaf ? 0u : g.rank[s0];
  const uint32_t k1 = (leaf || s1 == UINT32_MAX) ? 0u : g.rank[s1];
  const uint32_t rows = leaf ? g.size[c] : k0 + k1;
  const uint32_t cols = (uint32_t) K;
  for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) {
    rowid[r] = leaf ? g.idx[g.off[c] + r]
                    : (r < k0 ? g.piv[(size_t) s0 * K + r] : g.piv[(size_t) s1 * K + (r - k0)]);
    rpiv[r] = r;
  }
  for (uint32_t j = threadIdx.x; j < cols; j += blockDim.x) cpiv[j] = j;
  for (int q = (int) threadIdx.x; q < ns; q += (int) blockDim.x) {
    sx[q] = g.xs[q];
    sy[q] = g.ys[q];
    sw[3 * ns + q] = g.ws[q];
    for (int l = 0; l < 3; l++) sw[l * ns + q] = LINEAR ? g.wsl[l * ns + q] : 0.0;
  }
  box_quadpoints(g, g.box + 6 * (size_t) c, Z, N);
  __syncthreads();
  fill_matrix<LINEAR, DCOL>(g, A, rows, rowid, Z, N, k2, sw, sx, sy);
  __syncthreads();

  // cross approximation with full pivoting (decomp_fullaca_rkmatrix, Library/aca.c:18): pivot
  // row and column swapped to position k, the column below scaled by the pivot's reciprocal,
  // rank-one update of the rest, until the largest remaining |a|^2 is at most |a_max,0|^2 accur^2
  const uint32_t maxrank = rows < cols ? rows : cols;
  Best bst = block_argmax(A, rows, cols, 0, red);
  const double tol = bst.v * g.accur * g.accur;
  uint32_t k = 0;
  while (k < maxrank && bst.v > tol) {
    const uint32_t imax = bst.l % rows, jmax = bst.l / rows;
    if (threadIdx.x == 0) {
      uint32_t t = rpiv[k];
      rpiv[k] = rpiv[imax];
      rpiv[imax] = t;
      t = cpiv[k];
      cpiv[k] = cpiv[jmax];
      cpiv[jmax] = t;
    }
    if (jmax != k)
      for (uint32_t i = threadIdx.x; i < rows; i += blockDim.x) {
        const double y = A[i + (size_t) jmax * rows];
        A[i + (size_t) jmax * rows] = A[i + (size_t) k * rows];
        A[i + (size_t) k * rows] = y;
      }
    __syncthreads();
    if (imax != k)
      for (uint32_t j = threadIdx.x; j < cols; j += blockDim.x) {
        const double y = A[imax + (size_t) j * rows];
        A[imax + (size_t) j * rows] = A[k + (size_t) j * rows];
        A[k + (size_t) j * rows] = y;
      }
    __syncthreads();
    const double aij = 1.0 / A[k + (size_t) k * rows];
    for (uint32_t i = k + 1 + threadIdx.x; i < rows; i += blockDim.x) A[i + (size_t) k * rows] *= aij;
    __syncthreads();
    // the rank-one update, and the next pivot search over the entries it writes (the remaining
    // submatrix is exactly those)
    const uint32_t nr = rows - k - 1, nc = cols - k - 1;
    Best cand{0.0, 0xFFFFFFFFu};
    for (uint32_t e = threadIdx.x; e < nr * nc; e += blockDim.x) {
      const uint32_t i = k + 1 + e % nr, j = k + 1 + e / nr;
      // no contraction: a - (l u) rounded as the reference's scalar loop rounds it
      const double v = __dsub_rn(A[i + (size_t) j * rows],
                                 __dmul_rn(A[i + (size_t) k * rows], A[k + (size_t) j * rows]));
      A[i + (size_t) j * rows] = v;
      cand = better(cand, Best{v * v, j * rows + i});
    }
    k++;
    bst = block_best(cand, red);  // its barriers also order the update before the next swaps
    if (k >= maxrank) break;
  }

  // V = C (C on the pivot rows)^-1 (copy_lower_aca_amatrix + triangularsolve_amatrix,
  // Library/bem3d.c:6244): in pivot order the first k rows become the identity, the others
  // solve x L11 = c with L11 the unit lower triangle of the first k rows
  for (uint32_t p = k + threadIdx.x; p < rows; p += blockDim.x)
    for (uint32_t j = k; j-- > 0;) {
      double x = A[p + (size_t) j * rows];
      for (uint32_t l = j + 1; l < k; l++) x -= A[p + (size_t) l * rows] * A[l + (size_t) j * rows];
      A[p + (size_t) j * rows] = x;
    }
  __syncthreads();
  if (threadIdx.x == 0) g.rank[c] = k;
  for (uint32_t j = threadIdx.x; j < cols; j += blockDim.x)
    g.piv[(size_t) c * K + j] = j < k ? rowid[rpiv[j]] : 0u;
  // row p of the pivot order is row rpiv[p] of A_t's own order
  for (uint32_t e = threadIdx.x; e < rows * cols; e += blockDim.x) {
    const uint32_t p = e % rows, j = e / rows;
    const double v = j >= k ? 0.0 : (p < k ? (p == j ? 1.0 : 0.0) : A[p + (size_t) j * rows]);
    const uint32_t i = rpiv[p];
    if (leaf) {
      double *V = g.V + g.voff[c];
      if (g.transposed) V[j + (size_t) i * K] = v;
      else V[i + (size_t) j * rows] = v;
    } else {
      const uint32_t s = i < k0 ? s0 : s1, ii = i < k0 ? i : i - k0;
      g.E[(size_t) s * K * K + ii + (size_t) j * K] = v;
    }
  }
}

// W_t rows of son s = W_s E_s (the son's rank columns of W_s): one CTA per item of at most
// H2B_GREEN_FLAT_ROWS rows of one son, E_s in shared memory.
__global__ void __launch_bounds__(GT) green_flatten_kernel(GreenFlatArgs a) {
  extern __shared__ double sE[];
  const uint4 it = reinterpret_cast<const uint4 *>(a.items)[blockIdx.x];
  const uint32_t t = it.x, s = it.y, r0 = it.z, nr = it.w;
  const int K = a.K;
  const uint32_t ks = a.rank[s], o = a.off[s] - a.off[t];
  const double *E = a.E + (size_t) s * K * K;
  const double *Ws = a.W + a.woff[s];
  double *Wt = a.W + a.woff[t];
  for (int e = (int) threadIdx.x; e < K * K; e += (int) blockDim.x) sE[e] = E[e];
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < nr * (uint32_t) K; e += blockDim.x) {
    const uint32_t r = r0 + e / (uint32_t) K, nu = e % (uint32_t) K;
    const double *w = Ws + (size_t) r * K;
    double v = 0.0;
    for (uint32_t mu = 0; mu < ks; mu++) v = fma(w[mu], sE[mu + (size_t) nu * K], v);
    Wt[(size_t) (o + r) * K + nu] = v;
  }
}

}  // namespace

extern "C" size_t h2b_green_smem(uint32_t max_rows, int K) {
  const int k2 = K / 2;
  return sizeof(double) * ((size_t) max_rows * K + 6 * (size_t) k2 + 6 * 64) +
         sizeof(Best) * (GT / 32 + 1) + sizeof(uint32_t) * (2 * (size_t) max_rows + K);
}

template <bool L, bool D>
static int launch_basis(const GreenArgs *a, size_t smem, cudaStream_t st) {
  H2B_CUDA_TRY((h2b_allow_smem<green_basis_kernel<L, D>>()));
  green_basis_kernel<L, D><<<a->n, GT, smem, st>>>(*a);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

extern "C" int h2b_green_basis(const GreenArgs *a, cudaStream_t st) {
  if (a->n == 0) return H2B_OK;
  if (a->K != 12 * a->ml * a->ml || a->ml < 1 || a->ml > H2B_GREEN_MLMAX || a->ns > 64) {
    h2b_set_error("greenhybrid basis: %d points per axis and face outside 1..%d", a->ml,
                  H2B_GREEN_MLMAX);
    return H2B_ERR_ARG;
  }
  const size_t smem = h2b_green_smem(a->max_rows, a->K);
  if (smem > H2B_MAX_DYN_SMEM) {
    h2b_set_error("greenhybrid basis: %u rows x %d columns exceed shared memory", a->max_rows,
                  a->K);
    return H2B_ERR_ARG;
  }
  if (a->linear) return a->dcol ? launch_basis<true, true>(a, smem, st)
                                : launch_basis<true, false>(a, smem, st);
  return a->dcol ? launch_basis<false, true>(a, smem, st) : launch_basis<false, false>(a, smem, st);
}

extern "C" int h2b_green_flatten(const GreenFlatArgs *a, cudaStream_t st) {
  if (a->n == 0) return H2B_OK;
  const size_t smem = sizeof(double) * (size_t) a->K * a->K;
  H2B_CUDA_TRY((h2b_allow_smem<green_flatten_kernel>()));
  green_flatten_kernel<<<a->n, GT, smem, st>>>(*a);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}
