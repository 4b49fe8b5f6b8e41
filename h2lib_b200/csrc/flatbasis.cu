// Flattened cluster bases for the H2 matvec (sm_100a, FP64).
//
// For every cluster t that needs one, W_t is the |t| x k matrix that the nested basis represents
// on t's indices: W_leaf = V_leaf and, for a father f with sons s,
//   W_f restricted to the rows of s = W_s E_s
// (the recursion of the reference's forward/backward transforms, Library/clusterbasis.c:524/749,
// multiplied out once after assembly), i.e. the rows of a leaf l inside W_f are
// W_l E_l E_{father(l)} ... up to f.  Every E is a tensor product of three one-dimensional
// transfers, so the path's product is too: it is formed per (leaf, ancestor) pair as three m x m
// matrices, and all ancestors' rows are then written in one launch, with no level-to-level
// dependence.  With W the forward transform is xt_t = W_t^T x_t and the
// backward transform y_t += W_t yt_t for all clusters at once: no level-to-level dependence, so
// the matvec streams W at HBM bandwidth instead of climbing the tree one level per step.
// Both sides store W transposed (W^T: k x |t|, column-major, ld = k), so that a slice of rows of
// t is one contiguous panel that the matvec copies to shared memory in one bulk transfer.  The
// column basis keeps V and E transposed as well (V^T, E^T); the row basis keeps them as H2Lib
// does (V: |t| x k, E: k x k), and its leaves are transposed on the copy into W.
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "farfield.h"

namespace {

constexpr int FLAT_TPB = 256;

// dst[e] = src(e) for e < n by the whole CTA, eight loads in flight per thread before the
// stores (a plain strided loop issues one global load per iteration and waits on each).
template <typename F>
__device__ __forceinline__ void cta_copy(double *dst, size_t n, F src) {
  constexpr int U = 8;
  for (size_t e0 = threadIdx.x; e0 < n; e0 += (size_t) blockDim.x * U) {
    double v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const size_t e = e0 + (size_t) u * blockDim.x;
      v[u] = e < n ? src(e) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const size_t e = e0 + (size_t) u * blockDim.x;
      if (e < n) dst[e] = v[u];
    }
  }
}

// Transfer products of the (leaf, ancestor) pairs: CTA per needed leaf l, walking up its
// ancestors f_1 = father(l), f_2, ... (the pairs of l, nearest first).  For every axis d,
//   P_1 = L_d(l -> f_1),  P_q = P_{q-1} L_d(f_{q-1} -> f_q),
// with L_d(c -> f)[a][mu] = polynomial mu of f's nodes at c's node a (the one-dimensional factor
// of the transfer E_c); E_l E_{f_1} ... E_{f_{q-1}} is then the tensor product of the three P_q.
template <int M>
__global__ void __launch_bounds__(128) flatten_paths_kernel(FlatArgs a) {
  constexpr int MM = M * M;
  __shared__ double P[3][M][M], L[3][M][M];
  const uint32_t p0 = a.pfirst[blockIdx.x], p1 = a.pfirst[blockIdx.x + 1];
  uint32_t node = a.leaves[blockIdx.x];
  const int e = (int) threadIdx.x, d = e / MM, pa = (e / M) % M, mu = e % M;
  for (uint32_t p = p0; p < p1; p++) {
    const uint32_t f = a.pairs[2 * (size_t) p + 1];
    if (e < 3 * MM)
      L[d][pa][mu] = lagrange_1d(a.pts[(size_t) node * 3 * M + d * M + pa],
                                 a.pts + (size_t) f * 3 * M + d * M, mu, M);
    __syncthreads();
    double v = 0.0;
    if (e < 3 * MM) {
      if (p == p0) {
        v = L[d][pa][mu];
      } else {
#pragma unroll
        for (int b = 0; b < M; b++) v = fma(P[d][pa][b], L[d][b][mu], v);
      }
    }
    __syncthreads();  // P and L are read
    if (e < 3 * MM) {
      P[d][pa][mu] = v;
      a.P[(size_t) p * 3 * MM + e] = v;
    }
    node = f;
  }
}

// CTA per item = ((leaf l, ancestor f) pair, first row r0 of l, rows nr <= H2B_FLAT_ROWS): the nr
// rows of W_l times the pair's transfer product land in the rows of l inside W_f.  The product is
// the tensor product of the three m x m factors P_d, so each row, an m x m x m tensor w[a][b][c],
// is multiplied one axis at a time:
//   t1[a][b][jz] = sum_c w[a][b][c] Pz[c][jz],  t2[a][jy][jz] = sum_b t1[a][b][jz] Py[b][jy],
//   W_f[jx][jy][jz] = sum_a t2[a][jy][jz] Px[a][jx]
// -- 3 m^4 multiply-adds per row instead of the k^2 = m^6 of the full product.  The rows are
// staged in shared memory in chunks of RB; a thread takes one fibre of m inputs and writes its m
// outputs, so every input is read once per step.
template <int M>
struct FlatShape {
  static constexpr int K = M * M * M;
  // rows per chunk: two K-double buffers per row within 96 KiB (at most H2B_FLAT_ROWS)
  static constexpr int RB = (96 * 1024) / (16 * K) < H2B_FLAT_ROWS ? (96 * 1024) / (16 * K)
                                                                   : H2B_FLAT_ROWS;
  static_assert(RB >= 1, "rank too large for the staged flatten");
};

template <int M>
__global__ void __launch_bounds__(FLAT_TPB) flatten_rows_kernel(FlatArgs a) {
  constexpr int K = FlatShape<M>::K, RB = FlatShape<M>::RB, MM = M * M;
  extern __shared__ double sm[];
  __shared__ double L[3][M][M];  // the pair's three transfer products
  const uint32_t *it = a.items + 4 * (size_t) blockIdx.x;
  const uint32_t pid = it[0], r0 = it[1], nr = it[2];
  const uint32_t l = a.pairs[2 * (size_t) pid], f = a.pairs[2 * (size_t) pid + 1];
  for (int e = (int) threadIdx.x; e < 3 * MM; e += (int) blockDim.x)
    (&L[0][0][0])[e] = a.P[(size_t) pid * 3 * MM + e];
  double *A = sm, *B = sm + (size_t) RB * K;
  const uint32_t rf = a.off[l] - a.off[f] + r0;  // first row inside f
  const double *Ws = a.W + a.woff[l] + (size_t) r0 * K;
  double *Wf = a.W + a.woff[f] + (size_t) rf * K;
  for (uint32_t c0 = 0; c0 < nr; c0 += RB) {
    const uint32_t nc = min((uint32_t) RB, nr - c0);
    __syncthreads();  // L is ready; the previous chunk's last step has read A
    // W_l^T rows are contiguous (ld K)
    for (uint32_t e = threadIdx.x; e < nc * K; e += blockDim.x) A[e] = Ws[(size_t) c0 * K + e];
    __syncthreads();
    // z: fibre g = (row, a, b) of A -> B[row][a][b][jz]
    for (uint32_t g = threadIdx.x; g < nc * MM; g += blockDim.x) {
      double in[M];
#pragma unroll
      for (int c = 0; c < M; c++) in[c] = A[(size_t) g * M + c];
#pragma unroll
      for (int jz = 0; jz < M; jz++) {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < M; c++) acc = fma(in[c], L[2][c][jz], acc);
        B[(size_t) g * M + jz] = acc;
      }
    }
    __syncthreads();
    // y: fibre g = (row, a, jz) of B (stride M) -> A[row][a][jy][jz]
    for (uint32_t g = threadIdx.x; g < nc * MM; g += blockDim.x) {
      const uint32_t jz = g % M, ra = g / M;
      const double *x = B + (size_t) ra * MM + jz;
      double in[M];
#pragma unroll
      for (int b = 0; b < M; b++) in[b] = x[b * M];
#pragma unroll
      for (int jy = 0; jy < M; jy++) {
        double acc = 0.0;
#pragma unroll
        for (int b = 0; b < M; b++) acc = fma(in[b], L[1][b][jy], acc);
        A[(size_t) ra * MM + jy * M + jz] = acc;
      }
    }
    __syncthreads();
    // x: fibre g = (row, jy, jz) of A (stride M^2) -> W_f rows, consecutive threads writing
    // consecutive (jy, jz)
    for (uint32_t g = threadIdx.x; g < nc * MM; g += blockDim.x) {
      const uint32_t yz = g % MM, row = g / MM;
      const double *x = A + (size_t) row * K + yz;
      double in[M];
#pragma unroll
      for (int p = 0; p < M; p++) in[p] = x[p * MM];
      double *o = Wf + (size_t) (c0 + row) * K + yz;
#pragma unroll
      for (int jx = 0; jx < M; jx++) {
        double acc = 0.0;
#pragma unroll
        for (int p = 0; p < M; p++) acc = fma(in[p], L[0][p][jx], acc);
        o[jx * MM] = acc;
      }
    }
  }
}

// W_leaf^T from V_leaf: a copy when V is stored transposed (column side), a transposition when V
// is stored |t| x k (row side).
__global__ void __launch_bounds__(FLAT_TPB) leaf_copy_kernel(FlatLeafArgs a) {
  const uint32_t l = a.leaves[blockIdx.x];
  const uint32_t nt = a.size[l], k = (uint32_t) a.k;
  const size_t n = (size_t) nt * k;
  const double *src = a.V + a.voff[l];
  double *dst = a.W + a.woff[l];
  if (a.transpose)
    cta_copy(dst, n, [&](size_t e) {  // dst[nu + i k] = V[i + nu nt]
      const uint32_t nu = (uint32_t) (e % k), i = (uint32_t) (e / k);
      return src[i + (size_t) nu * nt];
    });
  else
    cta_copy(dst, n, [&](size_t e) { return src[e]; });
}

// out[i] = (float) in[i] (round to nearest)
__global__ void to_single_kernel(const double *__restrict__ in, float *__restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n;
       i += (size_t) gridDim.x * blockDim.x)
    out[i] = __double2float_rn(in[i]);
}

}  // namespace

extern "C" int h2b_to_single(const double *in, float *out, size_t n, int num_sms,
                             cudaStream_t st) {
  if (n == 0) return H2B_OK;
  const size_t want = (n + FLAT_TPB - 1) / FLAT_TPB, cap = (size_t) 8 * (num_sms > 0 ? num_sms : 148);
  to_single_kernel<<<(unsigned) (want < cap ? want : cap), FLAT_TPB, 0, st>>>(in, out, n);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

extern "C" int h2b_flat_leaves(const FlatLeafArgs *a, cudaStream_t st) {
  if (a->nleaves) {
    leaf_copy_kernel<<<a->nleaves, FLAT_TPB, 0, st>>>(*a);
    h2b_note_launch();
  }
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

template <int M>
static int launch_flatten(const FlatArgs *a, int rows, cudaStream_t st) {
  if (!rows) {
    flatten_paths_kernel<M><<<a->nleaves, 128, 0, st>>>(*a);
  } else {
    constexpr size_t smem = sizeof(double) * 2 * FlatShape<M>::RB * FlatShape<M>::K;
    H2B_CUDA_TRY(h2b_allow_smem<flatten_rows_kernel<M>>());
    flatten_rows_kernel<M><<<a->nitems, FLAT_TPB, smem, st>>>(*a);
  }
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

static int flatten_dispatch(const FlatArgs *a, int rows, cudaStream_t st) {
  if ((rows ? a->nitems : a->nleaves) == 0) return H2B_OK;
  if (a->k != a->m * a->m * a->m) {
    h2b_set_error("flattened bases: rank %d is not m^3 for m = %d", a->k, a->m);
    return H2B_ERR_ARG;
  }
  switch (a->m) {
    case 1: return launch_flatten<1>(a, rows, st);
    case 2: return launch_flatten<2>(a, rows, st);
    case 3: return launch_flatten<3>(a, rows, st);
    case 4: return launch_flatten<4>(a, rows, st);
    case 5: return launch_flatten<5>(a, rows, st);
    default:
      h2b_set_error("flattened bases: interpolation order %d outside 1..5", a->m);
      return H2B_ERR_ARG;
  }
}

extern "C" int h2b_flat_paths(const FlatArgs *a, cudaStream_t st) {
  return flatten_dispatch(a, 0, st);
}

extern "C" int h2b_flat_rows(const FlatArgs *a, cudaStream_t st) {
  return flatten_dispatch(a, 1, st);
}
