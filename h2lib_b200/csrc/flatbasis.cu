// Flattened cluster bases for the H2 matvec (sm_100a, FP64).
//
// For every cluster t that needs one, W_t is the |t| x k matrix that the nested basis represents
// on t's indices: W_leaf = V_leaf and, for a father f with sons s,
//   W_f restricted to the rows of s = W_s E_s
// (the recursion of the reference's forward/backward transforms, Library/clusterbasis.c:524/749,
// multiplied out once after assembly).  With W the forward transform is xt_t = W_t^T x_t and the
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

// CTA per item = (father f, son s, first row r0 of s, rows nr <= H2B_FLAT_ROWS): the nr rows of
// W_s times E_s land in the rows of s inside W_f.  E_s is the tensor product of three m x m
// one-dimensional transfers, E_s[(a, b, c), (jx, jy, jz)] = Lx[a][jx] Ly[b][jy] Lz[c][jz] with
// L_d[a][mu] = father polynomial mu of axis d at son node a (the factors of transfer_kernel), so
// each row, an m x m x m tensor w[a][b][c], is multiplied one axis at a time:
//   t1[a][b][jz] = sum_c w[a][b][c] Lz[c][jz],  t2[a][jy][jz] = sum_b t1[a][b][jz] Ly[b][jy],
//   W_f[jx][jy][jz] = sum_a t2[a][jy][jz] Lx[a][jx]
// -- 3 m^4 multiply-adds per row instead of the k^2 = m^6 of the full product (the same sum,
// bracketed by axis).  The rows are staged in shared memory in chunks of RB; a thread takes one
// fibre of m inputs and writes its m outputs, so every input is read once per step.
template <int M>
struct FlatShape {
  static constexpr int K = M * M * M;
  // rows per chunk: two K-double buffers per row within 96 KiB (at most H2B_FLAT_ROWS)
  static constexpr int RB = (96 * 1024) / (16 * K) < H2B_FLAT_ROWS ? (96 * 1024) / (16 * K)
                                                                   : H2B_FLAT_ROWS;
  static_assert(RB >= 1, "rank too large for the staged flatten");
};

template <int M>
__global__ void __launch_bounds__(FLAT_TPB) flatten_kernel(FlatArgs a) {
  constexpr int K = FlatShape<M>::K, RB = FlatShape<M>::RB, MM = M * M;
  extern __shared__ double sm[];
  __shared__ double L[3][M][M];  // L[d][son node][father polynomial]
  const uint32_t *it = a.items + 4 * (size_t) blockIdx.x;
  const uint32_t f = it[0], s = it[1], r0 = it[2], nr = it[3];
  const double *fp = a.pts + (size_t) f * 3 * M, *sp = a.pts + (size_t) s * 3 * M;
  for (int e = (int) threadIdx.x; e < 3 * MM; e += (int) blockDim.x) {
    const int d = e / MM, p = (e / M) % M, mu = e % M;
    L[d][p][mu] = lagrange_1d(sp[d * M + p], fp + d * M, mu, M);
  }
  double *A = sm, *B = sm + (size_t) RB * K;
  const uint32_t rf = a.off[s] - a.off[f] + r0;  // first row inside f
  const double *Ws = a.W + a.woff[s] + (size_t) r0 * K;
  double *Wf = a.W + a.woff[f] + (size_t) rf * K;
  for (uint32_t c0 = 0; c0 < nr; c0 += RB) {
    const uint32_t nc = min((uint32_t) RB, nr - c0);
    __syncthreads();  // L is ready; the previous chunk's last step has read A
    // W_s^T rows are contiguous (ld K)
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
static int launch_flatten(const FlatArgs *a, cudaStream_t st) {
  constexpr size_t smem = sizeof(double) * 2 * FlatShape<M>::RB * FlatShape<M>::K;
  H2B_CUDA_TRY(h2b_allow_smem<flatten_kernel<M>>());
  flatten_kernel<M><<<a->nitems, FLAT_TPB, smem, st>>>(*a);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

extern "C" int h2b_flat_level(const FlatArgs *a, cudaStream_t st) {
  if (a->nitems == 0) return H2B_OK;
  if (a->k != a->m * a->m * a->m) {
    h2b_set_error("flattened bases: rank %d is not m^3 for m = %d", a->k, a->m);
    return H2B_ERR_ARG;
  }
  switch (a->m) {
    case 1: return launch_flatten<1>(a, st);
    case 2: return launch_flatten<2>(a, st);
    case 3: return launch_flatten<3>(a, st);
    case 4: return launch_flatten<4>(a, st);
    case 5: return launch_flatten<5>(a, st);
    case 6: return launch_flatten<6>(a, st);
    case 7: return launch_flatten<7>(a, st);
    case 8: return launch_flatten<8>(a, st);
    default:
      h2b_set_error("flattened bases: interpolation order %d outside 1..8", a->m);
      return H2B_ERR_ARG;
  }
}
