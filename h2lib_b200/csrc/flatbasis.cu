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

// CTA (item, part): item = (father f, son s, first row r0 of s, rows nr <= H2B_FLAT_ROWS), part =
// up to FLAT_COLS consecutive columns nu of the product (one part for k <= 64); the nr rows of
// W_s times those columns of E_s land in the rows of s inside W_f.  Short row slices give every
// level's launch enough CTAs and read each son's rows once; E_s is read by every slice of the son
// (from L2).  W^T is stored k x |t| (ld k) on both sides.
constexpr int FLAT_COLS = 64;
__global__ void __launch_bounds__(FLAT_TPB) flatten_kernel(FlatArgs a) {
  extern __shared__ double sm[];
  const uint32_t k = (uint32_t) a.k;
  const uint32_t nparts = (k + FLAT_COLS - 1) / FLAT_COLS;
  const uint32_t item = blockIdx.x / nparts, part = blockIdx.x % nparts;
  const uint32_t *it = a.items + 4 * (size_t) item;
  const uint32_t f = it[0], s = it[1], r0 = it[2], nr = it[3];
  const uint32_t c0 = part * FLAT_COLS, nc = min((uint32_t) FLAT_COLS, k - c0);
  double *sE = sm;                  // sE[j + mu nc] = E_s[mu, c0 + j]
  double *sW = sm + k * FLAT_COLS;  // W_s[r0 + i, mu] at sW[mu + i (k + 1)]
  const double *E = a.E + (size_t) (s - 1) * k * k;
  const uint32_t rf = a.off[s] - a.off[f] + r0;  // first row inside f
  const double *Ws = a.W + a.woff[s];
  double *Wf = a.W + a.woff[f];
  // E_s from E^T (column side: E_s[mu, nu] = E^T[nu + mu k]) or from E itself (row side:
  // E_s[mu, nu] = E[mu + nu k])
  for (uint32_t e = threadIdx.x; e < k * nc; e += blockDim.x) {
    const uint32_t j = e % nc, mu = e / nc;
    sE[j + mu * nc] = a.e_transposed ? E[c0 + j + (size_t) mu * k] : E[mu + (size_t) (c0 + j) * k];
  }
  // W_s^T (k x |s|, ld k) is contiguous over the item's rows: sW[mu + i (k + 1)] (padded stride,
  // so that a warp's rows fall in different banks)
  for (uint32_t e = threadIdx.x; e < nr * k; e += blockDim.x) {
    const uint32_t mu = e % k, i = e / k;
    sW[mu + i * (k + 1)] = Ws[(size_t) r0 * k + e];
  }
  __syncthreads();
  // thread = column j = t % 64, rows ig + 4 r (ig = t / 64); a warp writes 32 consecutive nu of
  // one row of W_f^T
  static_assert(FLAT_TPB / FLAT_COLS == 4 && H2B_FLAT_ROWS % 4 == 0, "thread mapping");
  constexpr int RC = H2B_FLAT_ROWS / 4;
  const uint32_t j = threadIdx.x % FLAT_COLS, ig = threadIdx.x / FLAT_COLS;
  if (j < nc) {
    double acc[RC];
#pragma unroll
    for (int r = 0; r < RC; r++) acc[r] = 0.0;
    for (uint32_t mu = 0; mu < k; mu++) {
      const double y = sE[j + mu * nc];
#pragma unroll
      for (int r = 0; r < RC; r++) {
        const uint32_t i = ig + 4u * r;
        if (i < nr) acc[r] = fma(sW[mu + i * (k + 1)], y, acc[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < RC; r++) {
      const uint32_t i = ig + 4u * r;
      if (i < nr) Wf[(size_t) (rf + i) * k + c0 + j] = acc[r];
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

extern "C" int h2b_flat_level(const FlatArgs *a, cudaStream_t st) {
  if (a->nitems == 0) return H2B_OK;
  const size_t smem = sizeof(double) * ((size_t) a->k * FLAT_COLS + (size_t) H2B_FLAT_ROWS * (a->k + 1));
  if (smem > H2B_MAX_DYN_SMEM) {
    h2b_set_error("flattened bases: rank %d needs %zu bytes of shared memory", a->k, smem);
    return H2B_ERR_ARG;
  }
  H2B_CUDA_TRY(h2b_allow_smem<flatten_kernel>());
  const uint32_t nparts = ((uint32_t) a->k + FLAT_COLS - 1) / FLAT_COLS;
  flatten_kernel<<<a->nitems * nparts, FLAT_TPB, smem, st>>>(*a);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}
