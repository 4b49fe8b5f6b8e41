// Device-side building blocks shared by the h2b200 CUDA sources (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "h2b200_internal.h"

#define H2B_CUDA_TRY(call)                                                                     \
  do {                                                                                        \
    cudaError_t err__ = (call);                                                               \
    if (err__ != cudaSuccess) {                                                               \
      h2b_set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(err__));  \
      return H2B_ERR_CUDA;                                                                    \
    }                                                                                         \
  } while (0)

// Counts kernel launches made by the library (every host thread), read with h2b_launch_count.
// Each direct launch site of the assembly, classification and matvec kernels calls it once.
void h2b_note_launch(void);

// 1/(4 pi): constant of the fundamental solutions of Laplace and Helmholtz
// (KERNEL_CONST_LAPLACEBEM3D, Library/laplacebem3d.c:33; KERNEL_CONST_HELMHOLTZBEM3D,
// Library/helmholtzbem3d.c:25).
#define H2B_KERNEL_CONST 0.0795774715459476679

// One triangle as the quadrature kernels read it: 128 bytes, 16-byte aligned, loaded with eight
// 16-byte vector loads.  Vertices are in the triangle's own order (H2Lib's gr->t[i]).
struct __align__(16) TriRec {
  double a[3], b[3], c[3];  // vertex coordinates
  double n[3];              // unit normal
  double g;                 // Gram determinant = 2 * area
  uint32_t v[3];            // vertex ids
  uint32_t pad0;
  double pad1;
};
static_assert(sizeof(TriRec) == 128, "TriRec must be 128 bytes");

// A triangle referenced by a nearfield tile: its id and the local output row/column index of each
// of its three vertices (linear basis) or of the triangle itself in l[0] (constant basis); -1 when
// the vertex is outside the tile.
struct TriRef {
  uint32_t t;
  int16_t l[3];
  int16_t pad;
};
static_assert(sizeof(TriRef) == 12, "TriRef must be 12 bytes");

// Reciprocal square root in FP64, full precision.
// Seed: the FP64 approximate reciprocal square root instruction (rsqrt.approx.ftz.f64, relative
// error below 1e-6 measured on B200); two Newton-Raphson steps y <- y + y/2 (1 - x y^2) in FP64
// (the classical iteration for x^{-1/2}; each step squares the relative error, so the result is
// within 1.2 ulp, measured against 1/sqrt over 4M arguments in [1e-12, 16]).  Inputs are squared
// distances of quadrature points: positive and normal.  (Measured in the nearfield kernel: 4%
// faster than an FP32 seed, which needs two conversions, and 7% faster than CUDA's rsqrt().)
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double h = x * y;
  double e = fma(-h, y, 1.0);
  y = fma(0.5 * y, e, y);
  h = x * y;
  e = fma(-h, y, 1.0);
  return fma(0.5 * y, e, y);
}

// Lagrange polynomial mu of the nodes xi[0..m) at x, prod_{l != mu} (x - xi_l) / (xi_mu - xi_l)
// (the one-dimensional factor of the tensor interpolation, Library/bem3d.c:8497).
__device__ __forceinline__ double lagrange_1d(double x, const double *xi, int mu, int m) {
  double v = 1.0;
  for (int l = 0; l < m; l++)
    if (l != mu) v *= (x - xi[l]) / (xi[mu] - xi[l]);
  return v;
}

// Allow kernel K up to H2B_MAX_DYN_SMEM bytes of dynamic shared memory, once per process
// (thread-safe static initialisation).  Launches pass the size they need; the attribute never
// changes afterwards, so launches from several host threads (a solve server's workers) cannot
// race on it.
#define H2B_MAX_DYN_SMEM (200u * 1024u)
template <auto K>
inline cudaError_t h2b_allow_smem() {
  static const cudaError_t rc = cudaFuncSetAttribute(
      K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) H2B_MAX_DYN_SMEM);
  return rc;
}

struct dcomplex {
  double re, im;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
