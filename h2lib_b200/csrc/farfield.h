// Launch descriptions of the farfield fill kernels (farfield.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"

struct FarLeafArgs {
  const TriRec *tri;
  const TriRef *refs;       // per leaf: triangles touching it with local rows
  const uint32_t *leaves;   // leaf cluster ids
  const uint32_t *tr_off, *tr_len;  // per leaf (index into refs)
  const uint32_t *size;     // per cluster
  const uint64_t *voff;     // per cluster: offset of its leaf basis
  const double *pts;        // per cluster: 3 x m interpolation nodes
  const double *xs, *ys;    // single-triangle rule (ns points)
  const double *ws;         // raw weights (ns)
  const double *wsl;        // linear-basis weighted weights (3 x ns)
  double *V;
  uint32_t nleaves, max_rows;
  int m, k, ns;
  int transposed;           // store V^T (k x rows) instead of V (rows x k)
  int split;                // CTAs per leaf (each a contiguous range of the k columns), 1..k
};

struct FarTransferArgs {
  const uint32_t *clusters;  // non-root cluster ids
  const uint32_t *father;
  const double *pts;
  double *E;                 // (n_clusters - 1) x k x k, cluster c at (c-1)*k*k
  uint32_t n;
  int m, k;
  int transposed;            // store E^T
};

struct FarCouplingArgs {
  const uint32_t *rc, *cc;   // per admissible block
  const double *rpts, *cpts;
  double *S;                 // per block k x k (complex: interleaved)
  uint32_t n;
  int m, k;
  double kconst, k_re, k_imn;
};

// Flattened bases (flatbasis.cu): items of at most H2B_FLAT_ROWS rows of one leaf.
#define H2B_FLAT_ROWS 32
struct FlatArgs {
  const uint32_t *items;     // 4 per item: (leaf, ancestor) pair, first row in the leaf, rows, 0
  const uint32_t *pairs;     // 2 per pair: leaf, ancestor
  const uint32_t *pfirst;    // per needed leaf: its first pair (nleaves + 1 entries)
  const uint32_t *leaves;    // needed leaves
  const uint32_t *off, *size;
  const uint64_t *woff;      // per cluster: offset of W_t (doubles); W^T is k x |t| (ld k)
  const double *pts;         // per cluster: the m one-dimensional nodes per axis (3 m doubles)
  double *P;                 // per pair: 3 m x m transfer products (written by h2b_flat_paths)
  double *W;
  uint32_t nitems, nleaves;
  int m, k;
};

struct FlatLeafArgs {
  const uint32_t *leaves, *size;
  const uint64_t *voff, *woff;
  const double *V;
  double *W;
  uint32_t nleaves;
  int k;
  int transpose;             // V stored |t| x k (row side): W^T = V^T is written
};

extern "C" int h2b_flat_leaves(const FlatLeafArgs *a, cudaStream_t st);
extern "C" int h2b_to_single(const double *in, float *out, size_t n, int num_sms,
                             cudaStream_t st);
extern "C" int h2b_flat_paths(const FlatArgs *a, cudaStream_t st);
extern "C" int h2b_flat_rows(const FlatArgs *a, cudaStream_t st);

extern "C" int h2b_far_leaf_basis(const FarLeafArgs *a, int linear, int dn, cudaStream_t st);
extern "C" int h2b_far_transfer(const FarTransferArgs *a, cudaStream_t st);
extern "C" int h2b_far_coupling(const FarCouplingArgs *a, int cx, cudaStream_t st);
