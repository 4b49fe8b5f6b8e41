// Device layout of an H2 matrix as the matvec kernels read it (h2mvm.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

struct MvmCoupleArgs {
  const uint32_t *adm_rc, *adm_cc;
  const double *S;
  const uint32_t *near_rc, *near_cc;
  const uint64_t *near_off;
  const double *N;
  const float *Ss, *Ns;       // FP32 copies of S and N (NULL until made)
  const uint32_t *rsize, *csize, *roff, *coff;
  const double *xt, *xp;
  double *yt, *yp;
  uint32_t nadm, nnear;
  int k;
};

// Flattened-basis transforms (flatbasis.cu builds W): one item = rows [r0, r0 + nr) of cluster c.
#define H2B_MVM_FLAT_ROWS 128
#ifndef H2B_MVM_BACK_ROWS
#define H2B_MVM_BACK_ROWS 32
#endif
struct MvmFlatArgs {
  const uint32_t *items;      // 3 per item: cluster, first row, rows
  const uint32_t *off, *size; // per cluster
  const uint64_t *woff;       // per cluster: offset of W_t
  const double *W;            // row side |t| x k (ld |t|); column side k x |t| (ld k)
  const float *Ws;            // FP32 copy of W (NULL until made)
  uint32_t nitems;
  int k;
};

struct MvmPlan {
  int cx, num_sms;
  MvmFlatArgs ffwd, fbwd;        // forward (column side) and backward (row side) slices
  const uint32_t *rseg, *cseg;   // surface of every row / column cluster (forest trees)
  int k;
  uint32_t nrow, ncol, nrow_clusters, ncol_clusters;
  const uint32_t *ridx, *cidx;   // device index arrays of the row / column tree
  double *xp, *yp, *xt, *yt;     // work vectors
  MvmCoupleArgs cpl;
};

extern "C" int h2b_mvm_launch(const MvmPlan *p, const double *x, double *y, double ar, double ai,
                              cudaStream_t st);
// The same product from the FP32 copies of N, S and W: matrix entries are
// read as FP32 and widened, vectors and sums stay FP64, so the product reads half the bytes.
extern "C" int h2b_mvm_launch_single(const MvmPlan *p, const double *x, double *y, double ar,
                                     double ai, cudaStream_t st);
// y[:, r] += alpha A x[:, r] for nrhs columns (leading dimensions ldx, ldy in doubles) in one
// launch sequence that reads the matrix about once; `work` holds h2b_mvm_work_doubles(p, nrhs)
// doubles.  mask (optional, forest matrices): column r of surface s is computed only when
// mask[s + r * nseg] != 0 (the others receive nothing).  single: the FP32 copies.
extern "C" size_t h2b_mvm_work_doubles(const MvmPlan *p, uint32_t nrhs);
extern "C" int h2b_mvm_launch_batch(const MvmPlan *p, int single, uint32_t nrhs, const double *x,
                                    size_t ldx, double *y, size_t ldy, double ar, double ai,
                                    double *work, const uint32_t *mask, uint32_t nseg,
                                    cudaStream_t st);
