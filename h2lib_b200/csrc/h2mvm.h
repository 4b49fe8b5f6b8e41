// Device layout of an H2 matrix as the matvec kernels read it (h2mvm.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// One GEMV work item of a product: a panel P (rows x cols, column-major, ld = rows, contiguous)
// of one of a launch's two panel arrays, applied as y[0, rows) += P x[0, cols) or, transposed,
// y[0, cols) += P^T x[0, rows); x and y are slices of the launch's work vectors.
#define H2B_MV_SRC1 1u       // panel, x and y from the launch's second triple (else the first)
#define H2B_MV_TRANS 2u      // y += P^T x
struct MvItem {
  uint64_t p;                // element offset of the panel in its array
  uint32_t rows, cols;
  uint32_t xo, yo;           // element offsets of the x and y slices in one vector column
  uint32_t seg;              // surface of the item (masked batched products)
  uint32_t flags;
};
static_assert(sizeof(MvItem) == 32, "MvItem is 32 bytes");

// Items of one launch.  Panels of array 0 are real; panels of array 1 are complex when the
// operator is.  The shared-memory stage of a launch holds its largest panel.
struct MvPhase {
  const MvItem *items;       // device
  uint32_t n;
  uint32_t max_bytes;        // largest panel in bytes at FP64 storage
  uint32_t max_rows;         // largest rows of an untransposed item
};

// Panels are split so that none exceeds this many bytes at FP64 storage.
#define H2B_MV_PANEL_BYTES (32u * 1024u)

struct MvmPlan {
  int cx, num_sms;
  int k;
  uint32_t nrow, ncol, nrow_clusters, ncol_clusters;
  const uint32_t *ridx, *cidx;   // device index arrays of the row / column tree
  double *xp, *yp, *xt, *yt;     // work vectors of one column
  // the three launches: forward transform + nearfield, coupling, backward transform
  MvPhase ph[3];
  // panel arrays (FP64) and their FP32 copies (NULL until made)
  const double *Wc, *Wr, *N, *S;
  const float *fWc, *fWr, *fN, *fS;
  int *err;                      // device flag: a panel copy did not complete
  // launch shape of the item kernel: resident CTAs per SM and pipeline stages
  int ctas_per_sm, stages;
};

extern "C" int h2b_mvm_launch(const MvmPlan *p, const double *x, double *y, double ar, double ai,
                              cudaStream_t st);
// The same product from the FP32 copies of N, S and W: matrix entries are read as FP32 and
// widened, vectors and sums stay FP64, so the product reads half the bytes.
extern "C" int h2b_mvm_launch_single(const MvmPlan *p, const double *x, double *y, double ar,
                                     double ai, cudaStream_t st);
// y[:, r] += alpha A x[:, r] for nrhs columns (leading dimensions ldx, ldy in doubles) in one
// launch sequence that reads the matrix once; `work` holds h2b_mvm_work_doubles(p, nrhs)
// doubles.  mask (optional, forest matrices): column r of surface s is computed only when
// mask[s + r * nseg] != 0 (the others receive nothing).  single: the FP32 copies.
extern "C" size_t h2b_mvm_work_doubles(const MvmPlan *p, uint32_t nrhs);
extern "C" int h2b_mvm_launch_batch(const MvmPlan *p, int single, uint32_t nrhs, const double *x,
                                    size_t ldx, double *y, size_t ldy, double ar, double ai,
                                    double *work, const uint32_t *mask, uint32_t nseg,
                                    cudaStream_t st);
// Sets the item kernel's shared-memory limit (once per process); called when a matrix is made,
// so that no later launch, possibly inside a CUDA graph capture, has to.
extern "C" int h2b_mvm_prepare(void);
// Shared-memory bytes of the item kernel for a launch shape (for the autotuner's candidates).
extern "C" size_t h2b_mvm_smem_bytes(const MvmPlan *p, int phase, int single, int stages);
