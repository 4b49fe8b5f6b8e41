// Device layout of an H2 matrix as the matvec kernels read it (h2mvm.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// One GEMV work item of a product: a panel P (rows x cols, column-major, ld = rows, contiguous),
// applied as y[0, rows) += P x[0, cols) or, transposed, y[0, cols) += P^T x[0, rows); x and y
// are slices of the product's work vectors.  The kind selects the panel array and the vectors:
//   forward    W_c^T slice, x = xp, y = xt
//   nearfield  N block panel, x = xp, y = yp
//   coupling   S block panel, x = xt, y = yt
//   backward   W_r^T slice (transposed), x = yt, y = yp
#define H2B_MV_FORWARD 0u
#define H2B_MV_NEAR 1u
#define H2B_MV_COUPLING 2u
#define H2B_MV_BACKWARD 3u
#define H2B_MV_KIND 3u       // flags & H2B_MV_KIND: the kind
#define H2B_MV_TRANS 4u      // y += P^T x
struct MvItem {
  uint64_t p;                // element offset of the panel in its array
  uint32_t rows, cols;
  uint32_t xo, yo;           // element offsets of the x and y slices in one vector column
  uint32_t seg;              // surface of the item (masked batched products)
  uint32_t flags;
};
static_assert(sizeof(MvItem) == 32, "MvItem is 32 bytes");

// The items of a product, ordered by kind: start[k] is the first item of kind k.
struct MvItems {
  const MvItem *items;       // device
  uint32_t n;
  uint32_t start[4];
  uint32_t max_bytes;        // largest panel in bytes at FP64 storage
  uint32_t max_rows;         // largest rows of an untransposed item
  uint32_t max_cols_t;       // largest columns of a transposed item
  uint32_t max_x;            // longest x slice (elements: cols, or rows when transposed)
};

// Default largest panel of a work item (bytes at FP64 storage); blocks and slices are split to fit.
#define H2B_MV_PANEL_BYTES (16u * 1024u)

struct MvmPlan {
  int cx, num_sms;
  int k;
  uint32_t nrow, ncol, nrow_clusters, ncol_clusters;
  const uint32_t *ridx, *cidx;   // device index arrays of the row / column tree
  double *xp, *yp, *xt, *yt;     // work vectors of one column
  MvItems items;                 // the FP64 product's items
  MvItems items_single;          // the items of the product from the FP32 copies (larger panels)
  // panel arrays (FP64) and their FP32 copies (NULL until made)
  const double *Wc, *Wr, *N, *S;
  const float *fWc, *fWr, *fN, *fS;
  int *err;                      // device flag: a wait for a panel copy ran out
  // launch shape of the item kernel: resident CTAs per SM, consumer warps per CTA and ring
  // stages per consumer warp
  int ctas_per_sm, warps, stages;
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
// y += (ar + i ai) A x + (br + i bi) B x for the plans p (A) and q (B) of two matrices on one
// structure whose coupling matrices and row bases are equal: the coupling matrices and the row
// basis (p's) are read once.  single: the FP32 copies of both.  work: NULL (the plans' own work
// vectors) or h2b_mvm_pair_work_doubles(p) doubles.
extern "C" size_t h2b_mvm_pair_work_doubles(const MvmPlan *p);
extern "C" int h2b_mvm_launch_pair(const MvmPlan *p, const MvmPlan *q, int single,
                                   const double *x, double *y, double ar, double ai, double br,
                                   double bi, double *work, cudaStream_t st);
extern "C" size_t h2b_mvm_work_doubles(const MvmPlan *p, uint32_t nrhs);
extern "C" int h2b_mvm_launch_batch(const MvmPlan *p, int single, uint32_t nrhs, const double *x,
                                    size_t ldx, double *y, size_t ldy, double ar, double ai,
                                    double *work, const uint32_t *mask, uint32_t nseg,
                                    cudaStream_t st);
// Sets the item kernel's shared-memory limit (once per process); called when a matrix is made,
// so that no later launch, possibly inside a CUDA graph capture, has to.
extern "C" int h2b_mvm_prepare(void);
// Shared-memory bytes per CTA of the item kernel at the plan's launch shape.
extern "C" size_t h2b_mvm_smem_bytes(const MvmPlan *p, int single);
