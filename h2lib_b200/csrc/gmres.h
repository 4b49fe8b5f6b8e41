// Device GMRES state and operator callback (gmres.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define GMRES_KMAX 128
#define GMRES_TPB 256

// One system of a batch: rows [row0, row0 + n) of the global vectors (b, x, q, abuf), its
// Householder/Krylov matrix qr (n x kmax, column-major) at element offset qoff, and the vector
// blocks [blk0, blk0 + nblk) of GMRES_TPB rows that cover it.
struct GmresSys {
  uint32_t n, row0;
  uint64_t qoff;
  uint32_t blk0, nblk;
};

struct GmresState {    // per system
  uint32_t k;          // current Krylov dimension
  uint32_t active;     // 1: still iterating
  double err, bnorm;   // residual estimate |rhat_k|, |b|
  double gamma_re, gamma_im, alpha_re, alpha_im;  // Householder scalars of the last column
  double tol;          // eps * |b|
  uint32_t iter;       // steps taken (the reference's loop counter)
  uint32_t restart;    // 1: finish + init in the current iteration
  uint32_t nan;        // 1: the residual estimate became NaN
  uint32_t verify;     // mixed precision: restart to check the FP64 residual
};

struct GmresCtl {      // whole batch
  uint32_t maxiter;    // a system stops when iter + 1 == maxiter (0: no limit)
  uint32_t budget;     // steps left in the current graph launch
  uint32_t any_active, any_restart;
};

// Which systems a launch works on.
enum { GMRES_SEL_ALL = 0, GMRES_SEL_ACTIVE = 1, GMRES_SEL_RESTART = 2 };

struct GmresDev {
  int cx;
  int mixed;                 // 1: steps use op.apply_lo, restarts measure the FP64 residual
  int unitary;               // 1: unitary complex Givens rotations (see findapply_givens)
  uint32_t nsys, n, kmax, nblocks, ldpart;
  double eps;
  const GmresSys *sys;       // nsys
  const uint32_t *blk;       // nblocks: system of each block
  double *qr;                // sum_s n_s * kmax (complex: interleaved)
  double *tau;               // nsys x kmax (complex pairs)
  double *T;                 // nsys x kmax x kmax (complex pairs)
  double *rhat;              // nsys x (kmax + 1) (complex pairs)
  double *w, *u;             // nsys x (kmax + 1) (complex pairs)
  double *q;                 // n
  double *abuf;              // n
  double *part;              // nblocks x ldpart (complex pairs)
  GmresState *state;         // nsys
  GmresCtl *ctl;
  uint32_t *mask;            // nsys: 1 while the system is active (read by a masked operator)
};

// y += alpha * A x on stream st (x, y: the global vectors).  apply_lo (optional) is a cheaper,
// less accurate application used for the Arnoldi steps of a mixed-precision solve; residuals at
// (re)starts always use apply.
struct GmresOp {
  void *ctx;
  int (*apply)(void *ctx, const double *x, double *y, double ar, double ai, cudaStream_t st);
  int (*apply_lo)(void *ctx, const double *x, double *y, double ar, double ai, cudaStream_t st);
};

// Doubles of device work space for nsys systems of total size n (without b and x), and the
// number of vector blocks; h2b_gmres_layout fills the pointers of g from one array `p` and the
// host tables sys / blk (written to the device by the caller at g->sys / g->blk).
size_t h2b_gmres_workspace(int cx, uint32_t nsys, const uint32_t *sizes, uint32_t kmax,
                           uint32_t *nblocks);
void h2b_gmres_layout(GmresDev *g, double *p, int cx, uint32_t nsys, const uint32_t *sizes,
                      uint32_t kmax, GmresSys *sys_host, uint32_t *blk_host);

extern "C" int h2b_gmres_step(const GmresDev *g, const GmresOp *op, cudaStream_t st);
extern "C" int h2b_gmres_init(const GmresDev *g, const GmresOp *op, const double *b, double *x,
                              int sel, cudaStream_t st);
extern "C" int h2b_gmres_finish(const GmresDev *g, const GmresOp *op, const double *b, double *x,
                                int sel, cudaStream_t st);
extern "C" int h2b_gmres_bnorm(const GmresDev *g, const double *b, cudaStream_t st);
// finish without the restart: x += the current Krylov correction of the selected systems
extern "C" int h2b_gmres_update(const GmresDev *g, double *x, int sel, cudaStream_t st);
// One graph that runs restarted GMRES steps for every active system until none is active or
// ctl->budget steps have run: a WHILE conditional node whose body restarts the systems with
// k + 1 == kmax (finish + init inside an IF conditional node), takes one step and updates the
// loop condition on the device.  b and x are the device right-hand side and iterate.
extern "C" int h2b_gmres_loop_graph(const GmresDev *g, const GmresOp *op, const double *b,
                                    double *x, cudaStream_t st, cudaGraphExec_t *exec);
// Run a solve to the end with the loop graph: bnorm, init, loop launches, final finish.  Returns
// H2B_OK; per-system iteration counts are in state[s].iter (read back by the caller).
extern "C" int h2b_gmres_run(const GmresDev *g, const GmresOp *op, const double *b, double *x,
                             uint32_t maxiter, cudaStream_t st, GmresState *host_state);
