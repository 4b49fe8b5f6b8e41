// Device GMRES state and operator callback (gmres.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define GMRES_KMAX 128

struct GmresState {
  uint32_t k, pad;
  double err, bnorm;
  double gamma_re, gamma_im, alpha_re, alpha_im;
  // loop control of the graph-resident iteration (h2b_gmres_loop_graph)
  double tol;          // eps * |b|
  uint32_t iter;       // steps taken (the reference's loop counter)
  uint32_t maxiter;    // stop when iter + 1 == maxiter (0: no limit)
  uint32_t budget;     // steps left in the current graph launch
  uint32_t nan;        // 1: the residual estimate became NaN
};

struct GmresDev {
  int cx;
  uint32_t n, kmax, nblocks, ldpart;
  double *qr;      // n x kmax (complex: interleaved)
  double *tau;     // kmax (complex pairs)
  double *T;       // kmax x kmax (complex pairs)
  double *rhat;    // kmax + 1 (complex pairs)
  double *w, *u;   // kmax + 1 (complex pairs)
  double *q;       // n
  double *abuf;    // n
  double *part;    // nblocks x ldpart (complex pairs)
  GmresState *state;
};

// y += alpha * A x on stream st
struct GmresOp {
  void *ctx;
  int (*apply)(void *ctx, const double *x, double *y, double ar, double ai, cudaStream_t st);
};

extern "C" int h2b_gmres_step(const GmresDev *g, const GmresOp *op, cudaStream_t st);
extern "C" int h2b_gmres_init(const GmresDev *g, const GmresOp *op, const double *b, double *x,
                              cudaStream_t st);
extern "C" int h2b_gmres_finish(const GmresDev *g, const GmresOp *op, const double *b, double *x,
                                cudaStream_t st);
extern "C" int h2b_gmres_bnorm(const GmresDev *g, const double *b, cudaStream_t st);
// One graph that runs restarted GMRES steps until the residual estimate reaches state->tol, the
// step counter reaches maxiter or state->budget steps have run: a WHILE conditional node whose
// body restarts (finish + init, an IF conditional node) when k + 1 == kmax, takes one step and
// updates the loop condition on the device.  b and x are the device right-hand side and iterate.
extern "C" int h2b_gmres_loop_graph(const GmresDev *g, const GmresOp *op, const double *b,
                                    double *x, cudaStream_t st, cudaGraphExec_t *exec);
