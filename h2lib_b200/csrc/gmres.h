// Device GMRES state and operator callback (gmres.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define GMRES_KMAX 128

struct GmresState {
  uint32_t k, pad;
  double err, bnorm;
  double gamma_re, gamma_im, alpha_re, alpha_im;
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
