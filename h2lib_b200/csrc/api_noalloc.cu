// GMRES entry point that allocates no memory: its work space is a fixed, file-scope device array.
//
// Who needs it: callers that must not allocate device memory while they run a solve — code that
// runs under a strict device-memory budget fixed at start-up, callers whose allocator is owned by
// another framework (a memory pool they cannot enter), and real-time loops that forbid allocation
// calls and their synchronisation on the critical path.  h2b_solve_gmres allocates its Krylov
// work space per call (stream-ordered allocation) and captures a CUDA graph; this variant takes the
// work space from g_noalloc_scratch instead and launches the step kernels directly.
//
// The array is H2B_NOALLOC_SCRATCH_BYTES large; every GPU that loads the library holds it until
// the process exits.  All calls share it and it keeps the last call's contents, so calls that
// overlap on the GPU (different host threads, or different streams without ordering) race; the
// entries that must start at zero (T and the solver state) are cleared by every call.  Every call,
// failed ones included, waits for its own GPU work before it returns.
//
// Cost: the loop is driven from the host, one launch sequence per Arnoldi step followed by a read
// of the solver state (a device-to-host copy and a stream synchronisation), so each step pays a
// host round trip that h2b_solve_gmres, which runs up to 512 steps per CUDA graph launch, does
// not.  For small systems this makes the variant noticeably slower per step.
#include <cuda_runtime.h>
#include <string.h>

#include <vector>

#include "api_h2.h"
#include "gmres.h"

__device__ __align__(256) unsigned char g_noalloc_scratch[H2B_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of g_noalloc_scratch on the current device.  In host code the symbol's name is
// only a host-side stand-in, so the address is looked up with the device current.  It is looked
// up on every call (a cheap table lookup once the module is loaded): no cached address can go
// stale after cudaDeviceReset, and concurrent first calls share no host state.
int scratch_address(void **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    h2b_set_error("h2b_solve_gmres_noalloc: cudaGetSymbolAddress failed: %s",
                  cudaGetErrorString(e));
    return H2B_ERR_CUDA;
  }
  *out = p;
  return H2B_OK;
}

// Waits for the stream when a call returns early, so that no queued work of a failed call keeps
// using the shared array after the call has returned.
struct StreamDrain {
  cudaStream_t st;
  bool armed = false;
  ~StreamDrain() {
    if (armed) cudaStreamSynchronize(st);
  }
};

struct ComboNA {
  uint32_t nterms;
  const h2b_h2matrix *ops[16];
  double cre[16], cim[16];
};

int combo_apply_na(void *ctx, const double *x, double *y, double ar, double ai, cudaStream_t st) {
  const ComboNA *c = (const ComboNA *) ctx;
  for (uint32_t i = 0; i < c->nterms; i++) {
    const double br = ar * c->cre[i] - ai * c->cim[i], bi = ar * c->cim[i] + ai * c->cre[i];
    int rc = h2b_mvm_launch(&c->ops[i]->mvm, x, y, br, bi, st);
    if (rc != H2B_OK) return rc;
  }
  return H2B_OK;
}

}  // namespace

extern "C" int h2b_solve_gmres_noalloc(uint32_t nterms, const h2b_h2matrix *const *ops,
                                       const double *coef, const double *b, double *x,
                                       double eps, uint32_t maxiter, uint32_t kmax) {
  if (nterms < 1 || nterms > 16 || !ops || !coef || !b || !x) {
    h2b_set_error("h2b_solve_gmres_noalloc: between 1 and 16 operators and non-NULL vectors");
    return H2B_ERR_ARG;
  }
  if (kmax < 2 || kmax >= GMRES_KMAX) {
    h2b_set_error("h2b_solve_gmres_noalloc: kmax %u outside 2..%d", kmax, GMRES_KMAX - 1);
    return H2B_ERR_ARG;
  }
  ComboNA combo;
  combo.nterms = nterms;
  for (uint32_t i = 0; i < nterms; i++) {
    if (!ops[i] || ops[i]->rt.nidx != ops[0]->rt.nidx || ops[i]->ct.nidx != ops[0]->ct.nidx ||
        ops[i]->cx != ops[0]->cx || ops[i]->rt.nidx != ops[i]->ct.nidx) {
      h2b_set_error("h2b_solve_gmres_noalloc: operators must be square, of equal size and field");
      return H2B_ERR_ARG;
    }
    combo.ops[i] = ops[i];
    combo.cre[i] = coef[2 * i];
    combo.cim[i] = coef[2 * i + 1];
  }
  const h2b_h2matrix *A0 = ops[0];
  cudaStream_t st = A0->st;
  const uint32_t n = A0->rt.nidx;
  const size_t W = A0->cx ? 2 : 1;

  const uint32_t sizes[1] = {n};
  uint32_t nblocks = 0;
  const size_t ndoubles = h2b_gmres_workspace(A0->cx, 1, sizes, kmax, &nblocks) + 2 * W * (size_t) n;
  const size_t need = sizeof(double) * ndoubles + 512;
  if (need > H2B_NOALLOC_SCRATCH_BYTES) {
    h2b_set_error("h2b_solve_gmres_noalloc: needs %zu bytes of work space for n = %u, kmax = %u; "
                  "the fixed work space holds %u bytes (use h2b_solve_gmres)",
                  need, n, kmax, (unsigned) H2B_NOALLOC_SCRATCH_BYTES);
    return H2B_ERR_ARG;
  }
  void *base = nullptr;
  int rc = scratch_address(&base);
  if (rc != H2B_OK) return rc;
  double *db = (double *) base, *dx = db + W * n;
  GmresDev g;
  memset(&g, 0, sizeof(g));
  GmresSys sys;
  std::vector<uint32_t> blk(nblocks);  // host table, copied into the work space
  h2b_gmres_layout(&g, dx + W * n, A0->cx, 1, sizes, kmax, &sys, blk.data());
  g.eps = eps;
  StreamDrain drain{st};
  drain.armed = true;  // from here on, every return waits for the work queued on st
  // the scratch keeps the previous call's contents: clear what must start at zero
  H2B_CUDA_TRY(cudaMemsetAsync(g.T, 0, sizeof(double) * 2 * (size_t) kmax * kmax, st));
  H2B_CUDA_TRY(cudaMemsetAsync(g.state, 0, sizeof(GmresState), st));
  H2B_CUDA_TRY(cudaMemcpyAsync((void *) g.sys, &sys, sizeof(GmresSys), cudaMemcpyHostToDevice, st));
  H2B_CUDA_TRY(cudaMemcpyAsync((void *) g.blk, blk.data(), sizeof(uint32_t) * nblocks,
                               cudaMemcpyHostToDevice, st));
  H2B_CUDA_TRY(cudaMemcpyAsync(db, b, sizeof(double) * W * n, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaMemcpyAsync(dx, x, sizeof(double) * W * n, cudaMemcpyDefault, st));

  // host-driven loop: one step launch sequence per iteration, the residual estimate read back
  GmresOp op{&combo, combo_apply_na, nullptr};
  GmresState hs;
  auto read_state = [&]() -> int {
    H2B_CUDA_TRY(cudaMemcpyAsync(&hs, g.state, sizeof(GmresState), cudaMemcpyDeviceToHost, st));
    H2B_CUDA_TRY(cudaStreamSynchronize(st));
    return H2B_OK;
  };
  if ((rc = h2b_gmres_bnorm(&g, db, st)) != H2B_OK) return rc;
  if ((rc = h2b_gmres_init(&g, &op, db, dx, GMRES_SEL_ALL, st)) != H2B_OK) return rc;
  if ((rc = read_state()) != H2B_OK) return rc;
  const double bnorm = hs.bnorm;
  double err = hs.err;
  uint32_t k = 0, iter = 0;
  while (err > eps * bnorm && iter + 1 != maxiter) {
    if (k + 1 >= kmax) {
      if ((rc = h2b_gmres_finish(&g, &op, db, dx, GMRES_SEL_ALL, st)) != H2B_OK) return rc;
      k = 0;
    }
    if ((rc = h2b_gmres_step(&g, &op, st)) != H2B_OK) return rc;
    k++;
    if ((rc = read_state()) != H2B_OK) return rc;
    if (hs.k != k || !(hs.err == hs.err)) {
      h2b_set_error("h2b_solve_gmres_noalloc: inconsistent solver state after %u iterations",
                    iter + 1);
      return H2B_ERR_INTERNAL;
    }
    err = hs.err;
    iter++;
  }
  if ((rc = h2b_gmres_update(&g, dx, GMRES_SEL_ALL, st)) != H2B_OK) return rc;
  H2B_CUDA_TRY(cudaMemcpyAsync(x, dx, sizeof(double) * W * n, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  drain.armed = false;
  return (int) iter;
}
