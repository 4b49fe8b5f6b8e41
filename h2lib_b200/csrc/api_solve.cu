// C-ABI implementation: GMRES on combinations of H2 matrices, residuals, Laplace test data
// (L2 projection of the harmonic Dirichlet datum, L2 error of the Neumann trace).
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "api_h2.h"
#include "gmres.h"

namespace {

struct Combo {
  uint32_t nterms;
  const h2b_h2matrix *ops[16];
  double cre[16], cim[16];
  uint32_t nrhs = 1;  // vectors hold nrhs columns of the operator size
  // batched form: all columns in one launch sequence per term (work: h2b_mvm_work_doubles),
  // optionally skipping the columns of finished systems (mask[segment + r * nseg])
  double *work = nullptr;
  const uint32_t *mask = nullptr;
  uint32_t nseg = 1;
  // two operators on one structure with equal coupling matrices and row bases (a double layer
  // beside its single layer): applied as one product that reads those once
  bool pair = false;
};

// Two matrices built on one structure (h2b_h2matrix_new_like) for the same surface, PDE,
// wavenumber, interpolation order and row basis, neither an adjoint double layer: their coupling
// matrices (the kernel at the interpolation points) and their row bases (Lagrange polynomials)
// are computed from the same data by the same kernels, so they are equal.
static bool same_farfield(const h2b_h2matrix *a, const h2b_h2matrix *b) {
  const h2b_h2matrix *oa = a->shared ? a->owner : a, *ob = b->shared ? b->owner : b;
  const h2b_bem *ea = a->bem, *eb = b->bem;
  return oa == ob && a->cx == b->cx && a->m == b->m && ea->s == eb->s && ea->pde == eb->pde &&
         ea->k_re == eb->k_re && ea->k_im == eb->k_im && ea->kconst == eb->kconst &&
         ea->q == eb->q && ea->row_basis == eb->row_basis && ea->layer != H2B_ADLP &&
         eb->layer != H2B_ADLP;
}

template <bool SINGLE>
int combo_apply_t(void *ctx, const double *x, double *y, double ar, double ai, cudaStream_t st) {
  const Combo *c = (const Combo *) ctx;
  const size_t col = (size_t) (c->ops[0]->cx ? 2 : 1) * c->ops[0]->rt.nidx;
  if (c->pair && !c->mask && (c->nrhs == 1 || !c->work)) {
    const double a0r = ar * c->cre[0] - ai * c->cim[0], a0i = ar * c->cim[0] + ai * c->cre[0];
    const double a1r = ar * c->cre[1] - ai * c->cim[1], a1i = ar * c->cim[1] + ai * c->cre[1];
    for (uint32_t r = 0; r < c->nrhs; r++) {
      int rc = h2b_mvm_launch_pair(&c->ops[0]->mvm, &c->ops[1]->mvm, SINGLE ? 1 : 0, x + r * col,
                                   y + r * col, a0r, a0i, a1r, a1i, c->work, st);
      if (rc != H2B_OK) return rc;
    }
    return H2B_OK;
  }
  if (c->work) {
    for (uint32_t i = 0; i < c->nterms; i++) {
      const double br = ar * c->cre[i] - ai * c->cim[i], bi = ar * c->cim[i] + ai * c->cre[i];
      int rc = h2b_mvm_launch_batch(&c->ops[i]->mvm, SINGLE ? 1 : 0, c->nrhs, x, col, y, col, br,
                                    bi, c->work, c->mask, c->nseg, st);
      if (rc != H2B_OK) return rc;
    }
    return H2B_OK;
  }
  for (uint32_t r = 0; r < c->nrhs; r++)
    for (uint32_t i = 0; i < c->nterms; i++) {
      const double br = ar * c->cre[i] - ai * c->cim[i], bi = ar * c->cim[i] + ai * c->cre[i];
      int rc = SINGLE ? h2b_mvm_launch_single(&c->ops[i]->mvm, x + r * col, y + r * col, br, bi, st)
                      : h2b_mvm_launch(&c->ops[i]->mvm, x + r * col, y + r * col, br, bi, st);
      if (rc != H2B_OK) return rc;
    }
  return H2B_OK;
}

int combo_apply(void *ctx, const double *x, double *y, double ar, double ai, cudaStream_t st) {
  return combo_apply_t<false>(ctx, x, y, ar, ai, st);
}
int combo_apply_single(void *ctx, const double *x, double *y, double ar, double ai,
                       cudaStream_t st) {
  return combo_apply_t<true>(ctx, x, y, ar, ai, st);
}

int check_ops(uint32_t nterms, const h2b_h2matrix *const *ops, const double *coef, Combo *c) {
  if (nterms < 1 || nterms > 16 || !ops || !coef) {
    h2b_set_error("GMRES: between 1 and 16 operators are supported");
    return H2B_ERR_ARG;
  }
  c->nterms = nterms;
  for (uint32_t i = 0; i < nterms; i++) {
    if (!ops[i]) {
      h2b_set_error("GMRES: operator %u is NULL", i);
      return H2B_ERR_ARG;
    }
    if (ops[i]->rt.nidx != ops[0]->rt.nidx || ops[i]->ct.nidx != ops[0]->ct.nidx ||
        ops[i]->cx != ops[0]->cx || ops[i]->rt.nidx != ops[i]->ct.nidx) {
      h2b_set_error("GMRES: operators must be square, of equal size and field");
      return H2B_ERR_ARG;
    }
    c->ops[i] = ops[i];
    c->cre[i] = coef[2 * i];
    c->cim[i] = coef[2 * i + 1];
  }
  c->pair = nterms == 2 && same_farfield(ops[0], ops[1]);
  return H2B_OK;
}

struct DevBuf {
  void *p = nullptr;
  cudaStream_t st = nullptr;
  ~DevBuf() {
    if (p) cudaFreeAsync(p, st);
  }
};

}  // namespace

// Solve a batch of independent systems that share the operator (ops, coef) on the row ranges
// seg_off[s] .. seg_off[s+1] of the vectors (each segment must be closed under the operator:
// a forest H2 matrix, one block per surface).  iters[s] receives the step count of system s.
// With nrhs > 1 the vectors hold nrhs columns and system (s, r) is segment s of column r
// (iters[s + r * nseg]).  mixed: Arnoldi steps with the FP32 copies of the matrices, (re)start
// residuals and the final stopping test in FP64.
// True when the tree is a forest whose surfaces (roots, in order) hold exactly the index ranges
// seg_off[m] .. seg_off[m+1]: then the operator is block diagonal on the segments and a surface's
// blocks only touch its own segment.
static bool forest_matches(const DevCTree &t, uint32_t nseg, const uint32_t *seg_off) {
  if (t.roots.size() != nseg || !t.h_idx) return false;
  for (uint32_t m = 0; m < nseg; m++) {
    const uint32_t r = t.roots[m], lo = seg_off[m], hi = seg_off[m + 1];
    if (t.h_off[r] != lo || t.h_size[r] != hi - lo) return false;
    for (uint32_t i = lo; i < hi; i++)
      if (t.h_idx[i] < lo || t.h_idx[i] >= hi) return false;
  }
  return true;
}

static int solve_segments(Combo &combo, uint32_t nseg, const uint32_t *seg_off, uint32_t nrhs,
                          const double *b, double *x, double eps, uint32_t maxiter,
                          uint32_t kmax, int mixed, int unitary, uint32_t *iters,
                          const char *who) {
  const h2b_h2matrix *A0 = combo.ops[0];
  cudaStream_t st = A0->st;
  const uint32_t n1 = A0->rt.nidx;
  const size_t W = A0->cx ? 2 : 1;
  if (nrhs == 0 || (uint64_t) n1 * nrhs > 0xFFFFFFFFull) {
    h2b_set_error("%s: %u right-hand sides of size %u", who, nrhs, n1);
    return H2B_ERR_ARG;
  }
  const uint32_t n = n1 * nrhs;
  combo.nrhs = nrhs;
  if (mixed)
    for (uint32_t i = 0; i < combo.nterms; i++)
      if (!combo.ops[i]->mvm.fS) {
        h2b_set_error("%s: operator %u has no FP32 copy (h2b_h2matrix_make_single)", who, i);
        return H2B_ERR_ARG;
      }
  if (kmax < 2 || kmax >= GMRES_KMAX) {
    h2b_set_error("%s: kmax %u outside 2..%d", who, kmax, GMRES_KMAX - 1);
    return H2B_ERR_ARG;
  }
  if (nseg == 0 || !seg_off || seg_off[0] != 0 || seg_off[nseg] != n1) {
    h2b_set_error("%s: segments must start at 0 and end at the operator size %u", who, n1);
    return H2B_ERR_ARG;
  }
  std::vector<uint32_t> sizes((size_t) nseg * nrhs);
  for (uint32_t s = 0; s < nseg; s++) {
    if (seg_off[s + 1] <= seg_off[s]) {
      h2b_set_error("%s: segment %u is empty or the offsets decrease", who, s);
      return H2B_ERR_ARG;
    }
    for (uint32_t r = 0; r < nrhs; r++) sizes[s + (size_t) r * nseg] = seg_off[s + 1] - seg_off[s];
  }
  const uint32_t nsys = nseg * nrhs;
  uint32_t nblocks = 0;
  const size_t nws = h2b_gmres_workspace(A0->cx, nsys, sizes.data(), kmax, &nblocks);
  DevBuf buf;
  buf.st = st;
  H2B_CUDA_TRY(cudaMallocAsync(&buf.p, sizeof(double) * (nws + 2 * W * (size_t) n) + 512, st));
  GmresDev g;
  memset(&g, 0, sizeof(g));
  std::vector<GmresSys> sys(nsys);
  std::vector<uint32_t> blk(nblocks);
  double *db = (double *) buf.p, *dx = db + W * n;
  h2b_gmres_layout(&g, dx + W * n, A0->cx, nsys, sizes.data(), kmax, sys.data(), blk.data());
  g.eps = eps;
  g.mixed = mixed;
  g.unitary = unitary;
  H2B_CUDA_TRY(cudaMemcpyAsync((void *) g.sys, sys.data(), sizeof(GmresSys) * nsys,
                               cudaMemcpyHostToDevice, st));
  H2B_CUDA_TRY(cudaMemcpyAsync((void *) g.blk, blk.data(), sizeof(uint32_t) * nblocks,
                               cudaMemcpyHostToDevice, st));
  H2B_CUDA_TRY(cudaMemcpyAsync(db, b, sizeof(double) * W * n, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaMemcpyAsync(dx, x, sizeof(double) * W * n, cudaMemcpyDefault, st));
  // All columns of a term in one launch sequence; on a forest whose surfaces are exactly the
  // segments, the products skip the columns of systems that have stopped.
  DevBuf work;
  work.st = st;
  bool forest = nseg > 1;
  size_t nwork = 0;
  for (uint32_t i = 0; i < combo.nterms; i++) {
    const h2b_h2matrix *h = combo.ops[i];
    forest = forest && forest_matches(h->rt, nseg, seg_off) && forest_matches(h->ct, nseg, seg_off);
    nwork = std::max(nwork, h2b_mvm_work_doubles(&h->mvm, nrhs));
  }
  if (combo.pair) nwork = std::max(nwork, h2b_mvm_pair_work_doubles(&combo.ops[0]->mvm));
  H2B_CUDA_TRY(cudaMallocAsync(&work.p, sizeof(double) * nwork, st));
  combo.work = (double *) work.p;
  combo.mask = forest ? g.mask : nullptr;
  combo.nseg = nseg;
  GmresOp op{(void *) &combo, combo_apply, mixed ? combo_apply_single : nullptr};
  std::vector<GmresState> hs(nsys);
  int rc = h2b_gmres_run(&g, &op, db, dx, maxiter, st, hs.data());
  if (rc != H2B_OK) return rc;
  for (uint32_t s = 0; s < nsys; s++) {
    if (hs[s].nan) {
      h2b_set_error("%s: residual estimate of system %u is NaN after %u iterations", who, s,
                    hs[s].iter);
      return H2B_ERR_INTERNAL;
    }
    if (iters) iters[s] = hs[s].iter;
  }
  H2B_CUDA_TRY(cudaMemcpyAsync(x, dx, sizeof(double) * W * n, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  for (uint32_t i = 0; i < combo.nterms; i++)
    if ((rc = h2b_h2_check_mv_error(combo.ops[i])) != H2B_OK) return rc;
  return H2B_OK;
}

extern "C" int h2b_solve_gmres(uint32_t nterms, const h2b_h2matrix *const *ops,
                               const double *coef, const double *b, double *x, double eps,
                               uint32_t maxiter, uint32_t kmax) {
  Combo combo;
  int rc = check_ops(nterms, ops, coef, &combo);
  if (rc != H2B_OK) return rc;
  if (!b || !x) {
    h2b_set_error("h2b_solve_gmres: NULL vector");
    return H2B_ERR_ARG;
  }
  const uint32_t seg[2] = {0, ops[0]->rt.nidx};
  uint32_t iter = 0;
  rc = solve_segments(combo, 1, seg, 1, b, x, eps, maxiter, kmax, 0, 0, &iter,
                      "h2b_solve_gmres");
  return rc == H2B_OK ? (int) iter : rc;
}

extern "C" int h2b_solve_gmres_mixed(uint32_t nterms, const h2b_h2matrix *const *ops,
                                     const double *coef, const double *b, double *x, double eps,
                                     uint32_t maxiter, uint32_t kmax) {
  Combo combo;
  int rc = check_ops(nterms, ops, coef, &combo);
  if (rc != H2B_OK) return rc;
  if (!b || !x) {
    h2b_set_error("h2b_solve_gmres_mixed: NULL vector");
    return H2B_ERR_ARG;
  }
  const uint32_t seg[2] = {0, ops[0]->rt.nidx};
  uint32_t iter = 0;
  rc = solve_segments(combo, 1, seg, 1, b, x, eps, maxiter, kmax, 1, 1, &iter,
                      "h2b_solve_gmres_mixed");
  return rc == H2B_OK ? (int) iter : rc;
}

extern "C" int h2b_solve_gmres_batch(uint32_t nterms, const h2b_h2matrix *const *ops,
                                     const double *coef, uint32_t systems,
                                     const uint32_t *system_off, uint32_t nrhs, const double *b,
                                     double *x, double eps, uint32_t maxiter, uint32_t kmax,
                                     uint32_t flags, uint32_t *iterations) {
  Combo combo;
  int rc = check_ops(nterms, ops, coef, &combo);
  if (rc != H2B_OK) return rc;
  if (!b || !x) {
    h2b_set_error("h2b_solve_gmres_batch: NULL vector");
    return H2B_ERR_ARG;
  }
  if (flags & ~(H2B_SOLVE_MIXED | H2B_SOLVE_UNITARY)) {
    h2b_set_error("h2b_solve_gmres_batch: unknown flags 0x%x", flags);
    return H2B_ERR_ARG;
  }
  // the mixed iteration always uses the unitary rotations: its restarts compare the estimate
  // with the FP64 residual, which only an exact estimate makes cheap
  const int mixed = (flags & H2B_SOLVE_MIXED) ? 1 : 0;
  const int unitary = (mixed || (flags & H2B_SOLVE_UNITARY)) ? 1 : 0;
  return solve_segments(combo, systems, system_off, nrhs, b, x, eps, maxiter, kmax, mixed,
                        unitary, iterations, "h2b_solve_gmres_batch");
}

// ------------------------------------------------------------------------------------------
// residual norm
// ------------------------------------------------------------------------------------------

namespace {

__global__ void sumsq_kernel(const double *v, size_t n, double *out) {
  double s = 0.0;
  for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n;
       i += (size_t) gridDim.x * blockDim.x)
    s += v[i] * v[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

}  // namespace

extern "C" int h2b_residual_norm(uint32_t nterms, const h2b_h2matrix *const *ops,
                                 const double *coef, const double *b, const double *x,
                                 double *relres) {
  Combo combo;
  int rc = check_ops(nterms, ops, coef, &combo);
  if (rc != H2B_OK) return rc;
  if (!b || !x || !relres) return H2B_ERR_ARG;
  const h2b_h2matrix *A0 = ops[0];
  cudaStream_t st = A0->st;
  const uint32_t n = A0->rt.nidx;
  const size_t W = A0->cx ? 2 : 1;
  DevBuf buf;
  buf.st = st;
  H2B_CUDA_TRY(cudaMallocAsync(&buf.p, sizeof(double) * (2 * W * n + 2), st));
  double *dr = (double *) buf.p, *dx = dr + W * n, *sums = dx + W * n;
  H2B_CUDA_TRY(cudaMemcpyAsync(dr, b, sizeof(double) * W * n, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaMemcpyAsync(dx, x, sizeof(double) * W * n, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaMemsetAsync(sums, 0, 2 * sizeof(double), st));
  sumsq_kernel<<<64, 256, 0, st>>>(dr, W * n, sums);
  if ((rc = combo_apply(&combo, dx, dr, -1.0, 0.0, st)) != H2B_OK) return rc;
  sumsq_kernel<<<64, 256, 0, st>>>(dr, W * n, sums + 1);
  double h[2];
  H2B_CUDA_TRY(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  *relres = sqrt(h[1]) / sqrt(h[0]);
  return H2B_OK;
}

// ------------------------------------------------------------------------------------------
// Laplace test data: projection of 1/|x - z| and L2 error of the Neumann trace
// ------------------------------------------------------------------------------------------

namespace {

struct HarmArgs {
  const TriRec *tri;
  uint32_t nt;
  const double *xs, *ys, *ws, *wsl;  // single-triangle rule
  int ns;
  double z0, z1, z2;
};

__device__ __forceinline__ void tri_point(const TriRec &T, double tx, double sx, double X[3]) {
  const double Ax = 1.0 - tx, Bx = tx - sx, Cx = sx;
#pragma unroll
  for (int d = 0; d < 3; d++) X[d] = T.a[d] * Ax + T.b[d] * Bx + T.c[d] * Cx;
}

// v[vertex] += g_t * sum_q w_l(q) / |x_q - z|   (projectL2_bem3d_l_avector, Library/bem3d.c:9009)
__global__ void project_rhs_kernel(HarmArgs a, double *v) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nt) return;
  const TriRec &T = a.tri[t];
  double s[3] = {0.0, 0.0, 0.0};
  for (int q = 0; q < a.ns; q++) {
    double X[3];
    tri_point(T, a.xs[q], a.ys[q], X);
    const double d0 = X[0] - a.z0, d1 = X[1] - a.z1, d2 = X[2] - a.z2;
    const double f = 1.0 / sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    for (int l = 0; l < 3; l++) s[l] += a.wsl[l * a.ns + q] * f;
  }
  for (int l = 0; l < 3; l++) atomicAdd(&v[T.v[l]], s[l] * T.g);
}

// y = M x for the linear-basis mass matrix (addeval_mass_linear_bem3d, Library/bem3d.c:8878)
__global__ void mass_kernel(const TriRec *tri, uint32_t nt, const double *x, double *y) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const TriRec &T = tri[t];
  const double x0 = x[T.v[0]], x1 = x[T.v[1]], x2 = x[T.v[2]];
  const double c1 = T.g / 24.0, c2 = T.g / 12.0;
  atomicAdd(&y[T.v[0]], c2 * x0 + c1 * (x1 + x2));
  atomicAdd(&y[T.v[1]], c2 * x1 + c1 * (x0 + x2));
  atomicAdd(&y[T.v[2]], c2 * x2 + c1 * (x0 + x1));
}

// diagonal of the linear-basis mass matrix: sum over a vertex's triangles of g / 12
__global__ void mass_diag_kernel(const TriRec *tri, uint32_t nt, double *d) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const TriRec &T = tri[t];
  const double c2 = T.g / 12.0;
  atomicAdd(&d[T.v[0]], c2);
  atomicAdd(&d[T.v[1]], c2);
  atomicAdd(&d[T.v[2]], c2);
}

// z = r / d per column of nv entries (Jacobi preconditioner)
__global__ void jacobi_kernel(double *z, const double *r, const double *d, uint32_t n,
                              uint32_t nv) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    z[i] = r[i] / d[i % nv];
}

__global__ void dot_kernel(const double *a, const double *b, uint32_t n, double *out) {
  double s = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += a[i] * b[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// CG update: x += al p; r -= al ap   with al = rr / pap read from device
__global__ void cg_update_kernel(double *x, double *r, const double *p, const double *ap,
                                 uint32_t n, const double *sc) {
  const double al = sc[0] / sc[1];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += al * p[i];
    r[i] -= al * ap[i];
  }
}

// p = r + (rr_new / rr_old) p
__global__ void cg_dir_kernel(double *p, const double *r, uint32_t n, const double *sc) {
  const double be = sc[2] / sc[0];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = r[i] + be * p[i];
}

// per-triangle (error^2, norm^2) of the Neumann trace -(x - z).n / |x - z|^3
// (normL2diff_l_bem3d, Library/bem3d.c:8954; normL2_bem3d, :8704)
__global__ void l2err_kernel(HarmArgs a, const double *u, double *out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0, nn = 0.0;
  if (t < a.nt) {
    const TriRec &T = a.tri[t];
    for (int q = 0; q < a.ns; q++) {
      double X[3];
      const double tx = a.xs[q], sx = a.ys[q];
      tri_point(T, tx, sx, X);
      const double d0 = X[0] - a.z0, d1 = X[1] - a.z1, d2 = X[2] - a.z2;
      const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
      const double f = -(d0 * T.n[0] + d1 * T.n[1] + d2 * T.n[2]) / (r2 * sqrt(r2));
      const double bf = u[T.v[0]] * (1.0 - tx) + u[T.v[1]] * (tx - sx) + u[T.v[2]] * sx;
      e += a.ws[q] * (f - bf) * (f - bf);
      nn += a.ws[q] * f * f;
    }
    e *= T.g;
    nn *= T.g;
  }
  e = warp_sum(e);
  nn = warp_sum(nn);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[0], e);
    atomicAdd(&out[1], nn);
  }
}

// b[t] = coef * g_t * sum_q w_q exp(i kvec . (x_q - src))  (integrate_bem3d_c_avector,
// Library/bem3d.c:8579, with rhs_dirichlet_plane_helmholtzbem3d, Library/helmholtzbem3d.c:1611)
__global__ void plane_wave_kernel(HarmArgs a, double k0, double k1, double k2, double cre,
                                  double cim, double *b) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nt) return;
  const TriRec &T = a.tri[t];
  double sr = 0.0, si = 0.0;
  for (int q = 0; q < a.ns; q++) {
    double X[3];
    tri_point(T, a.xs[q], a.ys[q], X);
    const double ph = k0 * (X[0] - a.z0) + k1 * (X[1] - a.z1) + k2 * (X[2] - a.z2);
    double s, c;
    sincos(ph, &s, &c);
    sr += a.ws[q] * c;
    si += a.ws[q] * s;
  }
  sr *= T.g;
  si *= T.g;
  b[2 * t] = cre * sr - cim * si;
  b[2 * t + 1] = cre * si + cim * sr;
}

// e^{i k r} / r, the Helmholtz point source of rhs_dirichlet_point_helmholtzbem3d
// (Library/helmholtzbem3d.c:1521), at distance r
__device__ __forceinline__ void point_wave(double k, double r, double &re, double &im) {
  double s, c;
  sincos(k * r, &s, &c);
  re = c / r;
  im = s / r;
}

// Dirichlet datum of a point source at (z0, z1, z2) tested with the basis: b[t] =
// coef g_t sum_q w_q f(x_q) for the constant basis (integrate_bem3d_c_avector,
// Library/bem3d.c:8579), b[v] += coef g_t sum_q w_l(q) f(x_q) over the triangle's vertices v_l
// for the linear basis (integrate_bem3d_l_avector, :8631); f = e^{ik|x-z|} / |x-z|
__global__ void point_source_kernel(HarmArgs a, double k, double cre, double cim, int linear,
                                    double *b) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nt) return;
  const TriRec &T = a.tri[t];
  double sr[3] = {0.0, 0.0, 0.0}, si[3] = {0.0, 0.0, 0.0};
  for (int q = 0; q < a.ns; q++) {
    double X[3];
    tri_point(T, a.xs[q], a.ys[q], X);
    const double d0 = X[0] - a.z0, d1 = X[1] - a.z1, d2 = X[2] - a.z2;
    double fr, fi;
    point_wave(k, sqrt(d0 * d0 + d1 * d1 + d2 * d2), fr, fi);
    if (linear) {
      for (int l = 0; l < 3; l++) {
        sr[l] += a.wsl[l * a.ns + q] * fr;
        si[l] += a.wsl[l * a.ns + q] * fi;
      }
    } else {
      sr[0] += a.ws[q] * fr;
      si[0] += a.ws[q] * fi;
    }
  }
  for (int l = 0; l < (linear ? 3 : 1); l++) {
    const double re = sr[l] * T.g, im = si[l] * T.g;
    const double br = cre * re - cim * im, bi = cre * im + cim * re;
    if (linear) {
      atomicAdd(&b[2 * T.v[l]], br);
      atomicAdd(&b[2 * T.v[l] + 1], bi);
    } else {
      b[2 * t] = br;
      b[2 * t + 1] = bi;
    }
  }
}

// Brakhage-Werner potential u(x) = sum_t w_t int_t (d_n(y) G(x, y) - i eta G(x, y)) dy of the
// density w at points x outside the surface, G the Helmholtz fundamental solution with the
// operator's k (complex), by the single-triangle rule: per quadrature point y_q, with d = x - y_q
// and r = |d|, kconst g_t w_t(q) e^{ikr} / r^3 ((1 - ikr) d.n - i eta r^2); w_t(q) = w[t] w_q for
// the constant basis, sum_l w[v_l] w_l(q) for the linear basis.  One CTA per point, threads over
// triangles, a fixed-order reduction (the same sum on every run).  Evaluation of
// eval_brakhage_werner_c / _l (Tests/test_helmholtzbem3d.c:68 / :134).
constexpr int BW_THREADS = 256;
__global__ void __launch_bounds__(BW_THREADS)
    bw_eval_kernel(HarmArgs a, const double *pts, const double *w, int linear, double kr,
                   double ki, double er, double ei, double kconst, double *out) {
  __shared__ double red[2][BW_THREADS / 32];
  const double *x = pts + 3 * (size_t) blockIdx.x;
  const double x0 = x[0], x1 = x[1], x2 = x[2];
  double ur = 0.0, ui = 0.0;
  for (uint32_t t = threadIdx.x; t < a.nt; t += BW_THREADS) {
    const TriRec &T = a.tri[t];
    double wr[3], wi[3];
    if (linear) {
      for (int l = 0; l < 3; l++) wr[l] = w[2 * T.v[l]], wi[l] = w[2 * T.v[l] + 1];
    } else {
      wr[0] = w[2 * t], wi[0] = w[2 * t + 1];
    }
    double sr = 0.0, si = 0.0;
    for (int q = 0; q < a.ns; q++) {
      double Y[3];
      tri_point(T, a.xs[q], a.ys[q], Y);
      const double d0 = x0 - Y[0], d1 = x1 - Y[1], d2 = x2 - Y[2];
      const double r2 = d0 * d0 + d1 * d1 + d2 * d2, r = sqrt(r2);
      const double dn = d0 * T.n[0] + d1 * T.n[1] + d2 * T.n[2];
      double s, c;
      sincos(kr * r, &s, &c);
      const double e = exp(-ki * r) / (r2 * r);
      // (1 - ikr) dn - i eta r^2 with k = kr + i ki, eta = er + i ei
      const double pr = (1.0 + ki * r) * dn + ei * r2, pi = -kr * r * dn - er * r2;
      const double qr = e * (c * pr - s * pi), qi = e * (c * pi + s * pr);
      // weight of the point: the density at y_q
      double vr, vi;
      if (linear) {
        vr = vi = 0.0;
        for (int l = 0; l < 3; l++) {
          vr += a.wsl[l * a.ns + q] * wr[l];
          vi += a.wsl[l * a.ns + q] * wi[l];
        }
      } else {
        vr = a.ws[q] * wr[0];
        vi = a.ws[q] * wi[0];
      }
      sr += qr * vr - qi * vi;
      si += qr * vi + qi * vr;
    }
    ur += sr * T.g;
    ui += si * T.g;
  }
  ur = warp_sum(ur);
  ui = warp_sum(ui);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = ur;
    red[1][threadIdx.x >> 5] = ui;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a0 = 0.0, a1 = 0.0;
    for (int i = 0; i < BW_THREADS / 32; i++) a0 += red[0][i], a1 += red[1][i];
    out[2 * blockIdx.x] = kconst * a0;
    out[2 * blockIdx.x + 1] = kconst * a1;
  }
}

// Several surfaces (triangle ranges tri_off[s] .. tri_off[s+1]) and right-hand sides: the source
// of (surface s, column r) is zs[3 (s + r nseg)].  Columns of the vertex vectors are nv long.
struct MultiZ {
  const uint32_t *tri_off;
  const double *zs;
  uint32_t nseg, nv;
};

__device__ __forceinline__ uint32_t segment_of(const MultiZ &m, uint32_t t) {
  uint32_t lo = 0, hi = m.nseg;  // tri_off[lo] <= t < tri_off[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (m.tri_off[mid] <= t) lo = mid; else hi = mid;
  }
  return lo;
}

// project_rhs_kernel with the source of the triangle's surface; blockIdx.y = column
__global__ void project_rhs_multi_kernel(HarmArgs a, MultiZ m, double *v) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (t >= a.nt) return;
  const double *z = m.zs + 3 * ((size_t) segment_of(m, t) + (size_t) r * m.nseg);
  const TriRec &T = a.tri[t];
  double s[3] = {0.0, 0.0, 0.0};
  for (int q = 0; q < a.ns; q++) {
    double X[3];
    tri_point(T, a.xs[q], a.ys[q], X);
    const double d0 = X[0] - z[0], d1 = X[1] - z[1], d2 = X[2] - z[2];
    const double f = 1.0 / sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    for (int l = 0; l < 3; l++) s[l] += a.wsl[l * a.ns + q] * f;
  }
  for (int l = 0; l < 3; l++) atomicAdd(&v[(size_t) r * m.nv + T.v[l]], s[l] * T.g);
}

// mass_kernel on every column (blockIdx.y)
__global__ void mass_multi_kernel(const TriRec *tri, uint32_t nt, uint32_t nv, const double *x,
                                  double *y) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const size_t o = (size_t) blockIdx.y * nv;
  const TriRec &T = tri[t];
  const double x0 = x[o + T.v[0]], x1 = x[o + T.v[1]], x2 = x[o + T.v[2]];
  const double c1 = T.g / 24.0, c2 = T.g / 12.0;
  atomicAdd(&y[o + T.v[0]], c2 * x0 + c1 * (x1 + x2));
  atomicAdd(&y[o + T.v[1]], c2 * x1 + c1 * (x0 + x2));
  atomicAdd(&y[o + T.v[2]], c2 * x2 + c1 * (x0 + x1));
}

// l2err_kernel per (surface, column): out[2 (s + r nseg)] += (error^2, norm^2)
__global__ void l2err_multi_kernel(HarmArgs a, MultiZ m, const double *u, double *out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (t >= a.nt) return;
  const uint32_t sg = segment_of(m, t);
  const double *z = m.zs + 3 * ((size_t) sg + (size_t) r * m.nseg);
  const double *ur = u + (size_t) r * m.nv;
  const TriRec &T = a.tri[t];
  double e = 0.0, nn = 0.0;
  for (int q = 0; q < a.ns; q++) {
    double X[3];
    const double tx = a.xs[q], sx = a.ys[q];
    tri_point(T, tx, sx, X);
    const double d0 = X[0] - z[0], d1 = X[1] - z[1], d2 = X[2] - z[2];
    const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
    const double f = -(d0 * T.n[0] + d1 * T.n[1] + d2 * T.n[2]) / (r2 * sqrt(r2));
    const double bf = ur[T.v[0]] * (1.0 - tx) + ur[T.v[1]] * (tx - sx) + ur[T.v[2]] * sx;
    e += a.ws[q] * (f - bf) * (f - bf);
    nn += a.ws[q] * f * f;
  }
  atomicAdd(&out[2 * ((size_t) sg + (size_t) r * m.nseg)], e * T.g);
  atomicAdd(&out[2 * ((size_t) sg + (size_t) r * m.nseg) + 1], nn * T.g);
}

int harm_args(const h2b_bem *bem, const double z[3], double *scratch, HarmArgs *a,
              cudaStream_t st) {
  const h2b_quad &qd = bem->quad;
  const int ns = (int) qd.ns;
  std::vector<double> h(6 * (size_t) ns);
  for (int q = 0; q < ns; q++) {
    h[q] = qd.xs[q];
    h[ns + q] = qd.ys[q];
    h[2 * ns + q] = qd.ws[3 * ns + q];
    for (int l = 0; l < 3; l++) h[(3 + l) * ns + q] = qd.ws[l * ns + q];
  }
  H2B_CUDA_TRY(cudaMemcpyAsync(scratch, h.data(), sizeof(double) * h.size(),
                               cudaMemcpyHostToDevice, st));
  a->tri = bem->s->d_tri;
  a->nt = bem->s->nt;
  a->xs = scratch;
  a->ys = scratch + ns;
  a->ws = scratch + 2 * ns;
  a->wsl = scratch + 3 * ns;
  a->ns = ns;
  a->z0 = z[0];
  a->z1 = z[1];
  a->z2 = z[2];
  return H2B_OK;
}

}  // namespace

extern "C" int h2b_project_l2_harmonic(const h2b_bem *bem, const double z[3], double *w) {
  if (!bem || !z || !w || bem->row_basis != H2B_BASIS_LINEAR) {
    h2b_set_error("h2b_project_l2_harmonic: needs an operator with a linear row basis");
    return H2B_ERR_ARG;
  }
  const h2b_surface *s = bem->s;
  cudaStream_t st = s->stream;
  const uint32_t nv = s->nv, nt = s->nt;
  DevBuf buf;
  buf.st = st;
  H2B_CUDA_TRY(cudaMallocAsync(&buf.p, sizeof(double) * (5 * (size_t) nv + 6 * 64 + 4), st));
  double *v = (double *) buf.p, *x = v + nv, *r = x + nv, *p = r + nv, *ap = p + nv,
         *rule = ap + nv, *sc = rule + 6 * 64;
  HarmArgs a;
  int rc = harm_args(bem, z, rule, &a, st);
  if (rc != H2B_OK) return rc;
  H2B_CUDA_TRY(cudaMemsetAsync(v, 0, sizeof(double) * 2 * nv, st));
  project_rhs_kernel<<<(nt + 127) / 128, 128, 0, st>>>(a, v);
  // CG on M x = v from x = 0 to 1e-15 relative, at most 500 steps (solve_cg_avector,
  // Library/krylovsolvers.c:18 as called by projectL2_bem3d_l_avector)
  H2B_CUDA_TRY(cudaMemcpyAsync(r, v, sizeof(double) * nv, cudaMemcpyDeviceToDevice, st));
  H2B_CUDA_TRY(cudaMemcpyAsync(p, v, sizeof(double) * nv, cudaMemcpyDeviceToDevice, st));
  double hsc[4];
  H2B_CUDA_TRY(cudaMemsetAsync(sc, 0, sizeof(double) * 4, st));
  dot_kernel<<<64, 256, 0, st>>>(r, r, nv, sc);
  H2B_CUDA_TRY(cudaMemcpyAsync(hsc, sc, sizeof(double), cudaMemcpyDeviceToHost, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  const double norm = sqrt(hsc[0]);
  double rr = hsc[0];
  for (uint32_t it = 0; sqrt(rr) > 1e-15 * norm && it + 1 < 500; it++) {
    H2B_CUDA_TRY(cudaMemsetAsync(ap, 0, sizeof(double) * nv, st));
    mass_kernel<<<(nt + 127) / 128, 128, 0, st>>>(s->d_tri, nt, p, ap);
    H2B_CUDA_TRY(cudaMemsetAsync(sc + 1, 0, sizeof(double) * 2, st));
    dot_kernel<<<64, 256, 0, st>>>(p, ap, nv, sc + 1);
    cg_update_kernel<<<64, 256, 0, st>>>(x, r, p, ap, nv, sc);
    dot_kernel<<<64, 256, 0, st>>>(r, r, nv, sc + 2);
    cg_dir_kernel<<<64, 256, 0, st>>>(p, r, nv, sc);
    H2B_CUDA_TRY(cudaMemcpyAsync(sc, sc + 2, sizeof(double), cudaMemcpyDeviceToDevice, st));
    H2B_CUDA_TRY(cudaMemcpyAsync(hsc, sc, sizeof(double), cudaMemcpyDeviceToHost, st));
    H2B_CUDA_TRY(cudaStreamSynchronize(st));
    rr = hsc[0];
  }
  H2B_CUDA_TRY(cudaMemcpyAsync(w, x, sizeof(double) * nv, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  return H2B_OK;
}

extern "C" int h2b_l2_error_harmonic(const h2b_bem *bem, const double z[3], const double *u,
                                     double *err, double *norm) {
  if (!bem || !z || !u || !err || !norm) {
    h2b_set_error("h2b_l2_error_harmonic: NULL argument");
    return H2B_ERR_ARG;
  }
  const h2b_surface *s = bem->s;
  cudaStream_t st = s->stream;
  DevBuf buf;
  buf.st = st;
  H2B_CUDA_TRY(cudaMallocAsync(&buf.p, sizeof(double) * ((size_t) s->nv + 6 * 64 + 2), st));
  double *du = (double *) buf.p, *rule = du + s->nv, *out = rule + 6 * 64;
  HarmArgs a;
  int rc = harm_args(bem, z, rule, &a, st);
  if (rc != H2B_OK) return rc;
  H2B_CUDA_TRY(cudaMemcpyAsync(du, u, sizeof(double) * s->nv, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double) * 2, st));
  l2err_kernel<<<(s->nt + 127) / 128, 128, 0, st>>>(a, du, out);
  double h[2];
  H2B_CUDA_TRY(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  *err = sqrt(h[0]);
  *norm = sqrt(h[1]);
  return H2B_OK;
}

// Device copies of the surface offsets and sources of a multi-surface call.
static int multi_args(const h2b_bem *bem, uint32_t nseg, const uint32_t *tri_off, uint32_t nrhs,
                      const double *zs, void *dev, MultiZ *m, cudaStream_t st) {
  if (nseg == 0 || nrhs == 0 || !tri_off || !zs || tri_off[0] != 0 ||
      tri_off[nseg] != bem->s->nt) {
    h2b_set_error("harmonic data: triangle offsets must run from 0 to %u", bem->s->nt);
    return H2B_ERR_ARG;
  }
  for (uint32_t s = 0; s < nseg; s++)
    if (tri_off[s + 1] < tri_off[s]) {
      h2b_set_error("harmonic data: triangle offsets decrease at surface %u", s);
      return H2B_ERR_ARG;
    }
  uint32_t *doff = (uint32_t *) dev;
  double *dz = (double *) (((uintptr_t) (doff + nseg + 1) + 15) & ~(uintptr_t) 15);
  H2B_CUDA_TRY(cudaMemcpyAsync(doff, tri_off, sizeof(uint32_t) * (nseg + 1),
                               cudaMemcpyHostToDevice, st));
  H2B_CUDA_TRY(cudaMemcpyAsync(dz, zs, sizeof(double) * 3 * (size_t) nseg * nrhs,
                               cudaMemcpyHostToDevice, st));
  m->tri_off = doff;
  m->zs = dz;
  m->nseg = nseg;
  m->nv = bem->s->nv;
  return H2B_OK;
}

static size_t multi_bytes(uint32_t nseg, uint32_t nrhs) {
  return sizeof(uint32_t) * (nseg + 1) + 16 + sizeof(double) * 3 * (size_t) nseg * nrhs;
}

extern "C" int h2b_project_l2_harmonic_multi(const h2b_bem *bem, uint32_t surfaces,
                                             const uint32_t *triangle_off, uint32_t nrhs,
                                             const double *zs, double *w) {
  if (!bem || !w || bem->row_basis != H2B_BASIS_LINEAR) {
    h2b_set_error("h2b_project_l2_harmonic_multi: needs an operator with a linear row basis");
    return H2B_ERR_ARG;
  }
  const h2b_surface *s = bem->s;
  cudaStream_t st = s->stream;
  const uint32_t nv = s->nv, nt = s->nt;
  const size_t n = (size_t) nv * (nrhs ? nrhs : 1);
  DevBuf buf;
  buf.st = st;
  H2B_CUDA_TRY(cudaMallocAsync(&buf.p, sizeof(double) * (6 * n + nv + 6 * 64 + 4) +
                                           multi_bytes(surfaces, nrhs) + 64, st));
  double *v = (double *) buf.p, *x = v + n, *r = x + n, *p = r + n, *ap = p + n, *zv = ap + n,
         *dg = zv + n, *rule = dg + nv, *sc = rule + 6 * 64;
  HarmArgs a;
  MultiZ m;
  const double z0[3] = {0.0, 0.0, 0.0};
  int rc = harm_args(bem, z0, rule, &a, st);
  if (rc == H2B_OK) rc = multi_args(bem, surfaces, triangle_off, nrhs, zs, sc + 4, &m, st);
  if (rc != H2B_OK) return rc;
  H2B_CUDA_TRY(cudaMemsetAsync(v, 0, sizeof(double) * 2 * n, st));
  project_rhs_multi_kernel<<<dim3((nt + 127) / 128, nrhs), 128, 0, st>>>(a, m, v);
  // CG on the stacked block-diagonal mass system to the tolerance of h2b_project_l2_harmonic,
  // preconditioned by the mass matrix's diagonal: the surfaces' element sizes differ, and plain CG
  // on their union converges at the pace of the worst-scaled block (about 1000 steps for the
  // 256 ellipsoids of the batched workload, 32 with the diagonal)
  const uint32_t un = (uint32_t) n;
  H2B_CUDA_TRY(cudaMemsetAsync(dg, 0, sizeof(double) * nv, st));
  mass_diag_kernel<<<(nt + 127) / 128, 128, 0, st>>>(s->d_tri, nt, dg);
  H2B_CUDA_TRY(cudaMemcpyAsync(r, v, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  jacobi_kernel<<<64, 256, 0, st>>>(zv, r, dg, un, nv);
  H2B_CUDA_TRY(cudaMemcpyAsync(p, zv, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  double hsc[4];
  H2B_CUDA_TRY(cudaMemsetAsync(sc, 0, sizeof(double) * 4, st));
  dot_kernel<<<64, 256, 0, st>>>(r, zv, un, sc);
  dot_kernel<<<64, 256, 0, st>>>(r, r, un, sc + 3);
  H2B_CUDA_TRY(cudaMemcpyAsync(hsc, sc + 3, sizeof(double), cudaMemcpyDeviceToHost, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  const double norm = sqrt(hsc[0]);
  double rr = hsc[0];
  for (uint32_t it = 0; sqrt(rr) > 1e-15 * norm && it + 1 < 500; it++) {
    H2B_CUDA_TRY(cudaMemsetAsync(ap, 0, sizeof(double) * n, st));
    mass_multi_kernel<<<dim3((nt + 127) / 128, nrhs), 128, 0, st>>>(s->d_tri, nt, nv, p, ap);
    H2B_CUDA_TRY(cudaMemsetAsync(sc + 1, 0, sizeof(double) * 3, st));
    dot_kernel<<<64, 256, 0, st>>>(p, ap, un, sc + 1);
    cg_update_kernel<<<64, 256, 0, st>>>(x, r, p, ap, un, sc);  // al = (r.z) / (p.Ap)
    jacobi_kernel<<<64, 256, 0, st>>>(zv, r, dg, un, nv);
    dot_kernel<<<64, 256, 0, st>>>(r, zv, un, sc + 2);
    dot_kernel<<<64, 256, 0, st>>>(r, r, un, sc + 3);
    cg_dir_kernel<<<64, 256, 0, st>>>(p, zv, un, sc);  // p = z + (r.z)_new / (r.z) p
    H2B_CUDA_TRY(cudaMemcpyAsync(sc, sc + 2, sizeof(double), cudaMemcpyDeviceToDevice, st));
    H2B_CUDA_TRY(cudaMemcpyAsync(hsc, sc + 3, sizeof(double), cudaMemcpyDeviceToHost, st));
    H2B_CUDA_TRY(cudaStreamSynchronize(st));
    rr = hsc[0];
  }
  H2B_CUDA_TRY(cudaMemcpyAsync(w, x, sizeof(double) * n, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  return H2B_OK;
}

extern "C" int h2b_l2_error_harmonic_multi(const h2b_bem *bem, uint32_t surfaces,
                                           const uint32_t *triangle_off, uint32_t nrhs,
                                           const double *zs, const double *u, double *err,
                                           double *norm) {
  if (!bem || !u || !err || !norm) {
    h2b_set_error("h2b_l2_error_harmonic_multi: NULL argument");
    return H2B_ERR_ARG;
  }
  const h2b_surface *s = bem->s;
  cudaStream_t st = s->stream;
  const size_t n = (size_t) s->nv * (nrhs ? nrhs : 1), nsys = (size_t) surfaces * nrhs;
  DevBuf buf;
  buf.st = st;
  H2B_CUDA_TRY(cudaMallocAsync(&buf.p, sizeof(double) * (n + 6 * 64 + 2 * nsys) +
                                           multi_bytes(surfaces, nrhs) + 64, st));
  double *du = (double *) buf.p, *rule = du + n, *out = rule + 6 * 64;
  HarmArgs a;
  MultiZ m;
  const double z0[3] = {0.0, 0.0, 0.0};
  int rc = harm_args(bem, z0, rule, &a, st);
  if (rc == H2B_OK) rc = multi_args(bem, surfaces, triangle_off, nrhs, zs, out + 2 * nsys, &m, st);
  if (rc != H2B_OK) return rc;
  H2B_CUDA_TRY(cudaMemcpyAsync(du, u, sizeof(double) * n, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double) * 2 * nsys, st));
  l2err_multi_kernel<<<dim3((s->nt + 127) / 128, nrhs), 128, 0, st>>>(a, m, du, out);
  std::vector<double> h(2 * nsys);
  H2B_CUDA_TRY(cudaMemcpyAsync(h.data(), out, sizeof(double) * 2 * nsys, cudaMemcpyDeviceToHost,
                               st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  for (size_t i = 0; i < nsys; i++) {
    err[i] = sqrt(h[2 * i]);
    norm[i] = sqrt(h[2 * i + 1]);
  }
  return H2B_OK;
}

extern "C" int h2b_integrate_plane_wave(const h2b_bem *bem, const double kvec[3],
                                        const double src[3], double coef_re, double coef_im,
                                        double *b) {
  if (!bem || !kvec || !src || !b || bem->row_basis != H2B_BASIS_CONSTANT) {
    h2b_set_error("h2b_integrate_plane_wave: needs an operator with a constant row basis");
    return H2B_ERR_ARG;
  }
  const h2b_surface *s = bem->s;
  cudaStream_t st = s->stream;
  DevBuf buf;
  buf.st = st;
  H2B_CUDA_TRY(cudaMallocAsync(&buf.p, sizeof(double) * (2 * (size_t) s->nt + 6 * 64), st));
  double *db = (double *) buf.p, *rule = db + 2 * (size_t) s->nt;
  HarmArgs a;
  int rc = harm_args(bem, src, rule, &a, st);
  if (rc != H2B_OK) return rc;
  plane_wave_kernel<<<(s->nt + 127) / 128, 128, 0, st>>>(a, kvec[0], kvec[1], kvec[2], coef_re,
                                                          coef_im, db);
  H2B_CUDA_TRY(cudaGetLastError());
  H2B_CUDA_TRY(cudaMemcpyAsync(b, db, sizeof(double) * 2 * s->nt, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  return H2B_OK;
}

extern "C" int h2b_integrate_point_source(const h2b_bem *bem, const double src[3], double k,
                                          double coef_re, double coef_im, double *b) {
  if (!bem || !src || !b) {
    h2b_set_error("h2b_integrate_point_source: NULL argument");
    return H2B_ERR_ARG;
  }
  const h2b_surface *s = bem->s;
  const int linear = bem->row_basis == H2B_BASIS_LINEAR;
  const size_t n = linear ? s->nv : s->nt;
  cudaStream_t st = s->stream;
  DevBuf buf;
  buf.st = st;
  H2B_CUDA_TRY(cudaMallocAsync(&buf.p, sizeof(double) * (2 * n + 6 * 64), st));
  double *db = (double *) buf.p, *rule = db + 2 * n;
  HarmArgs a;
  int rc = harm_args(bem, src, rule, &a, st);
  if (rc != H2B_OK) return rc;
  if (linear) H2B_CUDA_TRY(cudaMemsetAsync(db, 0, sizeof(double) * 2 * n, st));
  point_source_kernel<<<(s->nt + 127) / 128, 128, 0, st>>>(a, k, coef_re, coef_im, linear, db);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  H2B_CUDA_TRY(cudaMemcpyAsync(b, db, sizeof(double) * 2 * n, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  return H2B_OK;
}

extern "C" int h2b_eval_brakhage_werner(const h2b_bem *bem, uint32_t npoints, const double *points,
                                        const double *w, double eta_re, double eta_im,
                                        double *u) {
  if (!bem || (npoints && (!points || !w || !u))) {
    h2b_set_error("h2b_eval_brakhage_werner: NULL argument");
    return H2B_ERR_ARG;
  }
  if (bem->pde != H2B_HELMHOLTZ) {
    h2b_set_error("h2b_eval_brakhage_werner: needs a Helmholtz operator");
    return H2B_ERR_ARG;
  }
  if (npoints == 0) return H2B_OK;
  if (npoints > (1u << 24)) {
    h2b_set_error("h2b_eval_brakhage_werner: at most 2^24 points per call");
    return H2B_ERR_ARG;
  }
  const h2b_surface *s = bem->s;
  const int linear = bem->col_basis == H2B_BASIS_LINEAR;
  const size_t n = linear ? s->nv : s->nt;
  cudaStream_t st = s->stream;
  DevBuf buf;
  buf.st = st;
  H2B_CUDA_TRY(cudaMallocAsync(&buf.p, sizeof(double) * (2 * n + 5 * (size_t) npoints + 6 * 64),
                               st));
  double *dw = (double *) buf.p, *dp = dw + 2 * n, *du = dp + 3 * (size_t) npoints,
         *rule = du + 2 * (size_t) npoints;
  const double z0[3] = {0.0, 0.0, 0.0};
  HarmArgs a;
  int rc = harm_args(bem, z0, rule, &a, st);
  if (rc != H2B_OK) return rc;
  H2B_CUDA_TRY(cudaMemcpyAsync(dw, w, sizeof(double) * 2 * n, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaMemcpyAsync(dp, points, sizeof(double) * 3 * npoints, cudaMemcpyDefault, st));
  bw_eval_kernel<<<npoints, BW_THREADS, 0, st>>>(a, dp, dw, linear, bem->k_re, bem->k_im, eta_re,
                                                 eta_im, bem->kconst, du);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  H2B_CUDA_TRY(cudaMemcpyAsync(u, du, sizeof(double) * 2 * npoints, cudaMemcpyDefault, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  return H2B_OK;
}
