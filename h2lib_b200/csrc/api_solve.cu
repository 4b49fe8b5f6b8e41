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
};

int combo_apply(void *ctx, const double *x, double *y, double ar, double ai, cudaStream_t st) {
  const Combo *c = (const Combo *) ctx;
  for (uint32_t i = 0; i < c->nterms; i++) {
    const double br = ar * c->cre[i] - ai * c->cim[i], bi = ar * c->cim[i] + ai * c->cre[i];
    int rc = h2b_mvm_launch(&c->ops[i]->mvm, x, y, br, bi, st);
    if (rc != H2B_OK) return rc;
  }
  return H2B_OK;
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
  if (kmax < 2 || kmax >= GMRES_KMAX) {
    h2b_set_error("h2b_solve_gmres: kmax %u outside 2..%d", kmax, GMRES_KMAX - 1);
    return H2B_ERR_ARG;
  }
  const h2b_h2matrix *A0 = ops[0];
  cudaStream_t st = A0->st;
  const uint32_t n = A0->rt.nidx;
  const size_t W = A0->cx ? 2 : 1;

  GmresDev g;
  memset(&g, 0, sizeof(g));
  g.cx = A0->cx;
  g.n = n;
  g.kmax = kmax;
  g.nblocks = (n + 255) / 256;
  g.ldpart = kmax + 1;
  // one allocation for all device state
  const size_t nq = W * (size_t) n * kmax, nT = 2 * (size_t) kmax * kmax, nsm = 2 * (size_t) (kmax + 1);
  const size_t npart = 2 * (size_t) g.nblocks * g.ldpart;
  const size_t total = nq + 2 * kmax + nT + 3 * nsm + 4 * W * (size_t) n + npart + 16;
  DevBuf buf;
  buf.st = st;
  H2B_CUDA_TRY(cudaMallocAsync(&buf.p, sizeof(double) * total + sizeof(GmresState) + 256, st));
  double *p = (double *) buf.p;
  g.qr = p; p += nq;
  g.tau = p; p += 2 * kmax;
  g.T = p; p += nT;
  g.rhat = p; p += nsm;
  g.w = p; p += nsm;
  g.u = p; p += nsm;
  g.q = p; p += W * n;
  g.abuf = p; p += W * n;
  double *db = p; p += W * n;
  double *dx = p; p += W * n;
  g.part = p; p += npart;
  g.state = (GmresState *) (((uintptr_t) p + 255) & ~(uintptr_t) 255);
  H2B_CUDA_TRY(cudaMemsetAsync(g.T, 0, sizeof(double) * nT, st));
  H2B_CUDA_TRY(cudaMemsetAsync(g.state, 0, sizeof(GmresState), st));

  const bool bdev = h2b_is_device_ptr(b), xdev = h2b_is_device_ptr(x);
  H2B_CUDA_TRY(cudaMemcpyAsync(db, b, sizeof(double) * W * n,
                               bdev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  H2B_CUDA_TRY(cudaMemcpyAsync(dx, x, sizeof(double) * W * n,
                               xdev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));

  GmresOp op{&combo, combo_apply};
  GmresState *hs = nullptr;
  H2B_CUDA_TRY(cudaMallocHost(&hs, sizeof(GmresState)));
  struct HostFree {
    GmresState *p;
    ~HostFree() { cudaFreeHost(p); }
  } hf{hs};

  // Default: the whole iteration runs inside one graph (WHILE/IF conditional nodes, the loop
  // condition set on the device).  H2B_GMRES_HOSTLOOP=1 selects a host loop that launches a
  // captured single step and reads the residual estimate after each one.
  cudaGraphExec_t loop_exec = nullptr;
  {
    const char *e = getenv("H2B_GMRES_HOSTLOOP");
    if (!(e && e[0] == '1') && (rc = h2b_gmres_loop_graph(&g, &op, db, dx, st, &loop_exec)) != H2B_OK)
      return rc;
  }
  struct LoopFree {
    cudaGraphExec_t e;
    ~LoopFree() {
      if (e) cudaGraphExecDestroy(e);
    }
  } lf{loop_exec};
  // the step is identical for every k (k is read on the device): capture it once
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (!loop_exec) {
    H2B_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    rc = h2b_gmres_step(&g, &op, st);
    cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (rc != H2B_OK || ce != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (rc == H2B_OK)
        h2b_set_error("h2b_solve_gmres: graph capture failed: %s", cudaGetErrorString(ce));
      return rc == H2B_OK ? H2B_ERR_CUDA : rc;
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
      h2b_set_error("h2b_solve_gmres: graph instantiation failed: %s", cudaGetErrorString(ce));
      return H2B_ERR_CUDA;
    }
  }
  struct ExecFree {
    cudaGraphExec_t e;
    ~ExecFree() {
      if (e) cudaGraphExecDestroy(e);
    }
  } ef{exec};

  auto read_state = [&]() -> int {
    H2B_CUDA_TRY(cudaMemcpyAsync(hs, g.state, sizeof(GmresState), cudaMemcpyDeviceToHost, st));
    H2B_CUDA_TRY(cudaStreamSynchronize(st));
    return H2B_OK;
  };

  if ((rc = h2b_gmres_bnorm(&g, db, st)) != H2B_OK) return rc;
  if ((rc = h2b_gmres_init(&g, &op, db, dx, st)) != H2B_OK) return rc;
  if ((rc = read_state()) != H2B_OK) return rc;
  const double bnorm = hs->bnorm;
  double err = hs->err;
  uint32_t k = 0, iter = 0;
  if (loop_exec) {
    // graph-resident loop: launches of at most kLoopBudget steps until the device stops it
    constexpr uint32_t kLoopBudget = 512;
    hs->tol = eps * bnorm;
    hs->iter = 0;
    hs->maxiter = maxiter;
    hs->nan = 0;
    while (true) {
      hs->budget = kLoopBudget;
      H2B_CUDA_TRY(cudaMemcpyAsync(g.state, hs, sizeof(GmresState), cudaMemcpyHostToDevice, st));
      H2B_CUDA_TRY(cudaGraphLaunch(loop_exec, st));
      if ((rc = read_state()) != H2B_OK) return rc;
      if (hs->nan) {
        h2b_set_error("h2b_solve_gmres: residual estimate is NaN after %u iterations", hs->iter);
        return H2B_ERR_INTERNAL;
      }
      if (!(hs->err > hs->tol) || (maxiter != 0 && hs->iter + 1 == maxiter)) break;
      if (hs->budget != 0) {
        h2b_set_error("h2b_solve_gmres: device loop stopped early at iteration %u", hs->iter);
        return H2B_ERR_INTERNAL;
      }
    }
    iter = hs->iter;
    err = hs->err;
  }
  while (!loop_exec && err > eps * bnorm && iter + 1 != maxiter) {
    if (k + 1 >= kmax) {
      if ((rc = h2b_gmres_finish(&g, &op, db, dx, st)) != H2B_OK) return rc;
      k = 0;
    }
    H2B_CUDA_TRY(cudaGraphLaunch(exec, st));
    k++;
    if ((rc = read_state()) != H2B_OK) return rc;
    if (hs->k != k) {
      h2b_set_error("h2b_solve_gmres: device step counter %u != %u", hs->k, k);
      return H2B_ERR_INTERNAL;
    }
    err = hs->err;
    if (!(err == err)) {
      h2b_set_error("h2b_solve_gmres: residual estimate is NaN after %u iterations", iter + 1);
      return H2B_ERR_INTERNAL;
    }
    iter++;
  }
  if ((rc = h2b_gmres_finish(&g, &op, db, dx, st)) != H2B_OK) return rc;
  H2B_CUDA_TRY(cudaMemcpyAsync(x, dx, sizeof(double) * W * n,
                               xdev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  return (int) iter;
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
