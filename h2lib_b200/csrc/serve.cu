// Device-resident solve server: continuous admission of Dirichlet BEM solves (sm_100a).
//
// Requests (a surface mesh, a PDE, boundary data, a tolerance) are queued on submission.  A pool
// of `slots` worker threads takes them in arrival order as soon as a slot is free and the
// request's device-memory estimate fits the remaining HBM budget.  A worker also takes the queued
// requests that can share the first one's operator (Laplace problems with the same solver
// settings, up to the budget and the batch limits): their meshes become one forest H2 matrix
// (one assembly, one batched GMRES in which every request keeps its own Krylov space and stop).
// Each admitted request (or batch) builds its trees on the host, then runs structure upload,
// assembly, right-hand side and GMRES on its own CUDA streams.  Requests that arrive while others are running are admitted as slots and
// memory free up, and the kernels of all running requests overlap on the device (every handle
// owns a non-blocking stream; device memory is stream-ordered, so one request's allocations and
// frees never synchronise the device under another).  The H2 matrices and the Krylov state of a
// request stay on the device from assembly to the end of its solve.
//
// Problems:
//   Laplace   interior Dirichlet problem of the harmonic u = 1/|x - z| (z outside the surface):
//             V du/dn = (K + M/2) g_D, piecewise-linear basis, q = 2/4, leaf 64, eta 1.4, m = 4
//             (the discretisation of Tests/test_laplacebem3d.c as used by the reference's
//             Dirichlet tests); the solution is the Neumann trace.
//   Helmholtz Brakhage-Werner exterior scattering of the plane wave exp(i k d.x):
//             ((K + M/2) - i k V) u = -g, piecewise-constant basis, m = 5 (Tests/
//             test_helmholtzbem3d.c:26-65); the solution is complex, interleaved.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "api_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  int64_t id = 0;
  h2b_request desc;
  std::vector<double> x;
  std::vector<uint32_t> t;
  uint64_t est = 0;
  // results
  int status = 1;  // 1 queued, 2 running, 0 done, < 0 error code
  std::vector<double> solution;
  h2b_request_result res;
  char err[256] = {0};
};

}  // namespace

struct h2b_server {
  int device = 0;
  uint32_t slots = 1;
  uint64_t budget = 0, reserved = 0;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req *> queue;
  std::unordered_map<int64_t, Req *> reqs;
  std::vector<std::thread> workers;
  int64_t next_id = 1;
  uint32_t running = 0;
  uint64_t done = 0;
  bool stop = false;
  uint32_t batch_max = 64;  // most requests one worker takes at once (1: no batching)
};

namespace {

double since(const h2b_server *s) {
  return std::chrono::duration<double>(Clock::now() - s->t0).count();
}

// Device memory a request may hold: nearfield, coupling and flattened bases of two operators
// plus the Krylov space, from the mesh size (upper estimate per triangle of the two
// discretisations above, plus a fixed part).
uint64_t estimate_bytes(const h2b_request &r) {
  const uint64_t per_tri = r.pde == H2B_HELMHOLTZ ? 288ull << 10 : 64ull << 10;
  return per_tri * r.triangles + (32ull << 20);
}

constexpr uint32_t kDeviceTreeTriangles = 8192;

// Run one request to the end on the calling (worker) thread.
int run_request(Req *q) {
  auto tick = [] { return Clock::now(); };
  auto secs = [](Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
  };
  const auto c0 = tick();
  const h2b_request &d = q->desc;
  const bool helm = d.pde == H2B_HELMHOLTZ;
  const uint32_t nv = d.vertices, nt = d.triangles;
  std::vector<double> n(3 * (size_t) nt), g(nt);
  int rc = h2b_prepare_surface(nv, q->x.data(), nt, q->t.data(), n.data(), g.data(), nullptr);
  if (rc != H2B_OK) return rc;
  h2b_surface *s = h2b_surface_new(nv, q->x.data(), nt, q->t.data(), n.data(), g.data());
  if (!s) return H2B_ERR_CUDA;
  const int basis = helm ? H2B_BASIS_CONSTANT : H2B_BASIS_LINEAR;
  const uint32_t m = helm ? 5 : 4;
  h2b_bem *slp = h2b_bem_new(s, d.pde, H2B_SLP, basis, basis, 2, 4, helm ? d.k : 0.0, 0.0, 0.0,
                             0.0);
  h2b_bem *dlp = h2b_bem_new(s, d.pde, H2B_DLP, basis, basis, 2, 4, helm ? d.k : 0.0, 0.0, 0.5,
                             0.0);
  // trees of larger meshes on the device (the same trees; faster from about 8k triangles, where
  // the host build's cost outgrows the device build's per-level round trips)
  auto tree_fn = nt >= kDeviceTreeTriangles ? h2b_tree_new_device : h2b_tree_new;
  h2b_tree *tr = (slp && dlp) ? tree_fn(nv, q->x.data(), nt, q->t.data(), basis, basis, 64, 1.4)
                              : nullptr;
  h2b_h2matrix *V = tr ? h2b_h2matrix_new(slp, tr, m) : nullptr;
  h2b_h2matrix *K = V ? h2b_h2matrix_new_like(dlp, V) : nullptr;  // shares V's structure
  // mixed precision: FP32 distant-pair quadrature too (singular pairs stay FP64)
  if (V && K && (d.flags & H2B_SOLVE_MIXED)) {
    h2b_h2matrix_set_precision(V, H2B_FP32);
    h2b_h2matrix_set_precision(K, H2B_FP32);
  }
  const auto c1 = tick();
  const uint32_t nd = helm ? nt : nv;
  const size_t W = helm ? 2 : 1;
  std::vector<double> b(W * nd, 0.0), u(W * nd, 0.0), gD;
  rc = (V && K) ? H2B_OK : H2B_ERR_CUDA;
  if (rc == H2B_OK) {
    // bases and coupling per operator, the nearfield of both in one pass (Laplace and Helmholtz)
    for (h2b_h2matrix *h : {V, K}) {
      if (rc == H2B_OK) rc = h2b_h2matrix_assemble_row_clusterbasis(h);
      if (rc == H2B_OK) rc = h2b_h2matrix_assemble_col_clusterbasis(h);
      if (rc == H2B_OK) rc = h2b_h2matrix_assemble_farfield(h);
    }
    if (rc == H2B_OK) rc = h2b_h2matrix_assemble_nearfield_pair(V, K);
  }
  const auto c2 = tick();
  const h2b_h2matrix *ops[2];
  double coef[4];
  uint32_t nterms = 1;
  if (rc == H2B_OK) {
    if (helm) {
      // b = -int exp(i k d.x) (rhs_dirichlet_plane_helmholtzbem3d), operator (K + M/2) - i k V
      const double kv[3] = {d.k * d.src[0], d.k * d.src[1], d.k * d.src[2]}, o[3] = {0, 0, 0};
      rc = h2b_integrate_plane_wave(slp, kv, o, -1.0, 0.0, b.data());
      ops[0] = K;
      ops[1] = V;
      coef[0] = 1.0;
      coef[1] = 0.0;
      coef[2] = 0.0;
      coef[3] = -d.k;
      nterms = 2;
    } else {
      gD.assign(nv, 0.0);
      rc = h2b_project_l2_harmonic(dlp, d.src, gD.data());
      if (rc == H2B_OK) rc = h2b_h2matrix_addeval(1.0, 0.0, K, gD.data(), b.data());
      ops[0] = V;
      coef[0] = 1.0;
      coef[1] = 0.0;
    }
  }
  const auto c3 = tick();
  const bool mixed = (d.flags & H2B_SOLVE_MIXED) != 0;
  if (rc == H2B_OK && mixed)
    for (uint32_t i = 0; i < nterms && rc == H2B_OK; i++)
      rc = h2b_h2matrix_make_single(const_cast<h2b_h2matrix *>(ops[i]));
  int it = 0;
  if (rc == H2B_OK) {
    // unitary rotations: the stop is decided by the true residual, also for complex systems
    const uint32_t seg[2] = {0, nd};
    uint32_t iters = 0;
    rc = h2b_solve_gmres_batch(nterms, ops, coef, 1, seg, 1, b.data(), u.data(), d.eps,
                               d.maxiter, d.kmax,
                               H2B_SOLVE_UNITARY | (mixed ? H2B_SOLVE_MIXED : 0u), &iters);
    it = (int) iters;
  }
  const auto c4 = tick();
  q->res.t_setup = secs(c0, c1);
  q->res.t_assembly = secs(c1, c2);
  q->res.t_rhs = secs(c2, c3);
  q->res.t_solve = secs(c3, c4);
  double relres = 0.0;
  if (rc == H2B_OK) rc = h2b_residual_norm(nterms, ops, coef, b.data(), u.data(), &relres);
  if (rc == H2B_OK) {
    q->solution.swap(u);
    q->res.iterations = (uint32_t) it;
    q->res.unknowns = nd;
    q->res.rel_residual = relres;
  }
  h2b_h2matrix_del(K);
  h2b_h2matrix_del(V);
  h2b_tree_del(tr);
  h2b_bem_del(dlp);
  h2b_bem_del(slp);
  h2b_surface_del(s);
  return rc;
}

// Requests that can share one operator: Laplace problems with the same solver settings (their
// meshes become one block-diagonal forest H2 matrix and one batched GMRES; each request keeps
// its own Krylov space, restarts and stop, so it ends as it would alone).
bool batchable(const Req *a, const Req *b) {
  return a->desc.pde == H2B_LAPLACE && b->desc.pde == H2B_LAPLACE &&
         a->desc.flags == b->desc.flags && a->desc.eps == b->desc.eps &&
         a->desc.maxiter == b->desc.maxiter && a->desc.kmax == b->desc.kmax;
}

// Run a batch of batchable Laplace requests on the calling worker thread: union mesh, forest
// trees, one assembly of V and K, per-surface right-hand sides, one batched GMRES.
int run_batch(const std::vector<Req *> &qs) {
  auto tick = [] { return Clock::now(); };
  auto secs = [](Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
  };
  const auto c0 = tick();
  const uint32_t ns = (uint32_t) qs.size();
  const h2b_request &d = qs[0]->desc;
  std::vector<uint32_t> voff(ns + 1, 0), toff(ns + 1, 0);
  for (uint32_t i = 0; i < ns; i++) {
    voff[i + 1] = voff[i] + qs[i]->desc.vertices;
    toff[i + 1] = toff[i] + qs[i]->desc.triangles;
  }
  const uint32_t nv = voff[ns], nt = toff[ns];
  std::vector<double> x(3 * (size_t) nv), n(3 * (size_t) nt), g(nt), zs(3 * (size_t) ns);
  std::vector<uint32_t> t(3 * (size_t) nt);
  for (uint32_t i = 0; i < ns; i++) {
    memcpy(x.data() + 3 * (size_t) voff[i], qs[i]->x.data(), sizeof(double) * qs[i]->x.size());
    for (size_t e = 0; e < qs[i]->t.size(); e++) t[3 * (size_t) toff[i] + e] = qs[i]->t[e] + voff[i];
    for (int c = 0; c < 3; c++) zs[3 * (size_t) i + c] = qs[i]->desc.src[c];
  }
  int rc = h2b_prepare_surface(nv, x.data(), nt, t.data(), n.data(), g.data(), nullptr);
  if (rc != H2B_OK) return rc;
  h2b_surface *s = h2b_surface_new(nv, x.data(), nt, t.data(), n.data(), g.data());
  if (!s) return H2B_ERR_CUDA;
  const int L = H2B_BASIS_LINEAR;
  h2b_bem *slp = h2b_bem_new(s, H2B_LAPLACE, H2B_SLP, L, L, 2, 4, 0.0, 0.0, 0.0, 0.0);
  h2b_bem *dlp = h2b_bem_new(s, H2B_LAPLACE, H2B_DLP, L, L, 2, 4, 0.0, 0.0, 0.5, 0.0);
  h2b_tree *tr = (slp && dlp) ? h2b_tree_new_forest(ns, voff.data(), toff.data(), x.data(),
                                                    t.data(), L, L, 64, 1.4)
                              : nullptr;
  h2b_h2matrix *V = tr ? h2b_h2matrix_new(slp, tr, 4) : nullptr;
  h2b_h2matrix *K = V ? h2b_h2matrix_new_like(dlp, V) : nullptr;
  const bool mixed = (d.flags & H2B_SOLVE_MIXED) != 0;
  if (V && K && mixed) {
    h2b_h2matrix_set_precision(V, H2B_FP32);
    h2b_h2matrix_set_precision(K, H2B_FP32);
  }
  const auto c1 = tick();
  rc = (V && K) ? H2B_OK : H2B_ERR_CUDA;
  for (h2b_h2matrix *h : {V, K}) {
    if (rc == H2B_OK) rc = h2b_h2matrix_assemble_row_clusterbasis(h);
    if (rc == H2B_OK) rc = h2b_h2matrix_assemble_col_clusterbasis(h);
    if (rc == H2B_OK) rc = h2b_h2matrix_assemble_farfield(h);
  }
  if (rc == H2B_OK) rc = h2b_h2matrix_assemble_nearfield_pair(V, K);
  const auto c2 = tick();
  std::vector<double> gD(nv, 0.0), b(nv, 0.0), u(nv, 0.0), y(nv, 0.0);
  if (rc == H2B_OK) rc = h2b_project_l2_harmonic_multi(dlp, ns, toff.data(), 1, zs.data(), gD.data());
  if (rc == H2B_OK) rc = h2b_h2matrix_addeval(1.0, 0.0, K, gD.data(), b.data());
  const auto c3 = tick();
  if (rc == H2B_OK && mixed) rc = h2b_h2matrix_make_single(V);
  std::vector<uint32_t> iters(ns, 0);
  const h2b_h2matrix *ops[1] = {V};
  const double coef[2] = {1.0, 0.0};
  if (rc == H2B_OK)
    rc = h2b_solve_gmres_batch(1, ops, coef, ns, voff.data(), 1, b.data(), u.data(), d.eps,
                               d.maxiter, d.kmax, H2B_SOLVE_UNITARY | (mixed ? H2B_SOLVE_MIXED : 0u),
                               iters.data());
  const auto c4 = tick();
  // FP64 residual of every system: y = V u, |b_s - y_s| / |b_s|
  if (rc == H2B_OK) rc = h2b_h2matrix_addeval(1.0, 0.0, V, u.data(), y.data());
  if (rc == H2B_OK) {
    for (uint32_t i = 0; i < ns; i++) {
      double rr = 0.0, bb = 0.0;
      for (uint32_t e = voff[i]; e < voff[i + 1]; e++) {
        rr += (b[e] - y[e]) * (b[e] - y[e]);
        bb += b[e] * b[e];
      }
      Req *q = qs[i];
      q->solution.assign(u.begin() + voff[i], u.begin() + voff[i + 1]);
      q->res.iterations = iters[i];
      q->res.unknowns = voff[i + 1] - voff[i];
      q->res.rel_residual = bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
      q->res.t_setup = secs(c0, c1);
      q->res.t_assembly = secs(c1, c2);
      q->res.t_rhs = secs(c2, c3);
      q->res.t_solve = secs(c3, c4);
    }
  }
  h2b_h2matrix_del(K);
  h2b_h2matrix_del(V);
  h2b_tree_del(tr);
  h2b_bem_del(dlp);
  h2b_bem_del(slp);
  h2b_surface_del(s);
  return rc;
}

// Most requests one batch may take, and the most triangles of a batch.
constexpr size_t BATCH_MAX_REQUESTS = 64;
constexpr uint64_t BATCH_MAX_TRIANGLES = 1u << 20;

void worker_main(h2b_server *sv) {
  if (h2b_device_init(sv->device) != H2B_OK) return;
  std::vector<Req *> batch;
  while (true) {
    Req *q = nullptr;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      // admission: the oldest queued request, when its estimate fits the remaining budget (a
      // request larger than the whole budget runs alone)
      sv->cv_work.wait(lk, [&] {
        if (sv->stop) return true;
        if (sv->queue.empty()) return false;
        const uint64_t e = sv->queue.front()->est;
        return sv->reserved + e <= sv->budget || sv->running == 0;
      });
      if (sv->stop) return;
      q = sv->queue.front();
      sv->queue.pop_front();
      batch.assign(1, q);
      sv->reserved += q->est;
      // continuous batching: queued requests that can share q's operator join it (in arrival
      // order, while they fit the budget and the batch limits)
      uint64_t tris = q->desc.triangles;
      for (auto it = sv->queue.begin(); it != sv->queue.end() && batch.size() < sv->batch_max &&
                                        batch.size() < BATCH_MAX_REQUESTS;) {
        Req *r = *it;
        if (batchable(q, r) && sv->reserved + r->est <= sv->budget &&
            tris + r->desc.triangles <= BATCH_MAX_TRIANGLES) {
          batch.push_back(r);
          sv->reserved += r->est;
          tris += r->desc.triangles;
          it = sv->queue.erase(it);
        } else {
          ++it;
        }
      }
      sv->running++;
      const double t = since(sv);
      for (Req *r : batch) {
        r->status = 2;
        r->res.t_start = t;
      }
    }
    const int rc = batch.size() > 1 ? run_batch(batch) : run_request(q);
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->running--;
      const double t = since(sv);
      for (Req *r : batch) {
        sv->reserved -= r->est;
        sv->done++;
        r->res.t_done = t;
        r->res.status = rc;
        if (rc != H2B_OK) snprintf(r->err, sizeof(r->err), "%s", h2b_last_error());
        r->status = rc == H2B_OK ? 0 : rc;
      }
    }
    sv->cv_done.notify_all();
    sv->cv_work.notify_all();
  }
}

}  // namespace

extern "C" h2b_server *h2b_server_new(int device, uint32_t slots, uint64_t hbm_budget_bytes) {
  if (slots == 0 || slots > 256 || hbm_budget_bytes == 0) {
    h2b_set_error("h2b_server_new: slots must be in 1..256 and the budget positive");
    return NULL;
  }
  if (h2b_device_init(device) != H2B_OK) return NULL;
  h2b_server *sv = new h2b_server();
  sv->device = device;
  sv->slots = slots;
  sv->budget = hbm_budget_bytes;
  sv->t0 = Clock::now();
  for (uint32_t i = 0; i < slots; i++) sv->workers.emplace_back(worker_main, sv);
  return sv;
}

extern "C" int64_t h2b_server_submit(h2b_server *sv, const h2b_request *r) {
  if (!sv || !r || !r->x || !r->t || r->vertices == 0 || r->triangles == 0) {
    h2b_set_error("h2b_server_submit: empty request");
    return H2B_ERR_ARG;
  }
  if (r->pde != H2B_LAPLACE && r->pde != H2B_HELMHOLTZ) {
    h2b_set_error("h2b_server_submit: unknown PDE %d", r->pde);
    return H2B_ERR_ARG;
  }
  if (r->kmax < 2 || r->kmax >= 128 || !(r->eps > 0.0)) {
    h2b_set_error("h2b_server_submit: kmax must be in 2..127 and eps positive");
    return H2B_ERR_ARG;
  }
  Req *q = new Req();
  q->desc = *r;
  q->x.assign(r->x, r->x + 3ull * r->vertices);
  q->t.assign(r->t, r->t + 3ull * r->triangles);
  q->desc.x = nullptr;
  q->desc.t = nullptr;
  q->est = estimate_bytes(*r);
  memset(&q->res, 0, sizeof(q->res));
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    q->id = sv->next_id++;
    q->res.t_submit = since(sv);
    q->res.bytes_reserved = q->est;
    sv->reqs[q->id] = q;
    sv->queue.push_back(q);
  }
  sv->cv_work.notify_all();
  return q->id;
}

extern "C" int h2b_server_wait(h2b_server *sv, int64_t id, double *solution,
                               h2b_request_result *res) {
  if (!sv) return H2B_ERR_ARG;
  Req *q = nullptr;
  {
    std::unique_lock<std::mutex> lk(sv->mu);
    auto itr = sv->reqs.find(id);
    if (itr == sv->reqs.end()) {
      h2b_set_error("h2b_server_wait: unknown request %lld", (long long) id);
      return H2B_ERR_ARG;
    }
    q = itr->second;
    sv->cv_done.wait(lk, [&] { return q->status <= 0 || sv->stop; });
    if (q->status > 0) {
      h2b_set_error("h2b_server_wait: server stopped");
      return H2B_ERR_STATE;
    }
    sv->reqs.erase(itr);
  }
  const int rc = q->status;
  if (res) *res = q->res;
  if (rc == 0 && solution) memcpy(solution, q->solution.data(), sizeof(double) * q->solution.size());
  if (rc != 0) h2b_set_error("request %lld: %s", (long long) id, q->err);
  delete q;
  return rc;
}

extern "C" int h2b_server_set_batching(h2b_server *sv, uint32_t max_requests) {
  if (!sv || max_requests == 0) {
    h2b_set_error("h2b_server_set_batching: NULL server or zero requests");
    return H2B_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->batch_max = max_requests;
  return H2B_OK;
}

extern "C" int h2b_server_stats(h2b_server *sv, uint64_t out[4]) {
  if (!sv || !out) return H2B_ERR_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  out[0] = sv->queue.size();
  out[1] = sv->running;
  out[2] = sv->done;
  out[3] = sv->reserved;
  return H2B_OK;
}

extern "C" void h2b_server_del(h2b_server *sv) {
  if (!sv) return;
  {
    std::unique_lock<std::mutex> lk(sv->mu);
    // queued requests are dropped; running ones finish
    for (Req *q : sv->queue) q->status = H2B_ERR_STATE;
    sv->queue.clear();
    sv->cv_done.wait(lk, [&] { return sv->running == 0; });
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  sv->cv_done.notify_all();
  for (auto &w : sv->workers) w.join();
  for (auto &kv : sv->reqs) delete kv.second;
  delete sv;
}
