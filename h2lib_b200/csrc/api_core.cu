// C-ABI implementation: status, device init, surfaces, operators and nearfield entry points.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <vector>

#include "api_internal.h"

// ------------------------------------------------------------------------------------------
// Status
// ------------------------------------------------------------------------------------------

static thread_local char g_err[1024] = "";

extern "C" void h2b_set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

extern "C" const char *h2b_last_error(void) { return g_err; }

extern "C" const char *h2b_version(void) { return "h2b200 0.1 (sm_100a)"; }

// Device whose constant tables are loaded; written under g_init_mutex (handles may be created
// from several host threads, e.g. the workers of a solve server).
static std::atomic<int> g_inited_device{-1};
static std::mutex g_init_mutex;

extern "C" int h2b_device_init(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    h2b_set_error("no CUDA device available");
    return H2B_ERR_CUDA;
  }
  if (device < 0 || device >= n) {
    h2b_set_error("device %d out of range (%d devices)", device, n);
    return H2B_ERR_ARG;
  }
  H2B_CUDA_TRY(cudaSetDevice(device));
  int major = 0, minor = 0;
  H2B_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  H2B_CUDA_TRY(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
  if (major != 10) {
    h2b_set_error("device %d is sm_%d%d; this library is built for sm_100a only", device,
                  major, minor);
    return H2B_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_init_mutex);
  if (g_inited_device != device) {
    int rc = h2b_near_upload_dist_rules();
    if (rc != H2B_OK) return rc;
    // keep freed stream-ordered memory in the device pool for reuse by later handles
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      // never make one handle's stream wait for another's to reuse a freed block
      int no = 0;
      cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    }
    cudaGetLastError();
    g_inited_device = device;
  }
  return H2B_OK;
}

int h2b_ensure_device(void) {
  int dev = 0;
  if (g_inited_device >= 0) {
    H2B_CUDA_TRY(cudaGetDevice(&dev));
    if (dev == g_inited_device) return H2B_OK;
  } else if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    dev = 0;
  }
  return h2b_device_init(dev);
}

static std::atomic<unsigned long long> g_launches{0};

void h2b_note_launch(void) { g_launches.fetch_add(1, std::memory_order_relaxed); }

extern "C" int h2b_launch_count(uint64_t *n) {
  if (!n) return H2B_ERR_ARG;
  *n = g_launches.load(std::memory_order_relaxed);
  return H2B_OK;
}

extern "C" int h2b_device_memory(uint64_t out[4]) {
  if (!out) return H2B_ERR_ARG;
  int dev = 0;
  size_t fr = 0, tot = 0;
  H2B_CUDA_TRY(cudaGetDevice(&dev));
  H2B_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
  cudaMemPool_t pool;
  uint64_t used = 0, reserved = 0;
  H2B_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, dev));
  H2B_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
  H2B_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
  out[0] = fr;
  out[1] = tot;
  out[2] = used;
  out[3] = reserved;
  return H2B_OK;
}

bool h2b_is_device_ptr(const void *p) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// ------------------------------------------------------------------------------------------
// Surfaces
// ------------------------------------------------------------------------------------------

extern "C" h2b_surface *h2b_surface_new(uint32_t vertices, const double *x, uint32_t triangles,
                                        const uint32_t *t, const double *n, const double *g) {
  if (!x || !t || !n || !g || vertices == 0 || triangles == 0) {
    h2b_set_error("h2b_surface_new: empty mesh or NULL array");
    return NULL;
  }
  for (uint64_t i = 0; i < 3ull * triangles; i++)
    if (t[i] >= vertices) {
      h2b_set_error("h2b_surface_new: triangle %llu references vertex %u >= %u",
                    (unsigned long long) (i / 3), t[i], vertices);
      return NULL;
    }
  if (h2b_ensure_device() != H2B_OK) return NULL;
  h2b_surface *s = new h2b_surface();
  s->nv = vertices;
  s->nt = triangles;
  s->x.assign(x, x + 3ull * vertices);
  s->t.assign(t, t + 3ull * triangles);
  s->n.assign(n, n + 3ull * triangles);
  s->g.assign(g, g + triangles);
  if (h2b_adjacency_build(vertices, triangles, s->t.data(), &s->adj) != H2B_OK) {
    delete s;
    h2b_set_error("h2b_surface_new: out of host memory");
    return NULL;
  }
  std::vector<TriRec> rec(triangles);
  for (uint32_t i = 0; i < triangles; i++) {
    TriRec &r = rec[i];
    memset(&r, 0, sizeof(r));
    const uint32_t *ti = t + 3ull * i;
    for (int d = 0; d < 3; d++) {
      r.a[d] = x[3ull * ti[0] + d];
      r.b[d] = x[3ull * ti[1] + d];
      r.c[d] = x[3ull * ti[2] + d];
      r.n[d] = n[3ull * i + d];
      r.v[d] = ti[d];
    }
    r.g = g[i];
  }
  // (an attribute query, not cudaGetDeviceProperties, which costs milliseconds per call)
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocAsync(&s->d_tri, sizeof(TriRec) * triangles, s->stream) != cudaSuccess ||
      cudaMallocAsync(&s->d_x, sizeof(double) * 3ull * vertices, s->stream) != cudaSuccess ||
      cudaMemcpyAsync(s->d_tri, rec.data(), sizeof(TriRec) * triangles, cudaMemcpyHostToDevice,
                      s->stream) != cudaSuccess ||
      cudaMemcpyAsync(s->d_x, x, sizeof(double) * 3ull * vertices, cudaMemcpyHostToDevice,
                      s->stream) != cudaSuccess ||
      cudaMallocAsync(&s->d_vt_off, sizeof(uint32_t) * (vertices + 1ull), s->stream) != cudaSuccess ||
      cudaMallocAsync(&s->d_vt_tri, sizeof(uint32_t) * 3ull * triangles, s->stream) != cudaSuccess ||
      cudaMemcpyAsync(s->d_vt_off, s->adj.off, sizeof(uint32_t) * (vertices + 1ull),
                      cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
      cudaMemcpyAsync(s->d_vt_tri, s->adj.tri, sizeof(uint32_t) * 3ull * triangles,
                      cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess) {
    h2b_set_error("h2b_surface_new: %s", cudaGetErrorString(cudaGetLastError()));
    h2b_surface_del(s);
    return NULL;
  }
  s->device = dev;
  s->num_sms = sms;
  return s;
}

extern "C" void h2b_surface_del(h2b_surface *s) {
  if (!s) return;
  // every entry point ends synchronised, so no kernel still reads these arrays; stream-ordered
  // frees do not synchronise the device (other handles keep running)
  if (s->d_tri) cudaFreeAsync(s->d_tri, s->stream);
  if (s->d_x) cudaFreeAsync(s->d_x, s->stream);
  if (s->d_vt_off) cudaFreeAsync(s->d_vt_off, s->stream);
  if (s->d_vt_tri) cudaFreeAsync(s->d_vt_tri, s->stream);
  if (s->stream) cudaStreamDestroy(s->stream);
  h2b_adjacency_free(&s->adj);
  delete s;
}

// ------------------------------------------------------------------------------------------
// Operators
// ------------------------------------------------------------------------------------------

extern "C" h2b_bem *h2b_bem_new(const h2b_surface *s, int pde, int layer, int row_basis,
                                int col_basis, uint32_t q_regular, uint32_t q_singular,
                                double k_re, double k_im, double alpha_re, double alpha_im) {
  if (!s) {
    h2b_set_error("h2b_bem_new: NULL surface");
    return NULL;
  }
  if ((pde != H2B_LAPLACE && pde != H2B_HELMHOLTZ) ||
      (layer != H2B_SLP && layer != H2B_DLP && layer != H2B_ADLP) ||
      (row_basis != H2B_BASIS_CONSTANT && row_basis != H2B_BASIS_LINEAR) ||
      (col_basis != H2B_BASIS_CONSTANT && col_basis != H2B_BASIS_LINEAR)) {
    h2b_set_error("h2b_bem_new: unknown pde/layer/basis (%d, %d, %d, %d)", pde, layer,
                  row_basis, col_basis);
    return NULL;
  }
  if (q_regular < 1 || q_regular > 5 || q_singular < 1 || q_singular > 8) {
    h2b_set_error("h2b_bem_new: quadrature orders (%u, %u) outside 1..5 / 1..8", q_regular,
                  q_singular);
    return NULL;
  }
  if (layer == H2B_SLP && (alpha_re != 0.0 || alpha_im != 0.0)) {
    h2b_set_error("h2b_bem_new: the single layer operator has no identity term (alpha must be 0)");
    return NULL;
  }
  h2b_bem *b = new h2b_bem();
  b->s = s;
  b->pde = pde;
  b->layer = layer;
  b->row_basis = row_basis;
  b->col_basis = col_basis;
  b->q = q_regular;
  b->q2 = q_singular;
  b->k_re = k_re;
  b->k_im = k_im;
  b->alpha_re = alpha_re;
  b->alpha_im = alpha_im;
  b->kconst = H2B_KERNEL_CONST;
  // Mass matrices of the reference triangle scaled by the Gram determinant
  // (Library/laplacebem3d.c:926-994): ll 1/12 diagonal, 1/24 off-diagonal; cl / lc 1/6.
  for (int i = 0; i < 9; i++) b->mass[i] = 0.0;
  if (row_basis == H2B_BASIS_LINEAR && col_basis == H2B_BASIS_LINEAR) {
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) b->mass[i + 3 * j] = (i == j) ? 1.0 / 12.0 : 1.0 / 24.0;
  } else if (row_basis != col_basis) {
    for (int i = 0; i < 3; i++) b->mass[i] = 1.0 / 6.0;
  }
  if (h2b_quad_build(q_regular, q_singular, row_basis, col_basis, &b->quad) != H2B_OK) {
    delete b;
    return NULL;
  }
  // Packed singular rules for the device, every block padded to an even number of doubles
  // (16-byte alignment).  Case 1 (common vertex): for q_singular = 4 the tensor form of
  // h2b_quad_vert_tensor (rule_n[1] = groups), otherwise x0, x1, y0, y1, w (raw), n_1 doubles
  // each.  Cases 2 and 3 (common edge, identical): the reduced rules of h2b_quad_reduce, a, b, c and
  // the basis-weighted weight rows (i + NR j) for the row / column basis functions i < NR,
  // j < NC (NR, NC = 3 for a linear basis, 1 for a constant one), n_c' doubles each.
  std::vector<double> pack;
  b->rule_n[0] = b->rule_off[0] = 0;
  const int NR = row_basis == H2B_BASIS_LINEAR ? 3 : 1, NC = col_basis == H2B_BASIS_LINEAR ? 3 : 1;
  for (int c = 1; c <= 3; c++) {
    const h2b_rule &r = b->quad.rule[c];
    b->rule_off[c] = (uint32_t) pack.size();
    if (c == 1 && q_singular == 4) {
      // tensor form (h2b_quad_vert_tensor): the kernel's specialised path for q2 = 4
      uint32_t ng = 0;
      double *t = nullptr;
      if (h2b_quad_vert_tensor(q_singular, row_basis, col_basis, &ng, &t) != H2B_OK) {
        h2b_bem_del(b);
        return NULL;
      }
      b->rule_n[c] = ng;
      b->vert_tensor = 1;
      pack.insert(pack.end(), t, t + (size_t) (4 + NR + NC) * q_singular * ng);
      free(t);
    } else if (c == 1) {
      b->rule_n[c] = r.n;
      const double *src[5] = {r.x0, r.x1, r.y0, r.y1, r.w + 9ull * r.n};
      for (int f = 0; f < 5; f++) pack.insert(pack.end(), src[f], src[f] + r.n);
    } else {
      uint32_t n = 0;
      double *abc = nullptr, *w9 = nullptr;
      if (h2b_quad_reduce(&r, c, q_singular, &n, &abc, &w9) != H2B_OK) {
        h2b_bem_del(b);
        return NULL;
      }
      b->rule_n[c] = n;
      pack.insert(pack.end(), abc, abc + 3ull * n);
      for (int j = 0; j < NC; j++)
        for (int i = 0; i < NR; i++)
          pack.insert(pack.end(), w9 + (size_t) (i + 3 * j) * n, w9 + (size_t) (i + 3 * j + 1) * n);
      free(abc);
      free(w9);
    }
    // offsets inside the block are multiples of n; keep n even by padding the whole block
    if (pack.size() & 1) pack.push_back(0.0);
  }
  if (q_singular == 4) {
    // slot 4: the common-vertex rule with the radial sum folded into moments
    // (h2b_quad_vert_merged), used for the Laplace kernels
    uint32_t nm = 0;
    double *t = nullptr;
    if (h2b_quad_vert_merged(q_singular, row_basis, col_basis, &nm, &t) != H2B_OK) {
      h2b_bem_del(b);
      return NULL;
    }
    b->rule_off[4] = (uint32_t) pack.size();
    b->rule_n[4] = nm;
    b->vert_merged = 1;
    pack.insert(pack.end(), t, t + (size_t) (4 + 2 * NR + 4 * NC) * nm);
    free(t);
    if (pack.size() & 1) pack.push_back(0.0);
  }
  // every field must start on a 16-byte boundary: n is a multiple of 2 (2 q2^4 and 6 q2^4)
  b->rule_total = (uint32_t) pack.size();
  cudaStream_t st = b->s->stream;
  if (cudaMallocAsync(&b->d_rule, sizeof(double) * pack.size(), st) != cudaSuccess ||
      cudaMemcpyAsync(b->d_rule, pack.data(), sizeof(double) * pack.size(),
                      cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMallocAsync(&b->d_err, sizeof(int), st) != cudaSuccess ||
      cudaMemsetAsync(b->d_err, 0, sizeof(int), st) != cudaSuccess ||
      cudaEventCreate(&b->ev[0]) != cudaSuccess || cudaEventCreate(&b->ev[1]) != cudaSuccess ||
      cudaEventCreate(&b->ev[2]) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
    h2b_set_error("h2b_bem_new: %s", cudaGetErrorString(cudaGetLastError()));
    h2b_bem_del(b);
    return NULL;
  }
  return b;
}

extern "C" void h2b_bem_del(h2b_bem *b) {
  if (!b) return;
  // the operator must be deleted before its surface (the frees are ordered on its stream)
  if (b->d_rule) cudaFreeAsync(b->d_rule, b->s->stream);
  if (b->d_err) cudaFreeAsync(b->d_err, b->s->stream);
  for (int i = 0; i < 3; i++)
    if (b->ev[i]) cudaEventDestroy(b->ev[i]);
  h2b_quad_free(&b->quad);
  delete b;
}

int h2b_bem_kernel_kind(const h2b_bem *b) {
  if (b->pde == H2B_LAPLACE)
    return b->layer == H2B_SLP ? H2B_KK_LSLP : b->layer == H2B_DLP ? H2B_KK_LDLP : H2B_KK_LADLP;
  return b->layer == H2B_SLP ? H2B_KK_HSLP : b->layer == H2B_DLP ? H2B_KK_HDLP : H2B_KK_HADLP;
}

void h2b_fill_launch(const h2b_bem *b, h2b_near_launch *L) {
  memset(L, 0, sizeof(*L));
  L->kk = h2b_bem_kernel_kind(b);
  L->row_linear = b->row_basis == H2B_BASIS_LINEAR;
  L->col_linear = b->col_basis == H2B_BASIS_LINEAR;
  L->q = b->q;
  L->tri = b->s->d_tri;
  L->kconst = b->kconst;
  L->k_re = b->k_re;
  L->k_imn = -b->k_im;
  L->alpha_re = b->alpha_re;
  L->alpha_im = b->alpha_im;
  for (int i = 0; i < 9; i++) L->mass[i] = b->mass[i];
  L->rule = b->d_rule;
  for (int i = 0; i < 5; i++) {
    L->rule_n[i] = b->rule_n[i];
    L->rule_off[i] = b->rule_off[i];
  }
  L->rule_total = b->rule_total;
  L->vert_tensor = b->vert_tensor;
  L->vert_merged = b->vert_merged;
  L->num_sms = b->s->num_sms;
  L->err = b->d_err;
  L->nvert = UINT32_MAX;
}

uint32_t h2b_bem_rows(const h2b_bem *b) {
  return b->row_basis == H2B_BASIS_LINEAR ? b->s->nv : b->s->nt;
}
uint32_t h2b_bem_cols(const h2b_bem *b) {
  return b->col_basis == H2B_BASIS_LINEAR ? b->s->nv : b->s->nt;
}

// Upload a finished plan; device arrays returned in *dp (freed by h2b_devplan_free).
int h2b_devplan_upload(const h2b_nearplan *p, cudaStream_t st, h2b_devplan *dp) {
  memset(dp, 0, sizeof(*dp));
  dp->ntiles = p->ntiles;
  dp->nsing = p->nsing;
  dp->nvert = p->nsing ? p->case_start[2] - p->case_start[1] : 0;
  if (p->ntiles) {
    H2B_CUDA_TRY(cudaMallocAsync(&dp->tiles, sizeof(h2b_tile) * p->ntiles, st));
    H2B_CUDA_TRY(cudaMemcpyAsync(dp->tiles, p->tiles, sizeof(h2b_tile) * p->ntiles,
                                 cudaMemcpyHostToDevice, st));
  }
  if (p->nrefs) {
    H2B_CUDA_TRY(cudaMallocAsync(&dp->refs, sizeof(h2b_triref) * p->nrefs, st));
    H2B_CUDA_TRY(cudaMemcpyAsync(dp->refs, p->refs, sizeof(h2b_triref) * p->nrefs,
                                 cudaMemcpyHostToDevice, st));
  }
  if (p->nsing) {
    H2B_CUDA_TRY(cudaMallocAsync(&dp->sing, sizeof(h2b_sing) * p->nsing, st));
    H2B_CUDA_TRY(cudaMemcpyAsync(dp->sing, p->sing, sizeof(h2b_sing) * p->nsing,
                                 cudaMemcpyHostToDevice, st));
  }
  return H2B_OK;
}

int h2b_classify_device(const h2b_surface *s, const void *refs, const h2b_tile *tiles,
                        uint32_t ntiles, cudaStream_t st, h2b_sing **d_sing, uint32_t cnt[4]) {
  *d_sing = nullptr;
  for (int c = 0; c < 4; c++) cnt[c] = 0;
  uint32_t *d_cur = nullptr;
  H2B_CUDA_TRY(cudaMallocAsync(&d_cur, sizeof(uint32_t) * 8, st));
  int rc = H2B_OK;
  uint32_t host[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (cudaMemsetAsync(d_cur, 0, sizeof(uint32_t) * 8, st) != cudaSuccess) rc = H2B_ERR_CUDA;
  if (rc == H2B_OK)
    rc = h2b_near_classify(s->d_tri, refs, tiles, ntiles, s->d_vt_off, s->d_vt_tri, d_cur, nullptr,
                           nullptr, st);
  if (rc == H2B_OK &&
      (cudaMemcpyAsync(host, d_cur, sizeof(uint32_t) * 4, cudaMemcpyDeviceToHost, st) !=
           cudaSuccess ||
       cudaStreamSynchronize(st) != cudaSuccess))
    rc = H2B_ERR_CUDA;
  const uint64_t nsing = (uint64_t) host[1] + host[2] + host[3];
  if (rc == H2B_OK && nsing > UINT32_MAX) {
    h2b_set_error("singular-pair classification: %llu pairs exceed the 32-bit pair list",
                  (unsigned long long) nsing);
    cudaFreeAsync(d_cur, st);
    return H2B_ERR_ARG;
  }
  if (rc == H2B_OK) {
    // base offsets of the cases in host[4..7]
    host[4] = 0;
    host[5] = 0;
    host[6] = host[1];
    host[7] = host[1] + host[2];
    if (nsing &&
        (cudaMallocAsync((void **) d_sing, sizeof(h2b_sing) * nsing, st) != cudaSuccess ||
         cudaMemsetAsync(d_cur, 0, sizeof(uint32_t) * 4, st) != cudaSuccess ||
         cudaMemcpyAsync(d_cur + 4, host + 4, sizeof(uint32_t) * 4, cudaMemcpyHostToDevice, st) !=
             cudaSuccess))
      rc = H2B_ERR_CUDA;
  }
  if (rc == H2B_OK && nsing)
    rc = h2b_near_classify(s->d_tri, refs, tiles, ntiles, s->d_vt_off, s->d_vt_tri, d_cur,
                           d_cur + 4, *d_sing, st);
  if (rc == H2B_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = H2B_ERR_CUDA;
  if (rc == H2B_ERR_CUDA)
    h2b_set_error("singular-pair classification: %s", cudaGetErrorString(cudaGetLastError()));
  cudaFreeAsync(d_cur, st);
  if (rc != H2B_OK && *d_sing) {
    cudaFreeAsync(*d_sing, st);
    *d_sing = nullptr;
  }
  if (rc == H2B_OK)
    for (int c = 1; c <= 3; c++) cnt[c] = host[c];
  return rc;
}

void h2b_devplan_free(h2b_devplan *dp, cudaStream_t st) {
  if (dp->tiles) cudaFreeAsync(dp->tiles, st);
  if (dp->refs) cudaFreeAsync(dp->refs, st);
  if (dp->sing) cudaFreeAsync(dp->sing, st);
  memset(dp, 0, sizeof(*dp));
}

int h2b_check_err_flag(const h2b_bem *b, cudaStream_t st) {
  int flag = 0;
  H2B_CUDA_TRY(cudaMemcpyAsync(&flag, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  H2B_CUDA_TRY(cudaStreamSynchronize(st));
  if (flag) {
    h2b_set_error("quadrature kernel: staging of the singular rules timed out");
    cudaMemsetAsync(b->d_err, 0, sizeof(int), st);
    return H2B_ERR_TIMEOUT;
  }
  return H2B_OK;
}

// ------------------------------------------------------------------------------------------
// Nearfield blocks
// ------------------------------------------------------------------------------------------

extern "C" int h2b_bem_nearfield(const h2b_bem *bem, const uint32_t *ridx, uint32_t rows,
                                 const uint32_t *cidx, uint32_t cols, int ntrans, double *N,
                                 uint64_t ld) {
  if (!bem || !N) {
    h2b_set_error("h2b_bem_nearfield: NULL operator or output");
    return H2B_ERR_ARG;
  }
  if (rows == 0 || cols == 0) return H2B_OK;
  const uint32_t out_rows = ntrans ? cols : rows, out_cols = ntrans ? rows : cols;
  if (ld < out_rows) {
    h2b_set_error("h2b_bem_nearfield: ld %llu < %u rows of the output",
                  (unsigned long long) ld, out_rows);
    return H2B_ERR_ARG;
  }
  int rc = h2b_ensure_device();
  if (rc != H2B_OK) return rc;
  const h2b_surface *s = bem->s;
  const uint32_t nr_all = h2b_bem_rows(bem), nc_all = h2b_bem_cols(bem);
  std::vector<uint32_t> ri, ci;
  if (!ridx) {
    ri.resize(rows);
    for (uint32_t i = 0; i < rows; i++) ri[i] = i;
    ridx = ri.data();
  }
  if (!cidx) {
    ci.resize(cols);
    for (uint32_t i = 0; i < cols; i++) ci[i] = i;
    cidx = ci.data();
  }
  // validate indices and reject duplicates (H2Lib index sets are permutations)
  {
    std::vector<uint8_t> seen(nr_all > nc_all ? nr_all : nc_all, 0);
    for (uint32_t i = 0; i < rows; i++) {
      if (ridx[i] >= nr_all || seen[ridx[i]]) {
        h2b_set_error("h2b_bem_nearfield: row index %u invalid or repeated", ridx[i]);
        return H2B_ERR_ARG;
      }
      seen[ridx[i]] = 1;
    }
    std::fill(seen.begin(), seen.end(), 0);
    for (uint32_t i = 0; i < cols; i++) {
      if (cidx[i] >= nc_all || seen[cidx[i]]) {
        h2b_set_error("h2b_bem_nearfield: column index %u invalid or repeated", cidx[i]);
        return H2B_ERR_ARG;
      }
      seen[cidx[i]] = 1;
    }
  }
  const int cplx = bem->pde == H2B_HELMHOLTZ;
  const size_t es = cplx ? 16 : 8;
  cudaStream_t st = s->stream;
  const bool dev_out = h2b_is_device_ptr(N);
  const uint64_t ld_dev = dev_out ? ld : out_rows;

  // small outputs: 32 x 32 tiles so that the grid covers the SMs
  uint64_t t64 = (uint64_t) ((rows + 63) / 64) * ((cols + 63) / 64);
  uint32_t tile = t64 < 2ull * s->num_sms ? 32 : 64;

  // the singular pairs are found on the device (h2b_classify_device): the host plan only lists
  // the tiles and their triangles
  h2b_nearplan plan;
  h2b_nearplan_init(&plan);
  plan.skip_sing = 1;
  rc = h2b_nearplan_add_block(&plan, const_cast<h2b_adjacency *>(&s->adj), bem->row_basis,
                              bem->col_basis, ridx, rows, cidx, cols, 0, (uint32_t) ld_dev,
                              ntrans, tile);
  if (rc == H2B_OK) rc = h2b_nearplan_finalize(&plan);
  if (rc != H2B_OK) {
    h2b_nearplan_free(&plan);
    h2b_set_error("h2b_bem_nearfield: out of host memory building the plan");
    return rc;
  }
  h2b_devplan dp;
  rc = h2b_devplan_upload(&plan, st, &dp);
  h2b_nearplan_free(&plan);
  if (rc != H2B_OK) {
    h2b_devplan_free(&dp, st);
    return rc;
  }
  {
    uint32_t cnt[4];
    rc = h2b_classify_device(s, dp.refs, dp.tiles, dp.ntiles, st, &dp.sing, cnt);
    if (rc != H2B_OK) {
      h2b_devplan_free(&dp, st);
      return rc;
    }
    dp.nsing = cnt[1] + cnt[2] + cnt[3];
    dp.nvert = cnt[1];
  }

  double *out = N;
  if (!dev_out) {
    if (cudaMallocAsync((void **) &out, es * ld_dev * out_cols, st) != cudaSuccess) {
      h2b_devplan_free(&dp, st);
      h2b_set_error("h2b_bem_nearfield: device allocation of %llu bytes failed",
                    (unsigned long long) (es * ld_dev * out_cols));
      return H2B_ERR_NOMEM;
    }
  }
  h2b_near_launch L;
  h2b_fill_launch(bem, &L);
  L.refs = dp.refs;
  L.tiles = dp.tiles;
  L.ntiles = dp.ntiles;
  L.sing = dp.sing;
  L.nsing = dp.nsing;
  L.nvert = dp.nvert;
  L.out0 = out;
  // the operator's own events time the two kernels (nearfield diagnostics, h2b_bem_timings)
  h2b_bem *mb = const_cast<h2b_bem *>(bem);
  L.ev_between = mb->ev[1];
  if (cudaEventRecord(mb->ev[0], st) != cudaSuccess) rc = H2B_ERR_CUDA;
  if (rc == H2B_OK) rc = h2b_near_launch_kernels(&L, st);
  if (rc == H2B_OK && cudaEventRecord(mb->ev[2], st) != cudaSuccess) rc = H2B_ERR_CUDA;
  if (rc == H2B_OK && !dev_out) {
    if (cudaMemcpy2DAsync(N, ld * es, out, ld_dev * es, out_rows * es, out_cols,
                          cudaMemcpyDeviceToHost, st) != cudaSuccess) {
      h2b_set_error("h2b_bem_nearfield: copy back failed: %s",
                    cudaGetErrorString(cudaGetLastError()));
      rc = H2B_ERR_CUDA;
    }
  }
  if (!dev_out) cudaFreeAsync(out, st);
  h2b_devplan_free(&dp, st);
  if (rc == H2B_OK) rc = h2b_check_err_flag(bem, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == H2B_OK) {
    h2b_set_error("h2b_bem_nearfield: %s", cudaGetErrorString(cudaGetLastError()));
    rc = H2B_ERR_CUDA;
  }
  if (rc == H2B_OK) {
    float a = 0.0f, b = 0.0f;
    // ev[1] is recorded only when the plan has distant tiles; otherwise both phases read 0
    if (cudaEventElapsedTime(&a, mb->ev[0], mb->ev[1]) != cudaSuccess ||
        cudaEventElapsedTime(&b, mb->ev[1], mb->ev[2]) != cudaSuccess) {
      cudaGetLastError();
      a = b = 0.0f;
    }
    mb->near_ms[0] = a;
    mb->near_ms[1] = b;
  }
  return rc;
}

extern "C" int h2b_bem_timings(const h2b_bem *bem, double ms[2]) {
  if (!bem || !ms) return H2B_ERR_ARG;
  ms[0] = bem->near_ms[0];
  ms[1] = bem->near_ms[1];
  return H2B_OK;
}

extern "C" int h2b_bem_assemble_amatrix(const h2b_bem *bem, double *G, uint64_t ld) {
  if (!bem) {
    h2b_set_error("h2b_bem_assemble_amatrix: NULL operator");
    return H2B_ERR_ARG;
  }
  // Like assemble_bem3d_amatrix (Library/bem3d.c:9988) the matrix is square: the column count is
  // taken from the row basis.
  const uint32_t n = h2b_bem_rows(bem);
  if (h2b_bem_cols(bem) != n) {
    h2b_set_error("h2b_bem_assemble_amatrix: row and column index sets differ in size");
    return H2B_ERR_ARG;
  }
  return h2b_bem_nearfield(bem, NULL, n, NULL, n, 0, G, ld);
}
