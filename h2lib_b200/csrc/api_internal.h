// Handle layouts and helpers shared by the api_*.cu translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "device_common.cuh"
#include "h2b200_internal.h"
#include "h2b200_plan.h"
#include "nearfield.h"

struct h2b_surface {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  uint32_t nv = 0, nt = 0;
  std::vector<double> x, n, g;  // host copies (3*nv, 3*nt, nt)
  std::vector<uint32_t> t;      // 3*nt
  h2b_adjacency adj{};
  TriRec *d_tri = nullptr;      // nt records
  double *d_x = nullptr;        // 3*nv
  uint32_t *d_vt_off = nullptr, *d_vt_tri = nullptr;  // vertex -> triangles (CSR, from adj)
};

struct h2b_bem {
  const h2b_surface *s = nullptr;
  int pde = 0, layer = 0, row_basis = 'c', col_basis = 'c';
  uint32_t q = 2, q2 = 4;
  double k_re = 0, k_im = 0, alpha_re = 0, alpha_im = 0, kconst = H2B_KERNEL_CONST;
  double mass[9];
  h2b_quad quad{};
  double *d_rule = nullptr;
  uint32_t rule_n[5] = {0, 0, 0, 0, 0}, rule_off[5] = {0, 0, 0, 0, 0}, rule_total = 0;
  int vert_merged = 0;  // 1: slot 4 holds h2b_quad_vert_merged's rule (q_singular == 4)
  int vert_tensor = 0;  // 1: the common-vertex rule is packed in tensor form (q_singular == 4)
  int *d_err = nullptr;
  // device time of the last h2b_bem_nearfield call: events around the distant and singular
  // kernels, and their elapsed ms (written by that call after its stream synchronises)
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  double near_ms[2] = {0.0, 0.0};
};

struct h2b_devplan {
  h2b_tile *tiles;
  h2b_triref *refs;
  h2b_sing *sing;
  uint32_t ntiles, nsing;
  uint32_t nvert;  // common-vertex pairs at the start of sing (the plan sorts them by case)
};

int h2b_ensure_device(void);
bool h2b_is_device_ptr(const void *p);
int h2b_bem_kernel_kind(const h2b_bem *b);
void h2b_fill_launch(const h2b_bem *b, h2b_near_launch *L);
uint32_t h2b_bem_rows(const h2b_bem *b);
uint32_t h2b_bem_cols(const h2b_bem *b);
int h2b_devplan_upload(const h2b_nearplan *p, cudaStream_t st, h2b_devplan *dp);
void h2b_devplan_free(h2b_devplan *dp, cudaStream_t st);
// Singular pairs of uploaded tiles, found on the device in two passes (count, then write grouped
// by Sauter-Schwab case: vertex, edge, identical; order inside a case not fixed).  *d_sing: a
// stream-ordered device array of cnt[1] + cnt[2] + cnt[3] pairs (nullptr when there are none);
// cnt[c]: pairs of case c = 1..3.  Synchronises st.
int h2b_classify_device(const h2b_surface *s, const void *refs, const h2b_tile *tiles,
                        uint32_t ntiles, cudaStream_t st, h2b_sing **d_sing, uint32_t cnt[4]);
int h2b_check_err_flag(const h2b_bem *b, cudaStream_t st);
