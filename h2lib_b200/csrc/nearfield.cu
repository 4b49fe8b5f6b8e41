// Nearfield quadrature kernels (sm_100a, FP64).
//
// Work is split by Sauter-Schwab case, as the reference's quadrature selection does per pair
// (select_quadrature_singquad2d, Library/singquad2d.c:549):
//   * near_dist_kernel — one CTA per output tile (<= 64 x 64 entries); one thread per distant
//     triangle pair (no shared vertex, q^4 tensor points, fully unrolled with the rule in
//     constant memory); pair results are accumulated in a shared-memory tile and the tile is
//     written to HBM once with coalesced column-major stores.  Singular pairs are skipped here.
//   * near_sing_kernel — one warp per singular pair (vertex: 2 q2^4 points; edge: 6 q2^3 and
//     identical: 6 q2^2 kernel evaluations, the rules reduced on the host because X - Y does not
//     depend on the inner Gauss variables there, see h2b_quad_reduce), lanes stride over the
//     points, the three Sauter-Schwab rules are staged once per
//     CTA into shared memory with bulk asynchronous copies (cp.async.bulk, global -> shared,
//     completion on an mbarrier), partial sums are combined with warp shuffles and the result is
//     written (constant basis) or added (linear basis) to the entries of its pair.
// The second kernel runs after the first on the same stream, so its stores/additions land on top
// of the distant-pair tile values.
//
// Per point the kernels evaluate the integrand of assemble_cc_near_bem3d (Library/bem3d.c:1151)
// and assemble_ll_near_bem3d (:3038) with the kernels of Library/laplacebem3d.c:36/84 and
// Library/helmholtzbem3d.c:27/140.  The quadrature point difference x - y is formed directly as
// (A_t - A_s) + t_x (B_t - A_t) + s_x (C_t - B_t) - t_y (B_s - A_s) - s_y (C_s - B_s), which is
// the reference's A(1-t) + B(t-s) + C s map on both triangles, without forming x and y first.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <type_traits>

#include "device_common.cuh"
#include "green.h"
#include "h2b200_plan.h"
#include "nearfield.h"

namespace {

constexpr int KK_LSLP = H2B_KK_LSLP;
constexpr int KK_LDLP = H2B_KK_LDLP;
constexpr int KK_LBOTH = H2B_KK_LBOTH;
constexpr int KK_HSLP = H2B_KK_HSLP;
constexpr int KK_HDLP = H2B_KK_HDLP;
constexpr int KK_LADLP = H2B_KK_LADLP;
constexpr int KK_HADLP = H2B_KK_HADLP;
constexpr int KK_HBOTH = H2B_KK_HBOTH;

template <int KK> struct KT;
template <> struct KT<KK_LSLP> { static constexpr int NCH = 1, NOUT = 1; static constexpr bool CPLX = false; };
template <> struct KT<KK_LDLP> { static constexpr int NCH = 1, NOUT = 1; static constexpr bool CPLX = false; };
template <> struct KT<KK_LBOTH> { static constexpr int NCH = 2, NOUT = 2; static constexpr bool CPLX = false; };
template <> struct KT<KK_HSLP> { static constexpr int NCH = 2, NOUT = 1; static constexpr bool CPLX = true; };
template <> struct KT<KK_HDLP> { static constexpr int NCH = 2, NOUT = 1; static constexpr bool CPLX = true; };
template <> struct KT<KK_LADLP> { static constexpr int NCH = 1, NOUT = 1; static constexpr bool CPLX = false; };
template <> struct KT<KK_HADLP> { static constexpr int NCH = 2, NOUT = 1; static constexpr bool CPLX = true; };
template <> struct KT<KK_HBOTH> { static constexpr int NCH = 4, NOUT = 2; static constexpr bool CPLX = true; };

// Distant tensor rules for q = 1..5 (q^4 points each): x0, x1, y0, y1, w.
constexpr int DIST_TOTAL = 1 + 16 + 81 + 256 + 625;
__host__ __device__ constexpr int dist_off(int q) {
  return q == 1 ? 0 : q == 2 ? 1 : q == 3 ? 17 : q == 4 ? 98 : 354;
}
__constant__ double c_dist[5][DIST_TOTAL];

// The distant rule is the tensor product of one q^2-point rule per triangle (the single-triangle
// rule of Library/singquad2d.c:25: t = g_i, s = g_i g_j, w = gw_i gw_j g_i), so its weight
// factors as w = w_x w_y.  Per order q and point p < q^2: rows t, s, w, w (1-t), w (t-s), w s
// (the raw weight and the three linear nodal functions times the weight).
constexpr int SIDE_MAXP = 25;
__constant__ double c_side[5][6][SIDE_MAXP];

// Kernel values from r^2 = |x - y|^2 and dot = <x - y, n> with n the unit normal of the column
// triangle (double layer) or of the row triangle (adjoint double layer, whose kernels take
// <y - x, n_x> = -dot: Library/laplacebem3d.c:136, Library/helmholtzbem3d.c:209).
template <int KK>
__device__ __forceinline__ void eval_kernel(double r2, double dot, double k_re, double k_imn,
                                            double kv[4]) {
  double rinv = rsqrt_nr(r2);
  if constexpr (KK == KK_LSLP) {
    kv[0] = rinv;
  } else if constexpr (KK == KK_LDLP) {
    kv[0] = dot * (rinv * rinv * rinv);
  } else if constexpr (KK == KK_LADLP) {
    kv[0] = -dot * (rinv * rinv * rinv);
  } else if constexpr (KK == KK_LBOTH) {
    kv[0] = rinv;
    kv[1] = dot * (rinv * rinv * rinv);
  } else if constexpr (KK == KK_HSLP) {
    double r = r2 * rinv, rn = rinv, s, c;
    if (k_imn != 0.0) rn *= exp(k_imn * r);
    sincos(k_re * r, &s, &c);
    kv[0] = rn * c;
    kv[1] = rn * s;
  } else if constexpr (KK == KK_HBOTH) {
    // single layer in kv[0..1], double layer in kv[2..3]: one sine and cosine for both
    double r = r2 * rinv, rn = rinv, re = (rinv * rinv * rinv) * dot, s, c;
    if (k_imn != 0.0) {
      const double e = exp(k_imn * r);
      rn *= e;
      re *= e;
    }
    const double kr = k_re * r;
    sincos(kr, &s, &c);
    kv[0] = rn * c;
    kv[1] = rn * s;
    kv[2] = fma(kr, s, c) * re;
    kv[3] = fma(-c, kr, s) * re;
  } else {  // KK_HDLP, KK_HADLP
    double re = (rinv * rinv * rinv) * (KK == KK_HADLP ? -dot : dot), r = r2 * rinv, s, c;
    if (k_imn != 0.0) re *= exp(k_imn * r);
    double kr = k_re * r;
    sincos(kr, &s, &c);
    kv[0] = fma(kr, s, c) * re;
    kv[1] = fma(-c, kr, s) * re;
  }
}

template <int KK>
constexpr bool uses_normal() {
  return KK == KK_LDLP || KK == KK_LBOTH || KK == KK_HDLP || KK == KK_LADLP || KK == KK_HADLP ||
         KK == KK_HBOTH;
}

// the adjoint double layer differentiates in the row triangle's normal direction
template <int KK>
constexpr bool row_normal() {
  return KK == KK_LADLP || KK == KK_HADLP;
}

__device__ __forceinline__ double vtx(const TriRec &T, int i, int d) {
  return i == 0 ? T.a[d] : (i == 1 ? T.b[d] : T.c[d]);
}

// Pair geometry: D0 = A_t - A_s, P1 = B_t - A_t, P2 = C_t - B_t, Q1 = B_s - A_s, Q2 = C_s - B_s.
struct PairGeo {
  double d0[3], p1[3], p2[3], q1[3], q2[3];
};

__device__ __forceinline__ void pair_geo(const TriRec &T, const TriRec &S, const int tp[3],
                                         const int sp[3], PairGeo &g) {
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double ta = vtx(T, tp[0], d), tb = vtx(T, tp[1], d), tc = vtx(T, tp[2], d);
    double sa = vtx(S, sp[0], d), sb = vtx(S, sp[1], d), sc = vtx(S, sp[2], d);
    g.d0[d] = ta - sa;
    g.p1[d] = tb - ta;
    g.p2[d] = tc - tb;
    g.q1[d] = sb - sa;
    g.q2[d] = sc - sb;
  }
}

// Accumulate one quadrature point into acc[ch][i][j] (i row basis, j column basis).
template <int KK, bool RL, bool CL>
__device__ __forceinline__ void quad_point(const PairGeo &g, double tx, double sx, double ty,
                                           double sy, double w, double n0, double n1, double n2,
                                           double k_re, double k_imn,
                                           double (&acc)[KT<KK>::NCH][RL ? 3 : 1][CL ? 3 : 1]) {
  constexpr int NCH = KT<KK>::NCH;
  double dx = fma(-sy, g.q2[0], fma(-ty, g.q1[0], fma(sx, g.p2[0], fma(tx, g.p1[0], g.d0[0]))));
  double dy = fma(-sy, g.q2[1], fma(-ty, g.q1[1], fma(sx, g.p2[1], fma(tx, g.p1[1], g.d0[1]))));
  double dz = fma(-sy, g.q2[2], fma(-ty, g.q1[2], fma(sx, g.p2[2], fma(tx, g.p1[2], g.d0[2]))));
  double kv[4];
  const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
  const double dot = uses_normal<KK>() ? fma(dx, n0, fma(dy, n1, dz * n2)) : 0.0;
  eval_kernel<KK>(r2, dot, k_re, k_imn, kv);
  if constexpr (!RL && !CL) {
#pragma unroll
    for (int c = 0; c < NCH; c++) acc[c][0][0] = fma(w, kv[c], acc[c][0][0]);
  } else {
    double pr[3] = {1.0 - tx, tx - sx, sx};
    double pc[3] = {1.0 - ty, ty - sy, sy};
#pragma unroll
    for (int c = 0; c < NCH; c++) {
      double u[CL ? 3 : 1];
#pragma unroll
      for (int j = 0; j < (CL ? 3 : 1); j++) u[j] = (CL ? pc[j] * w : w) * kv[c];
#pragma unroll
      for (int i = 0; i < (RL ? 3 : 1); i++)
#pragma unroll
        for (int j = 0; j < (CL ? 3 : 1); j++)
          acc[c][i][j] = RL ? fma(pr[i], u[j], acc[c][i][j]) : acc[c][i][j] + u[j];
    }
  }
}

// One point of a reduced singular rule (h2b_quad_reduce): X - Y = d0 + a p1 + b p2 - c q2, and
// the basis-weighted weights are precomputed, w[(i + NR j) * ld] for the row / column basis
// functions i, j.  Several points of the full rule share this kernel value.
template <int KK, bool RL, bool CL>
__device__ __forceinline__ void quad_point_red(const PairGeo &g, double ra, double rb, double rc,
                                               const double *w, uint32_t ld, double n0, double n1,
                                               double n2, double k_re, double k_imn,
                                               double (&acc)[KT<KK>::NCH][RL ? 3 : 1][CL ? 3 : 1]) {
  constexpr int NCH = KT<KK>::NCH, NR = RL ? 3 : 1, NC = CL ? 3 : 1;
  const double dx = fma(-rc, g.q2[0], fma(rb, g.p2[0], fma(ra, g.p1[0], g.d0[0])));
  const double dy = fma(-rc, g.q2[1], fma(rb, g.p2[1], fma(ra, g.p1[1], g.d0[1])));
  const double dz = fma(-rc, g.q2[2], fma(rb, g.p2[2], fma(ra, g.p1[2], g.d0[2])));
  double kv[4];
  const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
  const double dot = uses_normal<KK>() ? fma(dx, n0, fma(dy, n1, dz * n2)) : 0.0;
  eval_kernel<KK>(r2, dot, k_re, k_imn, kv);
#pragma unroll
  for (int j = 0; j < NC; j++)
#pragma unroll
    for (int i = 0; i < NR; i++) {
      const double wij = w[(size_t) (i + NR * j) * ld];
#pragma unroll
      for (int c = 0; c < NCH; c++) acc[c][i][j] = fma(wij, kv[c], acc[c][i][j]);
    }
}

// One group of the common-vertex rule in tensor form (h2b_quad_vert_tensor, q2 = VT_Q): VT_Q row
// points x VT_Q column points, summed column side first as for distant pairs, so the basis
// weights are applied once per point instead of once per point pair.  With the shared vertex
// first in both triangles, X_a - Y_b = (d0 + x0 p1 + x1 p2) - (y0 q1 + y1 q2).  `t` is the
// packed group arrays (gn groups each), the row weights include the group weight.
constexpr int VT_Q = 4;
template <int KK, bool RL, bool CL>
__device__ __forceinline__ void vert_group_tensor(const PairGeo &g, const double *t, uint32_t gn,
                                                  uint32_t grp, double n0, double n1, double n2,
                                                  double k_re, double k_imn,
                                                  double (&acc)[KT<KK>::NCH][RL ? 3 : 1][CL ? 3 : 1]) {
  constexpr int NCH = KT<KK>::NCH, NR = RL ? 3 : 1, NC = CL ? 3 : 1;
  constexpr bool DOT = uses_normal<KK>();
  const double *col = t + (size_t) (2 + NR) * VT_Q * gn;
#pragma unroll 1
  for (int a = 0; a < VT_Q; a++) {
    const double *rp = t + (size_t) a * (2 + NR) * gn + grp;
    const double x0 = rp[0], x1 = rp[gn];
    double xa[3];
#pragma unroll
    for (int d = 0; d < 3; d++) xa[d] = fma(x0, g.p1[d], fma(x1, g.p2[d], g.d0[d]));
    double in[NCH][NC];
#pragma unroll
    for (int c = 0; c < NCH; c++)
#pragma unroll
      for (int j = 0; j < NC; j++) in[c][j] = 0.0;
#pragma unroll
    for (int b = 0; b < VT_Q; b++) {
      // column point formed here rather than kept for all a (register budget of 128)
      const double *cp = col + (size_t) b * (2 + NC) * gn + grp;
      const double y0 = cp[0], y1 = cp[gn];
      const double dx = xa[0] - fma(y0, g.q1[0], y1 * g.q2[0]);
      const double dy = xa[1] - fma(y0, g.q1[1], y1 * g.q2[1]);
      const double dz = xa[2] - fma(y0, g.q1[2], y1 * g.q2[2]);
      const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
      const double dot = DOT ? fma(dx, n0, fma(dy, n1, dz * n2)) : 0.0;
      double kv[4];
      eval_kernel<KK>(r2, dot, k_re, k_imn, kv);
#pragma unroll
      for (int j = 0; j < NC; j++) {
        const double w = cp[(size_t) (2 + j) * gn];
#pragma unroll
        for (int c = 0; c < NCH; c++) in[c][j] = fma(w, kv[c], in[c][j]);
      }
    }
#pragma unroll
    for (int i = 0; i < NR; i++) {
      const double w = rp[(size_t) (2 + i) * gn];
#pragma unroll
      for (int c = 0; c < NCH; c++)
#pragma unroll
        for (int j = 0; j < NC; j++) acc[c][i][j] = fma(w, in[c][j], acc[c][i][j]);
    }
  }
}

// Laplace kernels are homogeneous in x - y: degree -1 (single layer) or -2 (double layer and
// its adjoint), per output channel.
template <int KK>
__device__ __forceinline__ constexpr bool homogeneous_kk() {
  return KK == KK_LSLP || KK == KK_LDLP || KK == KK_LBOTH || KK == KK_LADLP;
}
template <int KK>
__device__ __forceinline__ constexpr int kk_degree(int c) {
  return (KK == KK_LSLP || (KK == KK_LBOTH && c == 0)) ? 1 : 2;
}

// One item of the merged common-vertex rule (h2b_quad_vert_merged, q2 = VT_Q): row point a of
// group (i, s) against the group's VT_Q column points.  The points are the tensor form's divided
// by the radial variable xi; the radial Gauss sum is folded into the column weights, one set per
// homogeneity degree of the kernel channel, so each point pair needs one kernel evaluation where
// the tensor form needs VT_Q.  With the shared vertex the origin of both triangles, the scaled
// difference is xh0 p1 + xh1 p2 - (yh0 q1 + yh1 q2).
template <int KK, bool RL, bool CL>
__device__ __forceinline__ void vert_item_merged(const PairGeo &g, const double *t, uint32_t n,
                                                 uint32_t k, double n0, double n1, double n2,
                                                 double (&acc)[KT<KK>::NCH][RL ? 3 : 1][CL ? 3 : 1]) {
  constexpr int NCH = KT<KK>::NCH, NR = RL ? 3 : 1, NC = CL ? 3 : 1;
  constexpr bool DOT = uses_normal<KK>();
  const double *col = t + (size_t) (2 + 2 * NR) * n;
  const uint32_t c0 = (k / VT_Q) * VT_Q;
  const double x0 = t[k], x1 = t[n + k];
  double xa[3];
#pragma unroll
  for (int d = 0; d < 3; d++) xa[d] = fma(x0, g.p1[d], x1 * g.p2[d]);
  double in[NCH][2][NC];
#pragma unroll
  for (int c = 0; c < NCH; c++)
#pragma unroll
    for (int j = 0; j < NC; j++) in[c][0][j] = in[c][1][j] = 0.0;
#pragma unroll
  for (int b = 0; b < VT_Q; b++) {
    const uint32_t cb = c0 + b;
    const double y0 = col[cb], y1 = col[n + cb];
    const double dx = xa[0] - fma(y0, g.q1[0], y1 * g.q2[0]);
    const double dy = xa[1] - fma(y0, g.q1[1], y1 * g.q2[1]);
    const double dz = xa[2] - fma(y0, g.q1[2], y1 * g.q2[2]);
    const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
    const double dot = DOT ? fma(dx, n0, fma(dy, n1, dz * n2)) : 0.0;
    double kv[4];
    eval_kernel<KK>(r2, dot, 0.0, 0.0, kv);
#pragma unroll
    for (int c = 0; c < NCH; c++) {
      const double *wc = col + (size_t) (2 + (kk_degree<KK>(c) - 1) * 2 * NC) * n + cb;
#pragma unroll
      for (int j = 0; j < NC; j++) {
        in[c][0][j] = fma(wc[(size_t) j * n], kv[c], in[c][0][j]);
        in[c][1][j] = fma(wc[(size_t) (NC + j) * n], kv[c], in[c][1][j]);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < NR; i++) {
    const double u = t[(size_t) (2 + i) * n + k], v = t[(size_t) (2 + NR + i) * n + k];
#pragma unroll
    for (int c = 0; c < NCH; c++)
#pragma unroll
      for (int j = 0; j < NC; j++) acc[c][i][j] = fma(u, in[c][0][j], fma(v, in[c][1][j], acc[c][i][j]));
  }
}

// One distant pair with the q^4 tensor rule in FP32 (mixed-precision assembly), summed column
// side first (w = w_x w_y, as dist_pair_points): the pair geometry is formed in
// FP64 relative to the column triangle's first vertex and rounded once; points, kernel values
// (rsqrtf, sincosf, expf) and the q^4 sums run in FP32; the pair's sums are widened to FP64
// before they are added to the tile.  Entries carry FP32 accuracy (~1e-7 relative).
__constant__ float c_side_f[5][6][SIDE_MAXP];

template <int KK>
__device__ __forceinline__ void eval_kernel_f(float r2, float dot, float k_re, float k_imn,
                                              float kv[4]) {
  const float rinv = rsqrtf(r2);
  if constexpr (KK == KK_LSLP) {
    kv[0] = rinv;
  } else if constexpr (KK == KK_LDLP) {
    kv[0] = dot * (rinv * rinv * rinv);
  } else if constexpr (KK == KK_LADLP) {
    kv[0] = -dot * (rinv * rinv * rinv);
  } else if constexpr (KK == KK_LBOTH) {
    kv[0] = rinv;
    kv[1] = dot * (rinv * rinv * rinv);
  } else if constexpr (KK == KK_HSLP) {
    float r = r2 * rinv, rn = rinv, s, c;
    if (k_imn != 0.0f) rn *= expf(k_imn * r);
    sincosf(k_re * r, &s, &c);
    kv[0] = rn * c;
    kv[1] = rn * s;
  } else if constexpr (KK == KK_HBOTH) {
    float r = r2 * rinv, rn = rinv, re = (rinv * rinv * rinv) * dot, s, c;
    if (k_imn != 0.0f) {
      const float e = expf(k_imn * r);
      rn *= e;
      re *= e;
    }
    const float kr = k_re * r;
    sincosf(kr, &s, &c);
    kv[0] = rn * c;
    kv[1] = rn * s;
    kv[2] = fmaf(kr, s, c) * re;
    kv[3] = fmaf(-c, kr, s) * re;
  } else {  // KK_HDLP, KK_HADLP
    float re = (rinv * rinv * rinv) * (KK == KK_HADLP ? -dot : dot), r = r2 * rinv, s, c;
    if (k_imn != 0.0f) re *= expf(k_imn * r);
    const float kr = k_re * r;
    sincosf(kr, &s, &c);
    kv[0] = fmaf(kr, s, c) * re;
    kv[1] = fmaf(-c, kr, s) * re;
  }
}

template <int Q, int KK, bool RL, bool CL>
__device__ __forceinline__ void dist_pair_tensor_f32(const PairGeo &g, double n0d, double n1d,
                                                     double n2d, double k_re, double k_imn,
                                                     double (&acc)[KT<KK>::NCH][RL ? 3 : 1][CL ? 3 : 1]) {
  constexpr int NCH = KT<KK>::NCH, NC = CL ? 3 : 1, NR = RL ? 3 : 1, P = Q * Q;
  constexpr bool DOT = uses_normal<KK>();
  const float(&sd)[6][SIDE_MAXP] = c_side_f[Q - 1];
  const float n0 = (float) n0d, n1 = (float) n1d, n2 = (float) n2d;
  const float kr = (float) k_re, ki = (float) k_imn;
  float d0[3], p1[3], p2[3], q1[3], q2[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    d0[d] = (float) g.d0[d];
    p1[d] = (float) g.p1[d];
    p2[d] = (float) g.p2[d];
    q1[d] = (float) g.q1[d];
    q2[d] = (float) g.q2[d];
  }
  float yb[P][3], nyb[P];
#pragma unroll
  for (int b = 0; b < P; b++) {
#pragma unroll
    for (int d = 0; d < 3; d++) yb[b][d] = fmaf(sd[1][b], q2[d], sd[0][b] * q1[d]);
    nyb[b] = DOT ? fmaf(yb[b][0], n0, fmaf(yb[b][1], n1, yb[b][2] * n2)) : 0.0f;
  }
  float accf[NCH][NR][NC];
#pragma unroll
  for (int c = 0; c < NCH; c++)
#pragma unroll
    for (int i = 0; i < NR; i++)
#pragma unroll
      for (int j = 0; j < NC; j++) accf[c][i][j] = 0.0f;
#pragma unroll
  for (int a = 0; a < P; a++) {
    float xa[3];
#pragma unroll
    for (int d = 0; d < 3; d++) xa[d] = fmaf(sd[1][a], p2[d], fmaf(sd[0][a], p1[d], d0[d]));
    const float nxa = DOT ? fmaf(xa[0], n0, fmaf(xa[1], n1, xa[2] * n2)) : 0.0f;
    float in[NCH][NC];
#pragma unroll
    for (int c = 0; c < NCH; c++)
#pragma unroll
      for (int j = 0; j < NC; j++) in[c][j] = 0.0f;
#pragma unroll
    for (int b = 0; b < P; b++) {
      const float dx = xa[0] - yb[b][0], dy = xa[1] - yb[b][1], dz = xa[2] - yb[b][2];
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      float kv[4];
      eval_kernel_f<KK>(r2, nxa - nyb[b], kr, ki, kv);
#pragma unroll
      for (int c = 0; c < NCH; c++)
#pragma unroll
        for (int j = 0; j < NC; j++) in[c][j] = fmaf(sd[CL ? 3 + j : 2][b], kv[c], in[c][j]);
    }
#pragma unroll
    for (int c = 0; c < NCH; c++)
#pragma unroll
      for (int i = 0; i < NR; i++)
#pragma unroll
        for (int j = 0; j < NC; j++)
          accf[c][i][j] = fmaf(sd[RL ? 3 + i : 2][a], in[c][j], accf[c][i][j]);
  }
#pragma unroll
  for (int c = 0; c < NCH; c++)
#pragma unroll
    for (int i = 0; i < NR; i++)
#pragma unroll
      for (int j = 0; j < NC; j++) acc[c][i][j] = (double) accf[c][i][j];
}

struct DistArgs {
  const TriRec *tri;
  const TriRef *refs;
  const h2b_tile *tiles;
  double *out0, *out1;
  double kconst, k_re, k_imn;
  int q;  // runtime q for the generic variant
};

// Shared-memory accumulator tile: [NOUT*(CPLX?2:1)][64*64] doubles.
// Resident CTAs per SM of the distant-pair kernel (register budget of 128 per thread).
constexpr int DIST_MINBLOCKS = 2;
// The tile's row and column triangles are staged in shared memory, structure of arrays, in
// chunks of DIST_CHUNK triangles per side (the pair loop then reads consecutive words per warp
// instead of one 128-byte record per lane from L1).
constexpr int DIST_CHUNK = 128;

// Staged triangles of one chunk pair.  Edge vectors are formed once per triangle here (the same
// subtractions pair_geo makes with the identity permutation).
struct DistStage {
  double r[13][DIST_CHUNK];  // row triangles: A (3), B - A (3), C - B (3), Gram determinant, n
  double c[13][DIST_CHUNK];  // column triangles: A, B - A, C - B, Gram determinant * kconst, n
  uint32_t rv[3][DIST_CHUNK], cv[3][DIST_CHUNK];  // vertex ids
  int32_t rl[3][DIST_CHUNK], cl[3][DIST_CHUNK];   // local output row / column per vertex
};

// Staged triangles of the q = 2 FP64 kernels: the four points of the one-triangle rule are formed
// once per triangle here (the tensor rule's points are their pairs), with each point's component
// along the triangle's own normal, so a pair only forms the differences.
constexpr int PT_X = 0, PT_G = 12, PT_N = 13, PT_DN = 16, PT_ROWS = 20;
struct DistStagePts {
  double r[PT_ROWS][DIST_CHUNK];  // row triangles: x_a (3 a + d), Gram determinant, n, <x_a, n>
  double c[PT_ROWS][DIST_CHUNK];  // column triangles: y_b, Gram determinant * kconst, n, <y_b, n>
  uint32_t rv[3][DIST_CHUNK], cv[3][DIST_CHUNK];  // vertex ids
  int32_t rl[3][DIST_CHUNK], cl[3][DIST_CHUNK];   // local output row / column per vertex
};

// Point e < 4 of the q = 2 one-triangle rule on (A, B, C): A + s0 (B - A) + s1 (C - B), and its
// component along n, into rows PT_X.., PT_DN.. of a stage array; the triangle's Gram determinant
// (times gscale) and normal into PT_G, PT_N..
__device__ __forceinline__ void stage_points(double (&st)[PT_ROWS][DIST_CHUNK], uint32_t e,
                                             const TriRec &T, double gscale) {
  const double(&sd)[6][SIDE_MAXP] = c_side[1];
#pragma unroll
  for (int a = 0; a < 4; a++) {
    double x[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      x[d] = fma(sd[1][a], T.c[d] - T.b[d], fma(sd[0][a], T.b[d] - T.a[d], T.a[d]));
      st[PT_X + 3 * a + d][e] = x[d];
    }
    st[PT_DN + a][e] = fma(x[0], T.n[0], fma(x[1], T.n[1], x[2] * T.n[2]));
  }
#pragma unroll
  for (int d = 0; d < 3; d++) st[PT_N + d][e] = T.n[d];
  st[PT_G][e] = T.g * gscale;
}

// One distant pair with the q = 2 tensor rule from staged points, summed column side first:
//   acc[c][i][j] = sum_a w_a phi_i(x_a) sum_b w_b phi_j(y_b) k_c(x_a, y_b).
// The normal component of x_a - y_b takes the staged component on the normal's own triangle
// and forms the other one here.  Same sum as quad_point over the q^4 points, in another order
// (differences at rounding level).
template <int KK, bool RL, bool CL>
__device__ __forceinline__ void dist_pair_points(const DistStagePts &sg, uint32_t ri, uint32_t ci,
                                                 double k_re, double k_imn,
                                                 double (&acc)[KT<KK>::NCH][RL ? 3 : 1][CL ? 3 : 1]) {
  constexpr int NCH = KT<KK>::NCH, NC = CL ? 3 : 1, NR = RL ? 3 : 1, P = 4;
  constexpr bool DOT = uses_normal<KK>(), RN = row_normal<KK>();
  const double(&sd)[6][SIDE_MAXP] = c_side[1];
  double n[3] = {0.0, 0.0, 0.0};
  if (DOT) {
#pragma unroll
    for (int d = 0; d < 3; d++) n[d] = RN ? sg.r[PT_N + d][ri] : sg.c[PT_N + d][ci];
  }
  double yb[P][3], nyb[P];
#pragma unroll
  for (int b = 0; b < P; b++) {
#pragma unroll
    for (int d = 0; d < 3; d++) yb[b][d] = sg.c[PT_X + 3 * b + d][ci];
    nyb[b] = !DOT ? 0.0
                  : RN ? fma(yb[b][0], n[0], fma(yb[b][1], n[1], yb[b][2] * n[2]))
                       : sg.c[PT_DN + b][ci];
  }
#pragma unroll
  for (int a = 0; a < P; a++) {
    double xa[3];
#pragma unroll
    for (int d = 0; d < 3; d++) xa[d] = sg.r[PT_X + 3 * a + d][ri];
    const double nxa = !DOT ? 0.0
                            : RN ? sg.r[PT_DN + a][ri]
                                 : fma(xa[0], n[0], fma(xa[1], n[1], xa[2] * n[2]));
    double in[NCH][NC];
#pragma unroll
    for (int c = 0; c < NCH; c++)
#pragma unroll
      for (int j = 0; j < NC; j++) in[c][j] = 0.0;
#pragma unroll
    for (int b = 0; b < P; b++) {
      const double dx = xa[0] - yb[b][0], dy = xa[1] - yb[b][1], dz = xa[2] - yb[b][2];
      const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
      double kv[4];
      eval_kernel<KK>(r2, nxa - nyb[b], k_re, k_imn, kv);
#pragma unroll
      for (int c = 0; c < NCH; c++)
#pragma unroll
        for (int j = 0; j < NC; j++) in[c][j] = fma(sd[CL ? 3 + j : 2][b], kv[c], in[c][j]);
    }
#pragma unroll
    for (int c = 0; c < NCH; c++)
#pragma unroll
      for (int i = 0; i < NR; i++)
#pragma unroll
        for (int j = 0; j < NC; j++)
          acc[c][i][j] = fma(sd[RL ? 3 + i : 2][a], in[c][j], acc[c][i][j]);
  }
}

// the stage of a kernel variant: staged points for the q = 2 FP64 kernels
template <int Q, bool F32>
using DistStageOf = std::conditional_t<Q == 2 && !F32, DistStagePts, DistStage>;

// Threads and resident CTAs of the distant-pair kernel: the four accumulator planes of the fused
// Helmholtz single and double layer fill most of the shared memory of an SM, so that kind runs
// one CTA of twice the threads.
template <int KK>
constexpr int dist_threads() { return KT<KK>::NCH == 4 ? 512 : 256; }
template <int KK>
constexpr int dist_minblocks() { return KT<KK>::NCH == 4 ? 1 : DIST_MINBLOCKS; }

template <int Q, int KK, bool RL, bool CL, bool F32 = false>
__global__ void __launch_bounds__(dist_threads<KK>(), dist_minblocks<KK>())
    near_dist_kernel(DistArgs a) {
  constexpr int NCH = KT<KK>::NCH;
  constexpr int NR = RL ? 3 : 1, NC = CL ? 3 : 1;
  constexpr int PLANES = NCH;  // accumulator planes: one per real channel
  constexpr int TS = H2B_TILE_MAX * H2B_TILE_MAX;
  extern __shared__ double sacc[];

  const h2b_tile tl = a.tiles[blockIdx.x];
  const int rows = tl.rows, cols = tl.cols;
  for (int e = threadIdx.x; e < PLANES * TS; e += blockDim.x) sacc[e] = 0.0;
  __syncthreads();

  const uint32_t ntr = tl.tr_len, nsc = tl.sc_len;
  const int q = Q > 0 ? Q : a.q;
  const int nq = q * q * q * q;
  const double *cx0 = &c_dist[0][dist_off(Q > 0 ? Q : 1)];
  const double *cx1 = &c_dist[1][dist_off(Q > 0 ? Q : 1)];
  const double *cy0 = &c_dist[2][dist_off(Q > 0 ? Q : 1)];
  const double *cy1 = &c_dist[3][dist_off(Q > 0 ? Q : 1)];
  const double *cw = &c_dist[4][dist_off(Q > 0 ? Q : 1)];
  if (Q == 0) {
    cx0 = &c_dist[0][dist_off(q)];
    cx1 = &c_dist[1][dist_off(q)];
    cy0 = &c_dist[2][dist_off(q)];
    cy1 = &c_dist[3][dist_off(q)];
    cw = &c_dist[4][dist_off(q)];
  }

  // Chunk pairs (column chunk outer): rows are restaged per chunk pair only when the tile has
  // more than one row chunk.  Lanes of a warp take consecutive row triangles of one column
  // triangle: the row arrays are read as consecutive words, the column arrays as a broadcast.
  constexpr bool PTS = Q == 2 && !F32;
  DistStageOf<Q, F32> &sg = *reinterpret_cast<DistStageOf<Q, F32> *>(sacc + PLANES * TS);
  for (uint32_t c0 = 0; c0 < nsc; c0 += DIST_CHUNK) {
    const uint32_t nc = min((uint32_t) DIST_CHUNK, nsc - c0);
    for (uint32_t r0 = 0; r0 < ntr; r0 += DIST_CHUNK) {
      const uint32_t nr = min((uint32_t) DIST_CHUNK, ntr - r0);
      if (r0 == 0 || ntr > (uint32_t) DIST_CHUNK) {
        if (c0 + r0 > 0) __syncthreads();  // the previous chunk pair is done with the stage
        if (r0 == 0) {
          for (uint32_t e = threadIdx.x; e < nc; e += blockDim.x) {
            const TriRef st = a.refs[tl.sc_off + c0 + e];
            const TriRec &S = a.tri[st.t];
            if constexpr (PTS) {
              stage_points(sg.c, e, S, a.kconst);
            } else {
#pragma unroll
              for (int d = 0; d < 3; d++) {
                sg.c[d][e] = S.a[d];
                sg.c[3 + d][e] = S.b[d] - S.a[d];
                sg.c[6 + d][e] = S.c[d] - S.b[d];
                sg.c[10 + d][e] = S.n[d];
              }
              sg.c[9][e] = S.g * a.kconst;
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
              sg.cv[d][e] = S.v[d];
              sg.cl[d][e] = st.l[d];
            }
          }
        }
        if (c0 == 0 || ntr > (uint32_t) DIST_CHUNK) {
          for (uint32_t e = threadIdx.x; e < nr; e += blockDim.x) {
            const TriRef rt = a.refs[tl.tr_off + r0 + e];
            const TriRec &T = a.tri[rt.t];
            if constexpr (PTS) {
              stage_points(sg.r, e, T, 1.0);
            } else {
#pragma unroll
              for (int d = 0; d < 3; d++) {
                sg.r[d][e] = T.a[d];
                sg.r[3 + d][e] = T.b[d] - T.a[d];
                sg.r[6 + d][e] = T.c[d] - T.b[d];
                sg.r[10 + d][e] = T.n[d];
              }
              sg.r[9][e] = T.g;
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
              sg.rv[d][e] = T.v[d];
              sg.rl[d][e] = rt.l[d];
            }
          }
        }
        __syncthreads();
      }
      // pair p = is * nr + it; the step of blockDim.x pairs advances (is, it) by (dq, dr)
      const uint32_t np = nr * nc, dq = blockDim.x / nr, dr = blockDim.x - dq * nr;
      uint32_t is = threadIdx.x / nr, it = threadIdx.x - is * nr;
      for (uint32_t p = threadIdx.x; p < np; p += blockDim.x) {
        const uint32_t ci = is, ri = it;
        is += dq;
        it += dr;
        if (it >= nr) {
          it -= nr;
          is++;
        }
        const uint32_t tv0 = sg.rv[0][ri], tv1 = sg.rv[1][ri], tv2 = sg.rv[2][ri];
        const uint32_t sv0 = sg.cv[0][ci], sv1 = sg.cv[1][ci], sv2 = sg.cv[2][ci];
        const bool singular = tv0 == sv0 || tv0 == sv1 || tv0 == sv2 || tv1 == sv0 ||
                              tv1 == sv1 || tv1 == sv2 || tv2 == sv0 || tv2 == sv1 || tv2 == sv2;
        if (singular) continue;
        double acc[NCH][NR][NC];
#pragma unroll
        for (int c = 0; c < NCH; c++)
#pragma unroll
          for (int i = 0; i < NR; i++)
#pragma unroll
            for (int j = 0; j < NC; j++) acc[c][i][j] = 0.0;
        double f2;
        if constexpr (PTS) {
          dist_pair_points<KK, RL, CL>(sg, ri, ci, a.k_re, a.k_imn, acc);
          f2 = sg.c[PT_G][ci] * sg.r[PT_G][ri];
        } else {
          PairGeo g;
#pragma unroll
          for (int d = 0; d < 3; d++) {
            g.d0[d] = sg.r[d][ri] - sg.c[d][ci];
            g.p1[d] = sg.r[3 + d][ri];
            g.p2[d] = sg.r[6 + d][ri];
            g.q1[d] = sg.c[3 + d][ci];
            g.q2[d] = sg.c[6 + d][ci];
          }
          const double(&nn)[13][DIST_CHUNK] = row_normal<KK>() ? sg.r : sg.c;
          const uint32_t ni = row_normal<KK>() ? ri : ci;
          const double n0 = nn[10][ni], n1 = nn[11][ni], n2 = nn[12][ni];
          if constexpr (Q > 0) {  // q = 2 in FP32 (the FP64 kernels stage points)
            dist_pair_tensor_f32<Q, KK, RL, CL>(g, n0, n1, n2, a.k_re, a.k_imn, acc);
          } else {
            for (int k = 0; k < nq; k++)
              quad_point<KK, RL, CL>(g, cx0[k], cx1[k], cy0[k], cy1[k], cw[k], n0, n1, n2,
                                     a.k_re, a.k_imn, acc);
          }
          f2 = sg.c[9][ci] * sg.r[9][ri];
        }
#pragma unroll
        for (int i = 0; i < NR; i++) {
          const int lr = sg.rl[i][ri];
#pragma unroll
          for (int j = 0; j < NC; j++) {
            const int lc = sg.cl[j][ci];
            if (lr < 0 || lc < 0) continue;
            const int e = lr + H2B_TILE_MAX * lc;
#pragma unroll
            for (int c = 0; c < NCH; c++) {
              const double v = acc[c][i][j] * f2;
              if constexpr (RL || CL)
                atomicAdd(&sacc[c * TS + e], v);
              else
                sacc[c * TS + e] = v;
            }
          }
        }
      }
    }
  }
  __syncthreads();

  const bool ntrans = tl.flags & 1u;
  for (int e = threadIdx.x; e < rows * cols; e += blockDim.x) {
    const int r = e % rows, c = e / rows;
    const uint64_t o = ntrans ? tl.out_off + c + (uint64_t) r * tl.ld
                              : tl.out_off + r + (uint64_t) c * tl.ld;
    const int se = r + H2B_TILE_MAX * c;
    if constexpr (KT<KK>::CPLX) {
      a.out0[2 * o] = sacc[se];
      a.out0[2 * o + 1] = ntrans ? -sacc[TS + se] : sacc[TS + se];
      if constexpr (KT<KK>::NOUT == 2) {
        a.out1[2 * o] = sacc[2 * TS + se];
        a.out1[2 * o + 1] = ntrans ? -sacc[3 * TS + se] : sacc[3 * TS + se];
      }
    } else {
      a.out0[o] = sacc[se];
      if constexpr (KT<KK>::NOUT == 2) a.out1[o] = sacc[TS + se];
    }
  }
}

struct SingArgs {
  const TriRec *tri;
  const TriRef *refs;
  const h2b_tile *tiles;
  const h2b_sing *sing;
  uint32_t nsing;
  double *out0, *out1;
  double kconst, k_re, k_imn;
  double alpha_re, alpha_im;  // identity coefficient of the double layer output
  double mass[9];
  const double *rule;         // packed singular rules: case 1 {x0,x1,y0,y1,w} x n_1, cases 2, 3
                              // {a,b,c, NR*NC weight rows} x n_c (reduced rules)
  uint32_t rule_n[5];         // points per case (index 1..3; 4: merged common-vertex rule)
  uint32_t rule_off[5];       // offset (in doubles) of each case's block in `rule`
  uint32_t rule_total;        // doubles in `rule` (multiple of 2, 16-byte aligned)
  int vert_tensor;            // 1: case 1 in tensor form (rule_n[1] groups, q2 = 4)
  int staged;                 // 1: copy `rule` into shared memory first
  int *err;                   // set to 1 if the staging copy did not complete
};


// One warp per singular pair.  The three rules are copied into shared memory once per CTA.
// 512 threads: one CTA per SM holds the staged rules, 16 warps hide the FP64 latencies.
constexpr int SING_THREADS = 512;
// PART selects the pairs a launch takes and so the code it carries (fewer live registers per
// launch): 0 every case, 1 common vertex in tensor form, 2 common edge / identical (reduced
// rules), 3 common vertex with the full rule.  `a.sing` / `a.nsing` are the launch's pairs.
template <int KK, bool RL, bool CL, int PART>
__global__ void __launch_bounds__(SING_THREADS, 1) near_sing_kernel(SingArgs a) {
  constexpr int NCH = KT<KK>::NCH;
  constexpr int NR = RL ? 3 : 1, NC = CL ? 3 : 1;
  extern __shared__ __align__(16) double srule[];
  __shared__ __align__(8) uint64_t bar;

  // Stage the packed rule table: one bulk copy global -> shared, completion on an mbarrier.
  // Tables too large for shared memory are read from global memory (L2-resident) instead.
  const double *rules = a.rule;
  if (a.staged) {
    const uint32_t bytes = a.rule_total * 8u;
    const uint32_t sbar = (uint32_t) __cvta_generic_to_shared(&bar);
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sbar));
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t sdst = (uint32_t) __cvta_generic_to_shared(srule);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sbar), "r"(bytes)
                   : "memory");
      // chunks of at most 64 KiB; every chunk starts and ends on a 16-byte boundary
      for (uint32_t off = 0; off < bytes; off += 65536u) {
        const uint32_t n = bytes - off < 65536u ? bytes - off : 65536u;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                sdst + off),
            "l"(reinterpret_cast<const char *>(a.rule) + off), "r"(n), "r"(sbar)
            : "memory");
      }
    }
    // bounded wait on phase 0 of the barrier
    uint32_t done = 0;
    for (uint32_t spin = 0; spin < (1u << 24) && !done; spin++) {
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
          : "=r"(done)
          : "r"(sbar)
          : "memory");
    }
    if (!done) {
      if (threadIdx.x == 0) atomicExch(a.err, 1);
      return;
    }
    rules = srule;
  }

  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  // lanes per pair: a warp per pair for the full point rule; for the vertex rules (32 items of 4
  // kernel evaluations each in the merged form, 32 groups of 16 in the tensor form) and the
  // reduced edge / identical rules (384 / 96 items) 8 lanes take a pair and a warp four pairs,
  // so that the reduction over the lanes takes 3 shuffle steps instead of 5 per value.  A group
  // without a pair of its own repeats the warp's first pair and writes nothing, so every lane
  // takes part in the shuffles.
  constexpr int LPP = (PART == 4 || PART == 2 || PART == 1) ? 8 : 32;
  constexpr uint32_t PPW = 32 / LPP;
  const int sub = lane % LPP;

  for (uint32_t base = warp * PPW; base < a.nsing; base += nwarps * PPW) {
    const uint32_t pi = base + (uint32_t) (lane / LPP);
    const bool valid = pi < a.nsing;
    const h2b_sing sp = a.sing[valid ? pi : base];
    const uint32_t cs = sp.code & 3u;
    const int tp[3] = {(int) ((sp.code >> 2) & 3u), (int) ((sp.code >> 4) & 3u),
                       (int) ((sp.code >> 6) & 3u)};
    const int sq[3] = {(int) ((sp.code >> 8) & 3u), (int) ((sp.code >> 10) & 3u),
                       (int) ((sp.code >> 12) & 3u)};
    const TriRef rt = a.refs[sp.tr];
    const TriRef st = a.refs[sp.sc];
    const TriRec &T = a.tri[rt.t];
    const TriRec &S = a.tri[st.t];
    PairGeo g;
    pair_geo(T, S, tp, sq, g);
    const TriRec &NT = row_normal<KK>() ? T : S;  // triangle whose normal the kernel uses
    const double n0 = NT.n[0], n1 = NT.n[1], n2 = NT.n[2];
    const uint32_t n = a.rule_n[cs];
    const double *rx0 = rules + a.rule_off[cs];

    double acc[NCH][NR][NC];
#pragma unroll
    for (int c = 0; c < NCH; c++)
#pragma unroll
      for (int i = 0; i < NR; i++)
#pragma unroll
        for (int j = 0; j < NC; j++) acc[c][i][j] = 0.0;
    if (PART == 4) {
      // common vertex, Laplace kernel: the merged rule, one row point per lane
      const double *rm = rules + a.rule_off[4];
      for (uint32_t k = sub; k < a.rule_n[4]; k += LPP)
        vert_item_merged<KK, RL, CL>(g, rm, a.rule_n[4], k, n0, n1, n2, acc);
    } else if ((PART == 0 || PART == 1) && cs == 1u && (PART == 1 || a.vert_tensor)) {
      // common vertex, tensor form: a group of VT_Q x VT_Q points per lane
      for (uint32_t grp = sub; grp < n; grp += LPP)
        vert_group_tensor<KK, RL, CL>(g, rx0, n, grp, n0, n1, n2, a.k_re, a.k_imn, acc);
    } else if ((PART == 0 || PART == 3) && cs == 1u) {
      // common vertex: the full rule (x0, x1, y0, y1, raw weight)
      const double *rx1 = rx0 + n, *ry0 = rx0 + 2 * n, *ry1 = rx0 + 3 * n, *rw = rx0 + 4 * n;
#pragma unroll 1
      for (uint32_t k = lane; k < n; k += 32)
        quad_point<KK, RL, CL>(g, rx0[k], rx1[k], ry0[k], ry1[k], rw[k], n0, n1, n2, a.k_re,
                               a.k_imn, acc);
    } else if (PART == 0 || PART == 2) {
      // common edge / identical: the reduced rule (a, b, c, basis-weighted weights)
      const double *rb = rx0 + n, *rc = rx0 + 2 * n, *rwt = rx0 + 3 * n;
#pragma unroll 1
      for (uint32_t k = sub; k < n; k += LPP)
        quad_point_red<KK, RL, CL>(g, rx0[k], rb[k], rc[k], rwt + k, n, n0, n1, n2, a.k_re,
                                   a.k_imn, acc);
    }
#pragma unroll
    for (int c = 0; c < NCH; c++)
#pragma unroll
      for (int i = 0; i < NR; i++)
#pragma unroll
        for (int j = 0; j < NC; j++) {
#pragma unroll
          for (int o = LPP / 2; o > 0; o >>= 1)
            acc[c][i][j] += __shfl_xor_sync(0xffffffffu, acc[c][i][j], o);
        }

    if (sub == 0 && valid) {
      const h2b_tile tl = a.tiles[sp.tile];
      const bool ntrans = tl.flags & 1u;
      const double f2 = (S.g * a.kconst) * T.g;
      const bool ident = (cs == 3u) && (rt.t == st.t);
#pragma unroll
      for (int i = 0; i < NR; i++) {
        const int lr = RL ? rt.l[tp[i]] : rt.l[0];
#pragma unroll
        for (int j = 0; j < NC; j++) {
          const int lc = CL ? st.l[sq[j]] : st.l[0];
          if (lr < 0 || lc < 0) continue;
          const uint64_t o = ntrans ? tl.out_off + lc + (uint64_t) lr * tl.ld
                                    : tl.out_off + lr + (uint64_t) lc * tl.ld;
          if constexpr (!RL && !CL) {
            // constant basis: this pair is the whole entry
            if constexpr (KT<KK>::CPLX && KT<KK>::NOUT == 2) {
              // single layer to out0, double layer with the identity term to out1
              double re = acc[2][0][0] * f2, im = acc[3][0][0] * f2;
              if (ident) {
                re += 0.5 * a.alpha_re * T.g;
                im += 0.5 * a.alpha_im * T.g;
              }
              const double sre = acc[0][0][0] * f2, sim = acc[1][0][0] * f2;
              a.out0[2 * o] = sre;
              a.out0[2 * o + 1] = ntrans ? -sim : sim;
              a.out1[2 * o] = re;
              a.out1[2 * o + 1] = ntrans ? -im : im;
            } else if constexpr (KT<KK>::CPLX) {
              double re = acc[0][0][0] * f2, im = acc[1][0][0] * f2;
              if (ident) {
                re += 0.5 * a.alpha_re * T.g;
                im += 0.5 * a.alpha_im * T.g;
              }
              a.out0[2 * o] = re;
              a.out0[2 * o + 1] = ntrans ? -im : im;
            } else if constexpr (KT<KK>::NOUT == 2) {
              a.out0[o] = acc[0][0][0] * f2;
              a.out1[o] = acc[1][0][0] * f2 + (ident ? 0.5 * a.alpha_re * T.g : 0.0);
            } else {
              a.out0[o] = acc[0][0][0] * f2 + (ident ? 0.5 * a.alpha_re * T.g : 0.0);
            }
          } else {
            if constexpr (KT<KK>::CPLX) {
              atomicAdd(&a.out0[2 * o], acc[0][i][j] * f2);
              atomicAdd(&a.out0[2 * o + 1], (ntrans ? -1.0 : 1.0) * acc[1][i][j] * f2);
              if constexpr (KT<KK>::NOUT == 2) {
                atomicAdd(&a.out1[2 * o], acc[2][i][j] * f2);
                atomicAdd(&a.out1[2 * o + 1], (ntrans ? -1.0 : 1.0) * acc[3][i][j] * f2);
              }
            } else {
              atomicAdd(&a.out0[o], acc[0][i][j] * f2);
              if constexpr (KT<KK>::NOUT == 2) atomicAdd(&a.out1[o], acc[1][i][j] * f2);
            }
          }
        }
      }
      // identity term of linear bases: alpha * mass * g on the basis functions of the triangle
      // (ll: 3 x 3 mass matrix; cl / lc: 1/6 per vertex)
      if constexpr (RL || CL) {
        if (ident && (a.alpha_re != 0.0 || a.alpha_im != 0.0)) {
          double *dst = KT<KK>::NOUT == 2 ? a.out1 : a.out0;
          for (int l = 0; l < NR; l++)
            for (int k = 0; k < NC; k++) {
              const int lr = rt.l[l], lc = st.l[k];
              if (lr < 0 || lc < 0) continue;
              const uint64_t o = ntrans ? tl.out_off + lc + (uint64_t) lr * tl.ld
                                        : tl.out_off + lr + (uint64_t) lc * tl.ld;
              const double m = (RL && CL ? a.mass[l + 3 * k] : a.mass[RL ? l : k]) * T.g;
              if constexpr (KT<KK>::CPLX) {
                atomicAdd(&dst[2 * o], m * a.alpha_re);
                atomicAdd(&dst[2 * o + 1], (ntrans ? -1.0 : 1.0) * m * a.alpha_im);
              } else {
                atomicAdd(&dst[o], m * a.alpha_re);
              }
            }
        }
      }
    }
  }
}

template <int Q, int KK, bool RL, bool CL, bool F32 = false>
int launch_dist(const h2b_near_launch *L, cudaStream_t st) {
  constexpr int PLANES = KT<KK>::NCH;
  const size_t smem = sizeof(double) * PLANES * H2B_TILE_MAX * H2B_TILE_MAX +
                      sizeof(DistStageOf<Q, F32>);
  H2B_CUDA_TRY((h2b_allow_smem<near_dist_kernel<Q, KK, RL, CL, F32>>()));
  DistArgs a;
  a.tri = (const TriRec *) L->tri;
  a.refs = (const TriRef *) L->refs;
  a.tiles = L->tiles;
  a.out0 = L->out0;
  a.out1 = L->out1;
  a.kconst = L->kconst;
  a.k_re = L->k_re;
  a.k_imn = L->k_imn;
  a.q = (int) L->q;
  if (L->ntiles > 0) {
    near_dist_kernel<Q, KK, RL, CL, F32><<<L->ntiles, dist_threads<KK>(), smem, st>>>(a);
    h2b_note_launch();
  }
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

template <int KK, bool RL, bool CL, int PART>
int launch_sing_part(const h2b_near_launch *L, uint32_t first, uint32_t count, cudaStream_t st) {
  if (count == 0) return H2B_OK;
  const int staged = sizeof(double) * L->rule_total <= 200u * 1024u;
  const size_t smem = staged ? sizeof(double) * L->rule_total : 0;
  H2B_CUDA_TRY((h2b_allow_smem<near_sing_kernel<KK, RL, CL, PART>>()));
  SingArgs a;
  a.tri = (const TriRec *) L->tri;
  a.refs = (const TriRef *) L->refs;
  a.tiles = L->tiles;
  a.sing = L->sing + first;
  a.nsing = count;
  a.out0 = L->out0;
  a.out1 = L->out1;
  a.kconst = L->kconst;
  a.k_re = L->k_re;
  a.k_imn = L->k_imn;
  a.alpha_re = L->alpha_re;
  a.alpha_im = L->alpha_im;
  for (int i = 0; i < 9; i++) a.mass[i] = L->mass[i];
  a.rule = L->rule;
  for (int i = 0; i < 5; i++) {
    a.rule_n[i] = L->rule_n[i];
    a.rule_off[i] = L->rule_off[i];
  }
  a.rule_total = L->rule_total;
  a.vert_tensor = L->vert_tensor;
  a.staged = staged;
  a.err = L->err;
  int sms = L->num_sms > 0 ? L->num_sms : 148;
  const uint32_t wpc = SING_THREADS / 32;
  uint32_t want = (count + wpc - 1) / wpc;
  uint32_t grid = want < (uint32_t) sms ? want : (uint32_t) sms;
  near_sing_kernel<KK, RL, CL, PART><<<grid, SING_THREADS, smem, st>>>(a);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

// The singular pairs are sorted by case (common vertex first).  When the number of vertex pairs
// is known, the vertex pairs and the edge / identical pairs run as two launches of specialised
// kernels; otherwise one launch handles every case.
template <int KK, bool RL, bool CL>
int launch_sing(const h2b_near_launch *L, cudaStream_t st) {
  if (L->nsing == 0) return H2B_OK;
  if (L->nvert > L->nsing) return launch_sing_part<KK, RL, CL, 0>(L, 0, L->nsing, st);
  int rc;
  if constexpr (homogeneous_kk<KK>())
    rc = L->vert_merged   ? launch_sing_part<KK, RL, CL, 4>(L, 0, L->nvert, st)
         : L->vert_tensor ? launch_sing_part<KK, RL, CL, 1>(L, 0, L->nvert, st)
                          : launch_sing_part<KK, RL, CL, 3>(L, 0, L->nvert, st);
  else
    rc = L->vert_tensor ? launch_sing_part<KK, RL, CL, 1>(L, 0, L->nvert, st)
                        : launch_sing_part<KK, RL, CL, 3>(L, 0, L->nvert, st);
  if (rc != H2B_OK) return rc;
  return launch_sing_part<KK, RL, CL, 2>(L, L->nvert, L->nsing - L->nvert, st);
}

template <int KK, bool RL, bool CL>
int launch_kk_basis(const h2b_near_launch *L, cudaStream_t st) {
  int rc;
  if (L->q == 2 && L->fp32)
    rc = launch_dist<2, KK, RL, CL, true>(L, st);
  else if (L->q == 2)
    rc = launch_dist<2, KK, RL, CL>(L, st);
  else
    rc = launch_dist<0, KK, RL, CL>(L, st);
  if (rc != H2B_OK) return rc;
  if (L->ev_between) H2B_CUDA_TRY(cudaEventRecord(L->ev_between, st));
  return launch_sing<KK, RL, CL>(L, st);
}

template <int KK>
int launch_kk(const h2b_near_launch *L, cudaStream_t st) {
  if (L->row_linear && L->col_linear) return launch_kk_basis<KK, true, true>(L, st);
  if (L->row_linear) return launch_kk_basis<KK, true, false>(L, st);
  if (L->col_linear) return launch_kk_basis<KK, false, true>(L, st);
  return launch_kk_basis<KK, false, false>(L, st);
}

// Vertex permutation of a pair, the device twin of h2b_pair_code (host_plan.c): number of shared
// vertices in bits 0-1, the row triangle's order (shared vertices first) in bits 2-7, the column
// triangle's in bits 8-13 (select_quadrature_singquad2d, Library/singquad2d.c:549).
__device__ uint32_t pair_code_dev(const uint32_t tv[3], const uint32_t sv[3]) {
  uint32_t p = 0, tp[3] = {0, 1, 2}, sp[3] = {0, 1, 2};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) p += (tv[i] == sv[j]);
  if (p == 1 || p == 2) {
    uint32_t c = 0;
    for (uint32_t i = 0; i < 3; i++)
      for (uint32_t j = 0; j < 3; j++)
        if (tv[i] == sv[j]) {
          tp[c] = i;
          sp[c] = j;
          c++;
          break;
        }
    uint32_t q = c;
    for (uint32_t i = 0; i < 3; i++) {
      uint32_t j = 0;
      while (j < q && tv[i] != tv[tp[j]]) j++;
      if (j == q) tp[q++] = i;
    }
    q = c;
    for (uint32_t i = 0; i < 3; i++) {
      uint32_t j = 0;
      while (j < q && sv[i] != sv[sp[j]]) j++;
      if (j == q) sp[q++] = i;
    }
  }
  if (p > 3) p = 3;
  return p | (tp[0] << 2) | (tp[1] << 4) | (tp[2] << 6) | (sp[0] << 8) | (sp[1] << 10) |
         (sp[2] << 12);
}

// Every pair of one tile tested for a shared vertex (the fallback of classify_kernel for long
// column lists); warp-aggregated atomics per case.  The tile's vertex ids are staged in shared
// memory in chunks of CL_CHUNK triangles per side (a warp then reads consecutive words, or one
// broadcast word, instead of one triangle record per lane).
constexpr int CL_CHUNK = 256;
template <bool WRITE>
__device__ void classify_all_pairs(const TriRec *tri, const TriRef *refs, const h2b_tile &tl,
                                   uint32_t *cursor, const uint32_t *base, h2b_sing *out) {
  __shared__ uint32_t rv[3][CL_CHUNK], cv[3][CL_CHUNK];
  const uint32_t ntr = tl.tr_len, nsc = tl.sc_len;
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t c0 = 0; c0 < nsc; c0 += CL_CHUNK) {
    const uint32_t nc = min((uint32_t) CL_CHUNK, nsc - c0);
    for (uint32_t r0 = 0; r0 < ntr; r0 += CL_CHUNK) {
      const uint32_t nr = min((uint32_t) CL_CHUNK, ntr - r0);
      __syncthreads();  // the previous chunk pair is done with the stage
      for (uint32_t e = threadIdx.x; e < nr; e += blockDim.x) {
        const TriRec &T = tri[refs[tl.tr_off + r0 + e].t];
        rv[0][e] = T.v[0];
        rv[1][e] = T.v[1];
        rv[2][e] = T.v[2];
      }
      for (uint32_t e = threadIdx.x; e < nc; e += blockDim.x) {
        const TriRec &S = tri[refs[tl.sc_off + c0 + e].t];
        cv[0][e] = S.v[0];
        cv[1][e] = S.v[1];
        cv[2][e] = S.v[2];
      }
      __syncthreads();
      const uint32_t np = nr * nc;
      for (uint32_t p0 = 0; p0 < np; p0 += blockDim.x) {
        const uint32_t p = p0 + threadIdx.x;
        uint32_t code = 0, cs = 0, is = 0, it = 0;
        if (p < np) {
          is = p / nr;
          it = p - is * nr;
          const uint32_t tv[3] = {rv[0][it], rv[1][it], rv[2][it]};
          const uint32_t sv[3] = {cv[0][is], cv[1][is], cv[2][is]};
          bool shared = false;
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) shared |= tv[i] == sv[j];
          if (shared) {
            code = pair_code_dev(tv, sv);
            cs = code & 3u;
          }
        }
        // every thread of the warp reaches the ballots (the loop bound is uniform per CTA)
#pragma unroll
        for (uint32_t c = 1; c <= 3; c++) {
          const unsigned m = __ballot_sync(0xffffffffu, cs == c);
          if (m == 0) continue;
          const uint32_t leader = __ffs(m) - 1;
          uint32_t b = 0;
          if (lane == leader) b = atomicAdd(&cursor[c], (uint32_t) __popc(m));
          b = __shfl_sync(0xffffffffu, b, leader);
          if (WRITE && cs == c) {
            h2b_sing sg;
            sg.tile = blockIdx.x;
            sg.tr = tl.tr_off + r0 + it;
            sg.sc = tl.sc_off + c0 + is;
            sg.code = code;
            out[base[c] + b + __popc(m & ((1u << lane) - 1u))] = sg;
          }
        }
      }
    }
  }
}

// Distinct triangle pairs of a tile list: every pair (t, s) of a tile sets bit t * nt + s of a
// bitmap, and a pair whose bit was clear before counts once, by the number of vertices it shares
// (0 distant, 1 common vertex, 2 common edge, 3 identical).  Staged like classify_kernel.
__global__ void __launch_bounds__(256) unique_pairs_kernel(const TriRec *tri, const TriRef *refs,
                                                           const h2b_tile *tiles, uint64_t nt,
                                                           uint32_t *bitmap,
                                                           unsigned long long *counts) {
  __shared__ uint32_t rv[4][CL_CHUNK], cv[4][CL_CHUNK];
  __shared__ unsigned long long cnt[4];
  if (threadIdx.x < 4) cnt[threadIdx.x] = 0;
  const h2b_tile tl = tiles[blockIdx.x];
  const uint32_t ntr = tl.tr_len, nsc = tl.sc_len;
  for (uint32_t c0 = 0; c0 < nsc; c0 += CL_CHUNK) {
    const uint32_t nc = min((uint32_t) CL_CHUNK, nsc - c0);
    for (uint32_t r0 = 0; r0 < ntr; r0 += CL_CHUNK) {
      const uint32_t nr = min((uint32_t) CL_CHUNK, ntr - r0);
      __syncthreads();  // the previous chunk pair is done with the stage (and cnt is zeroed)
      for (uint32_t e = threadIdx.x; e < nr; e += blockDim.x) {
        const uint32_t t = refs[tl.tr_off + r0 + e].t;
        const TriRec &T = tri[t];
        rv[0][e] = T.v[0];
        rv[1][e] = T.v[1];
        rv[2][e] = T.v[2];
        rv[3][e] = t;
      }
      for (uint32_t e = threadIdx.x; e < nc; e += blockDim.x) {
        const uint32_t t = refs[tl.sc_off + c0 + e].t;
        const TriRec &S = tri[t];
        cv[0][e] = S.v[0];
        cv[1][e] = S.v[1];
        cv[2][e] = S.v[2];
        cv[3][e] = t;
      }
      __syncthreads();
      const uint32_t np = nr * nc;
      for (uint32_t p = threadIdx.x; p < np; p += blockDim.x) {
        const uint32_t is = p / nr, it = p - is * nr;
        uint32_t shared = 0;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) shared += rv[i][it] == cv[j][is];
        const uint64_t bit = (uint64_t) rv[3][it] * nt + cv[3][is];
        const uint32_t m = 1u << (bit & 31);
        if (!(atomicOr(&bitmap[bit >> 5], m) & m)) atomicAdd(&cnt[min(shared, 3u)], 1ull);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < 4 && cnt[threadIdx.x]) atomicAdd(&counts[threadIdx.x], cnt[threadIdx.x]);
}


// One CTA per tile.  The tile's column triangles go into a shared-memory hash table (triangle id
// -> position in the column list); a thread per row triangle t visits the triangles around t's
// vertices (the surface's vertex -> triangle lists) and looks each one up, so the pairs found are
// exactly the tile's pairs that share a vertex, without testing the others.  A triangle around
// several vertices of t is taken at the first of them.  Counts per case are gathered in shared
// memory: the count pass adds them to cursor[c]; the write pass reserves the tile's range of
// case c with one atomic and writes its pairs there.  Column lists longer than half the table
// take classify_all_pairs.
constexpr int CL_HASH = 1024;  // slots, a power of two
__device__ __forceinline__ uint32_t cl_slot(uint32_t t) { return (t * 2654435761u) >> 22; }

template <bool WRITE>
__global__ void __launch_bounds__(256) classify_kernel(const TriRec *tri, const TriRef *refs,
                                                       const h2b_tile *tiles,
                                                       const uint32_t *vt_off,
                                                       const uint32_t *vt_tri, uint32_t *cursor,
                                                       const uint32_t *base, h2b_sing *out) {
  __shared__ uint32_t hkey[CL_HASH];
  __shared__ uint32_t hval[CL_HASH];
  __shared__ uint32_t cnt[4], cur[4], rsv[4];
  const h2b_tile tl = tiles[blockIdx.x];
  const uint32_t ntr = tl.tr_len, nsc = tl.sc_len;
  if (nsc > (uint32_t) CL_HASH / 2) {
    classify_all_pairs<WRITE>(tri, refs, tl, cursor, base, out);
    return;
  }
  for (uint32_t e = threadIdx.x; e < (uint32_t) CL_HASH; e += blockDim.x) hkey[e] = UINT32_MAX;
  if (threadIdx.x < 4) cnt[threadIdx.x] = cur[threadIdx.x] = 0;
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < nsc; e += blockDim.x) {
    const uint32_t t = refs[tl.sc_off + e].t;
    uint32_t h = cl_slot(t);
    while (atomicCAS(&hkey[h], UINT32_MAX, t) != UINT32_MAX) h = (h + 1) & (CL_HASH - 1);
    hval[h] = e;
  }
  __syncthreads();
  // pass 0 counts the tile's pairs per case; pass 1 (write pass only) writes them
  for (int pass = 0; pass < (WRITE ? 2 : 1); pass++) {
    for (uint32_t i = threadIdx.x; i < ntr; i += blockDim.x) {
      const uint32_t t = refs[tl.tr_off + i].t;
      const uint32_t tv[3] = {tri[t].v[0], tri[t].v[1], tri[t].v[2]};
#pragma unroll
      for (int k = 0; k < 3; k++) {
        for (uint32_t a = vt_off[tv[k]]; a < vt_off[tv[k] + 1]; a++) {
          const uint32_t s = vt_tri[a];
          const uint32_t sv[3] = {tri[s].v[0], tri[s].v[1], tri[s].v[2]};
          bool seen = false;
#pragma unroll
          for (int k2 = 0; k2 < k; k2++) seen |= sv[0] == tv[k2] || sv[1] == tv[k2] || sv[2] == tv[k2];
          if (seen) continue;
          uint32_t h = cl_slot(s);
          while (hkey[h] != s && hkey[h] != UINT32_MAX) h = (h + 1) & (CL_HASH - 1);
          if (hkey[h] != s) continue;
          const uint32_t code = pair_code_dev(tv, sv), c = code & 3u;
          if (pass == 0) {
            atomicAdd(&cnt[c], 1u);
          } else {
            h2b_sing sg;
            sg.tile = blockIdx.x;
            sg.tr = tl.tr_off + i;
            sg.sc = tl.sc_off + hval[h];
            sg.code = code;
            out[base[c] + rsv[c] + atomicAdd(&cur[c], 1u)] = sg;
          }
        }
      }
    }
    __syncthreads();
    if (pass == 0 && threadIdx.x >= 1 && threadIdx.x <= 3 && cnt[threadIdx.x]) {
      const uint32_t b = atomicAdd(&cursor[threadIdx.x], cnt[threadIdx.x]);
      if (WRITE) rsv[threadIdx.x] = b;
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" int h2b_near_classify(const void *tri, const void *refs, const h2b_tile *tiles,
                                 uint32_t ntiles, const uint32_t *vt_off, const uint32_t *vt_tri,
                                 uint32_t *cursor, const uint32_t *base, h2b_sing *sing,
                                 cudaStream_t st) {
  if (ntiles == 0) return H2B_OK;
  if (sing)
    classify_kernel<true><<<ntiles, 256, 0, st>>>((const TriRec *) tri, (const TriRef *) refs,
                                                  tiles, vt_off, vt_tri, cursor, base, sing);
  else
    classify_kernel<false><<<ntiles, 256, 0, st>>>((const TriRec *) tri, (const TriRef *) refs,
                                                   tiles, vt_off, vt_tri, cursor, nullptr,
                                                   nullptr);
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

extern "C" int h2b_near_unique_pairs(const void *tri, const void *refs, const h2b_tile *tiles,
                                     uint32_t ntiles, uint32_t nt, uint64_t counts[4],
                                     cudaStream_t st) {
  for (int c = 0; c < 4; c++) counts[c] = 0;
  if (ntiles == 0) return H2B_OK;
  if (nt > H2B_UNIQUE_PAIRS_MAX_TRIANGLES) {
    h2b_set_error("unique pair count: %u triangles (the bitmap covers at most %u)", nt,
                  (unsigned) H2B_UNIQUE_PAIRS_MAX_TRIANGLES);
    return H2B_ERR_ARG;
  }
  const size_t words = ((uint64_t) nt * nt + 31) / 32;
  uint32_t *bitmap = nullptr;
  unsigned long long *d_cnt = nullptr;
  if (cudaMallocAsync((void **) &bitmap, 4 * words + 48, st) != cudaSuccess) {
    cudaGetLastError();
    h2b_set_error("unique pair count: no device memory for a %llu-byte bitmap",
                  (unsigned long long) (4 * words));
    return H2B_ERR_NOMEM;
  }
  d_cnt = (unsigned long long *) (bitmap + ((words + 1) & ~(size_t) 1));
  int rc = H2B_OK;
  unsigned long long host[4] = {0, 0, 0, 0};
  if (cudaMemsetAsync(bitmap, 0, 4 * words + 48, st) != cudaSuccess) rc = H2B_ERR_CUDA;
  if (rc == H2B_OK) {
    unique_pairs_kernel<<<ntiles, 256, 0, st>>>((const TriRec *) tri, (const TriRef *) refs,
                                                 tiles, nt, bitmap, d_cnt);
    h2b_note_launch();
    if (cudaGetLastError() != cudaSuccess) rc = H2B_ERR_CUDA;
  }
  if (rc == H2B_OK &&
      (cudaMemcpyAsync(host, d_cnt, sizeof(host), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
       cudaStreamSynchronize(st) != cudaSuccess))
    rc = H2B_ERR_CUDA;
  if (rc != H2B_OK) h2b_set_error("unique pair count: %s", cudaGetErrorString(cudaGetLastError()));
  cudaFreeAsync(bitmap, st);
  for (int c = 0; c < 4; c++) counts[c] = host[c];
  return rc;
}

// Greenhybrid coupling matrices S_b(i, j) = A(xihat_r[i], xihat_c[j]): the operator's entries
// between the pivot rows of the row cluster and the pivot columns of the column cluster
// (assemble_bem3d_greenhybrid_uniform, Library/bem3d.c:6493, through nearfield_far =
// assemble_{cc,ll}_far_bem3d, :1439 / :3264), the distant rule on every pair of triangles of the
// two basis functions.  K x K column-major per block, zero past the ranks.
template <int Q, bool RL, bool CL, bool DLP>
__global__ void __launch_bounds__(256) green_coupling_kernel(GreenCouplingArgs a) {
  const uint32_t b = blockIdx.x;
  const uint32_t rc = a.adm_rc[b], cc = a.adm_cc[b];
  const uint32_t K = (uint32_t) a.K, kr = a.rrank[rc], kc = a.crank[cc];
  const uint32_t *pr = a.rpiv + (size_t) rc * K, *pc = a.cpiv + (size_t) cc * K;
  double *S = a.S + (size_t) b * K * K;
  const int q = a.q, np = q * q * q * q, o = dist_off(q);
  for (uint32_t e = threadIdx.x; e < K * K; e += blockDim.x) {
    const uint32_t i = e % K, j = e / K;
    double acc = 0.0;
    if (i < kr && j < kc) {
      const uint32_t bi = pr[i], bj = pc[j];
      const uint32_t t0 = RL ? a.vt_off[bi] : 0u, t1 = RL ? a.vt_off[bi + 1] : 1u;
      const uint32_t u0 = CL ? a.vt_off[bj] : 0u, u1 = CL ? a.vt_off[bj + 1] : 1u;
      for (uint32_t ti = t0; ti < t1; ti++) {
        const TriRec &T = a.tri[RL ? a.vt_tri[ti] : bi];
        const int ct = RL ? (T.v[0] == bi ? 0 : (T.v[1] == bi ? 1 : 2)) : 0;
        if constexpr (Q > 0) {
          // the distant rule is one q^2-point rule per triangle (w = w_x w_y): the row
          // triangle's points and basis-weighted weights once per triangle, the column
          // triangle's once per pair
          constexpr int P = Q * Q;
          const double(&sd)[6][SIDE_MAXP] = c_side[Q - 1];
          double xa[P][3], wa[P];
#pragma unroll
          for (int p = 0; p < P; p++) {
            const double tx = sd[0][p], sx = sd[1][p];
            const double ax = 1.0 - tx, bx = tx - sx, cx = sx;
#pragma unroll
            for (int d = 0; d < 3; d++) xa[p][d] = T.a[d] * ax + T.b[d] * bx + T.c[d] * cx;
            wa[p] = RL ? sd[3 + ct][p] : sd[2][p];
          }
          for (uint32_t si = u0; si < u1; si++) {
            const TriRec &Sx = a.tri[CL ? a.vt_tri[si] : bj];
            const int cs = CL ? (Sx.v[0] == bj ? 0 : (Sx.v[1] == bj ? 1 : 2)) : 0;
            double part = 0.0;
#pragma unroll
            for (int p = 0; p < P; p++) {
              const double ty = sd[0][p], sy = sd[1][p];
              const double ay = 1.0 - ty, by = ty - sy, cy = sy;
              const double y0 = Sx.a[0] * ay + Sx.b[0] * by + Sx.c[0] * cy;
              const double y1 = Sx.a[1] * ay + Sx.b[1] * by + Sx.c[1] * cy;
              const double y2 = Sx.a[2] * ay + Sx.b[2] * by + Sx.c[2] * cy;
              double pb = 0.0;
#pragma unroll
              for (int r = 0; r < P; r++) {
                const double d0 = xa[r][0] - y0, d1 = xa[r][1] - y1, d2 = xa[r][2] - y2;
                const double ri = rsqrt_nr(fma(d0, d0, fma(d1, d1, d2 * d2)));
                const double f =
                    DLP ? fma(d0, Sx.n[0], fma(d1, Sx.n[1], d2 * Sx.n[2])) * (ri * ri * ri) : ri;
                pb = fma(wa[r], f, pb);
              }
              part = fma(CL ? sd[3 + cs][p] : sd[2][p], pb, part);
            }
            acc += part * (T.g * Sx.g * a.kconst);
          }
        } else {
          for (uint32_t si = u0; si < u1; si++) {
            const TriRec &Sx = a.tri[CL ? a.vt_tri[si] : bj];
            const int cs = CL ? (Sx.v[0] == bj ? 0 : (Sx.v[1] == bj ? 1 : 2)) : 0;
            double sum = 0.0;
            for (int p = 0; p < np; p++) {
              const double tx = c_dist[0][o + p], sx = c_dist[1][o + p];
              const double ty = c_dist[2][o + p], sy = c_dist[3][o + p], w = c_dist[4][o + p];
              const double ax = 1.0 - tx, bx = tx - sx, cx = sx;
              const double ay = 1.0 - ty, by = ty - sy, cy = sy;
              const double d0 = (T.a[0] * ax + T.b[0] * bx + T.c[0] * cx) -
                                (Sx.a[0] * ay + Sx.b[0] * by + Sx.c[0] * cy);
              const double d1 = (T.a[1] * ax + T.b[1] * bx + T.c[1] * cx) -
                                (Sx.a[1] * ay + Sx.b[1] * by + Sx.c[1] * cy);
              const double d2 = (T.a[2] * ax + T.b[2] * bx + T.c[2] * cx) -
                                (Sx.a[2] * ay + Sx.b[2] * by + Sx.c[2] * cy);
              const double ri = rsqrt_nr(d0 * d0 + d1 * d1 + d2 * d2);
              const double f =
                  DLP ? (d0 * Sx.n[0] + d1 * Sx.n[1] + d2 * Sx.n[2]) * (ri * ri * ri) : ri;
              const double pr_ = RL ? (ct == 0 ? ax : (ct == 1 ? bx : cx)) : 1.0;
              const double pc_ = CL ? (cs == 0 ? ay : (cs == 1 ? by : cy)) : 1.0;
              sum += w * pr_ * pc_ * f;
            }
            acc += sum * (T.g * Sx.g * a.kconst);
          }
        }
      }
    }
    S[i + (size_t) j * K] = acc;
  }
}

// The same entries with the column triangles staged once per block: for every pivot column its
// triangles' four rule points, their weights times the basis function, Gram determinant and
// 1/(4 pi), and the normal (q = 2).  A thread then reads its column's triangles from shared
// memory instead of forming their points once per row triangle.
template <bool RL, bool CL, bool DLP>
__global__ void __launch_bounds__(256) green_coupling_staged_kernel(GreenCouplingArgs a) {
  extern __shared__ __align__(16) unsigned char gsm[];
  constexpr int P = 4;
  const uint32_t b = blockIdx.x;
  const uint32_t rc = a.adm_rc[b], cc = a.adm_cc[b];
  const uint32_t K = (uint32_t) a.K, kr = a.rrank[rc], kc = a.crank[cc];
  const uint32_t *pr = a.rpiv + (size_t) rc * K, *pc = a.cpiv + (size_t) cc * K;
  double *S = a.S + (size_t) b * K * K;
  const double(&sd)[6][SIDE_MAXP] = c_side[1];
  uint32_t *coff = reinterpret_cast<uint32_t *>(gsm);           // K + 1 (padded to 16 bytes)
  double *cy = reinterpret_cast<double *>(gsm + 16 * ((4 * (K + 1) + 15) / 16));
  const uint32_t emax = (uint32_t) a.max_elems;
  double *cw = cy + (size_t) emax * 3 * P;                        // emax x P weights
  double *cn = cw + (size_t) emax * P;                            // emax x 3 normals
  if (threadIdx.x == 0) {
    uint32_t o = 0;
    for (uint32_t j = 0; j < kc; j++) {
      coff[j] = o;
      o += CL ? a.vt_off[pc[j] + 1] - a.vt_off[pc[j]] : 1u;
    }
    coff[kc] = o;
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < kc; j += blockDim.x) {
    const uint32_t bj = pc[j];
    const uint32_t u0 = CL ? a.vt_off[bj] : 0u, u1 = CL ? a.vt_off[bj + 1] : 1u;
    for (uint32_t u = u0; u < u1; u++) {
      const uint32_t f = coff[j] + (u - u0);
      const TriRec &Sx = a.tri[CL ? a.vt_tri[u] : bj];
      const int cs = CL ? (Sx.v[0] == bj ? 0 : (Sx.v[1] == bj ? 1 : 2)) : 0;
      const double gk = Sx.g * a.kconst;
      for (int p = 0; p < P; p++) {
        const double ty = sd[0][p], sy = sd[1][p];
        const double ay = 1.0 - ty, by = ty - sy, cy_ = sy;
        for (int d = 0; d < 3; d++)
          cy[((size_t) f * P + p) * 3 + d] = Sx.a[d] * ay + Sx.b[d] * by + Sx.c[d] * cy_;
        cw[(size_t) f * P + p] = (CL ? sd[3 + cs][p] : sd[2][p]) * gk;
      }
      for (int d = 0; d < 3; d++) cn[(size_t) f * 3 + d] = Sx.n[d];
    }
  }
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < K * K; e += blockDim.x) {
    const uint32_t i = e % K, j = e / K;
    double acc = 0.0;
    if (i < kr && j < kc) {
      const uint32_t bi = pr[i];
      const uint32_t t0 = RL ? a.vt_off[bi] : 0u, t1 = RL ? a.vt_off[bi + 1] : 1u;
      const uint32_t f0 = coff[j], f1 = coff[j + 1];
      for (uint32_t ti = t0; ti < t1; ti++) {
        const TriRec &T = a.tri[RL ? a.vt_tri[ti] : bi];
        const int ct = RL ? (T.v[0] == bi ? 0 : (T.v[1] == bi ? 1 : 2)) : 0;
        double xa[P][3], wa[P];
#pragma unroll
        for (int p = 0; p < P; p++) {
          const double tx = sd[0][p], sx = sd[1][p];
          const double ax = 1.0 - tx, bx = tx - sx, cx = sx;
#pragma unroll
          for (int d = 0; d < 3; d++) xa[p][d] = T.a[d] * ax + T.b[d] * bx + T.c[d] * cx;
          wa[p] = RL ? sd[3 + ct][p] : sd[2][p];
        }
        double part = 0.0;
        for (uint32_t f = f0; f < f1; f++) {
          const double *y = cy + (size_t) f * P * 3, *w = cw + (size_t) f * P;
          const double n0 = cn[3 * (size_t) f], n1 = cn[3 * (size_t) f + 1],
                       n2 = cn[3 * (size_t) f + 2];
#pragma unroll
          for (int p = 0; p < P; p++) {
            const double y0 = y[3 * p], y1 = y[3 * p + 1], y2 = y[3 * p + 2];
            double pb = 0.0;
#pragma unroll
            for (int r = 0; r < P; r++) {
              const double d0 = xa[r][0] - y0, d1 = xa[r][1] - y1, d2 = xa[r][2] - y2;
              const double ri = rsqrt_nr(fma(d0, d0, fma(d1, d1, d2 * d2)));
              const double fv = DLP ? fma(d0, n0, fma(d1, n1, d2 * n2)) * (ri * ri * ri) : ri;
              pb = fma(wa[r], fv, pb);
            }
            part = fma(w[p], pb, part);
          }
        }
        acc += part * T.g;
      }
    }
    S[i + (size_t) j * K] = acc;
  }
}

size_t green_coupling_smem(int K, uint32_t max_elems) {
  return 16 * ((4 * ((size_t) K + 1) + 15) / 16) + sizeof(double) * (size_t) max_elems * (12 + 4 + 3);
}

template <bool RL, bool CL, bool DLP>
static int launch_green_coupling(const GreenCouplingArgs *a, cudaStream_t st) {
  const size_t smem = green_coupling_smem(a->K, a->max_elems);
  if (a->q == 2 && smem <= H2B_MAX_DYN_SMEM) {
    H2B_CUDA_TRY((h2b_allow_smem<green_coupling_staged_kernel<RL, CL, DLP>>()));
    green_coupling_staged_kernel<RL, CL, DLP><<<a->n, 256, smem, st>>>(*a);
  } else if (a->q == 2) {
    green_coupling_kernel<2, RL, CL, DLP><<<a->n, 256, 0, st>>>(*a);
  } else {
    green_coupling_kernel<0, RL, CL, DLP><<<a->n, 256, 0, st>>>(*a);
  }
  h2b_note_launch();
  H2B_CUDA_TRY(cudaGetLastError());
  return H2B_OK;
}

template <bool RL, bool CL>
static int launch_green_coupling_l(const GreenCouplingArgs *a, cudaStream_t st) {
  return a->dlp ? launch_green_coupling<RL, CL, true>(a, st)
                : launch_green_coupling<RL, CL, false>(a, st);
}

extern "C" int h2b_green_coupling(const GreenCouplingArgs *a, cudaStream_t st) {
  if (a->n == 0) return H2B_OK;
  if (a->q < 1 || a->q > 5) {
    h2b_set_error("greenhybrid coupling: quadrature order %d outside 1..5", a->q);
    return H2B_ERR_ARG;
  }
  if (a->rlinear)
    return a->clinear ? launch_green_coupling_l<true, true>(a, st)
                      : launch_green_coupling_l<true, false>(a, st);
  return a->clinear ? launch_green_coupling_l<false, true>(a, st)
                    : launch_green_coupling_l<false, false>(a, st);
}

extern "C" int h2b_near_upload_dist_rules(void) {
  static double host[5][DIST_TOTAL];
  for (int q = 1; q <= 5; q++) {
    h2b_quad qd;
    int rc = h2b_quad_build((uint32_t) q, 1, H2B_BASIS_CONSTANT, H2B_BASIS_CONSTANT, &qd);
    if (rc != H2B_OK) return rc;
    const h2b_rule *r = &qd.rule[H2B_RULE_DIST];
    for (uint32_t k = 0; k < r->n; k++) {
      host[0][dist_off(q) + k] = r->x0[k];
      host[1][dist_off(q) + k] = r->x1[k];
      host[2][dist_off(q) + k] = r->y0[k];
      host[3][dist_off(q) + k] = r->y1[k];
      host[4][dist_off(q) + k] = r->w[9 * (size_t) r->n + k];
    }
    h2b_quad_free(&qd);
  }
  H2B_CUDA_TRY(cudaMemcpyToSymbol(c_dist, host, sizeof(host)));

  static double side[5][6][SIDE_MAXP];
  memset(side, 0, sizeof(side));
  for (int q = 1; q <= 5; q++) {
    double g[8], gw[8];
    int rc = h2b_gauss_legendre01((uint32_t) q, g, gw);
    if (rc != H2B_OK) return rc;
    for (int i = 0, p = 0; i < q; i++)
      for (int j = 0; j < q; j++, p++) {
        const double t = g[i], s = g[i] * g[j], w = gw[i] * gw[j] * g[i];
        side[q - 1][0][p] = t;
        side[q - 1][1][p] = s;
        side[q - 1][2][p] = w;
        side[q - 1][3][p] = w * (1.0 - t);
        side[q - 1][4][p] = w * (t - s);
        side[q - 1][5][p] = w * s;
      }
  }
  H2B_CUDA_TRY(cudaMemcpyToSymbol(c_side, side, sizeof(side)));
  static float side_f[5][6][SIDE_MAXP];
  for (int q = 0; q < 5; q++)
    for (int r = 0; r < 6; r++)
      for (int p = 0; p < SIDE_MAXP; p++) side_f[q][r][p] = (float) side[q][r][p];
  H2B_CUDA_TRY(cudaMemcpyToSymbol(c_side_f, side_f, sizeof(side_f)));
  return H2B_OK;
}

extern "C" int h2b_near_launch_kernels(const h2b_near_launch *L, cudaStream_t st) {
  if (L->q < 1 || L->q > 5) {
    h2b_set_error("regular quadrature order %u not supported (1..5)", L->q);
    return H2B_ERR_ARG;
  }
  switch (L->kk) {
    case KK_LSLP: return launch_kk<KK_LSLP>(L, st);
    case KK_LDLP: return launch_kk<KK_LDLP>(L, st);
    case KK_LBOTH: return launch_kk<KK_LBOTH>(L, st);
    case KK_HSLP: return launch_kk<KK_HSLP>(L, st);
    case KK_HDLP: return launch_kk<KK_HDLP>(L, st);
    case KK_LADLP: return launch_kk<KK_LADLP>(L, st);
    case KK_HADLP: return launch_kk<KK_HADLP>(L, st);
    case KK_HBOTH: return launch_kk<KK_HBOTH>(L, st);
    default: h2b_set_error("unknown kernel kind %d", L->kk); return H2B_ERR_ARG;
  }
}
