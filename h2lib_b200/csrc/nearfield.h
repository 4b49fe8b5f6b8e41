/* Launch description of the nearfield quadrature kernels (nearfield.cu). */
#ifndef H2B200_NEARFIELD_H
#define H2B200_NEARFIELD_H

#include <cuda_runtime.h>
#include <stdint.h>

#include "h2b200_plan.h"

#ifdef __cplusplus
extern "C" {
#endif

/* kernel kinds */
#define H2B_KK_LSLP 0   /* Laplace single layer, real */
#define H2B_KK_LDLP 1   /* Laplace double layer, real */
#define H2B_KK_LBOTH 2  /* Laplace single and double layer together (two real outputs) */
#define H2B_KK_HSLP 3   /* Helmholtz single layer, complex */
#define H2B_KK_HDLP 4   /* Helmholtz double layer, complex */
#define H2B_KK_LADLP 5  /* Laplace adjoint double layer (row normal), real */
#define H2B_KK_HADLP 6  /* Helmholtz adjoint double layer (row normal), complex */
#define H2B_KK_HBOTH 7  /* Helmholtz single and double layer together (two complex outputs) */

typedef struct {
  int kk;
  int row_linear, col_linear;
  uint32_t q;                    /* regular order: distant pairs use q^4 points */
  const void *tri;               /* TriRec[triangles] */
  const void *refs;              /* TriRef pool */
  const h2b_tile *tiles;
  uint32_t ntiles;
  const h2b_sing *sing;          /* sorted by case */
  uint32_t nsing;
  uint32_t nvert;                /* vertex pairs at the start of sing (UINT32_MAX: not known) */
  double *out0, *out1;           /* out1: double-layer output of H2B_KK_LBOTH / H2B_KK_HBOTH */
  double kconst, k_re, k_imn;    /* 1/(4 pi); Re k; -Im k */
  double alpha_re, alpha_im;     /* identity coefficient of the double layer output */
  double mass[9];                /* linear-basis mass matrix on the reference triangle */
  const double *rule;            /* packed singular rules (device) */
  uint32_t rule_n[5], rule_off[5], rule_total;  /* [4]: merged common-vertex rule (or 0) */
  int vert_tensor;               /* 1: common-vertex rule in tensor form (groups in rule_n[1]) */
  int vert_merged;               /* 1: merged common-vertex rule in slot 4 (items in rule_n[4]) */
  int num_sms;
  int *err;                      /* device flag */
  cudaEvent_t ev_between;        /* optional: recorded between the distant and singular kernels */
  int fp32;                      /* 1: distant pairs in FP32 (q = 2 only); singular pairs stay FP64 */
} h2b_near_launch;

int h2b_near_upload_dist_rules(void);
/* Singular pairs of a tile list on the device (the pairs that share a vertex, with the vertex
 * permutation code of h2b_pair_code).  vt_off / vt_tri: the surface's vertex -> triangle lists
 * (CSR).  sing == NULL: add the number of pairs of each case c to cursor[c] (c = 1 vertex,
 * 2 edge, 3 identical).  Otherwise write the pairs of case c to sing[base[c] + cursor[c]++]
 * (cursor zeroed by the caller); the order inside a case is not fixed. */
int h2b_near_classify(const void *tri, const void *refs, const h2b_tile *tiles, uint32_t ntiles,
                      const uint32_t *vt_off, const uint32_t *vt_tri, uint32_t *cursor,
                      const uint32_t *base, h2b_sing *sing, cudaStream_t st);
int h2b_near_launch_kernels(const h2b_near_launch *L, cudaStream_t st);
/* Distinct triangle pairs of a tile list, by vertices shared (counts[0] distant, [1] common
 * vertex, [2] common edge, [3] identical), from a bitmap of nt^2 bits in device memory (freed
 * before the call returns; synchronises st). */
#define H2B_UNIQUE_PAIRS_MAX_TRIANGLES 131072u
int h2b_near_unique_pairs(const void *tri, const void *refs, const h2b_tile *tiles,
                          uint32_t ntiles, uint32_t nt, uint64_t counts[4], cudaStream_t st);

#ifdef __cplusplus
}
#endif

#endif
