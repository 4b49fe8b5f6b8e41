/* Flat nearfield plans shared by host_plan.c (builder) and nearfield.cu (consumer). */
#ifndef H2B200_PLAN_H
#define H2B200_PLAN_H

#include <stdint.h>

#include "h2b200_internal.h"

#ifdef __cplusplus
extern "C" {
#endif

#define H2B_TILE_MAX 64

/* Same layout as TriRef in device_common.cuh. */
typedef struct {
  uint32_t t;
  int16_t l[3];
  int16_t pad;
} h2b_triref;

/* One output tile: rows x cols entries (<= 64 x 64) written at out_off + r + c*ld (or, with
 * flags bit 0 = ntrans, at out_off + c + r*ld, conjugated). */
typedef struct {
  uint32_t tr_off, tr_len;  /* row triangles in the TriRef pool */
  uint32_t sc_off, sc_len;  /* column triangles */
  uint64_t out_off;
  uint32_t ld;
  uint16_t rows, cols;
  uint32_t flags;
  uint32_t pad;
} h2b_tile;

/* One singular triangle pair of a tile (tr, sc: absolute positions in the TriRef pool). */
typedef struct {
  uint32_t tile, tr, sc, code;
} h2b_sing;

typedef struct {
  h2b_tile *tiles;
  uint32_t ntiles;
  size_t ctiles;
  h2b_triref *refs;
  uint32_t nrefs;
  size_t crefs;
  h2b_sing *sing;
  uint32_t nsing;
  size_t csing;
  uint32_t case_start[5];   /* after finalize: singular pairs of case c in [case_start[c], [c+1]) */
  /* triangle lists already in `refs`, keyed by (index pointer, length, basis): the tiles of one
   * cluster share a single list (open addressing, capacity a power of two) */
  const uint32_t **lkey;
  uint32_t *lkn, *loff, *llen;
  size_t lcap, lcount;
  /* 1: leave the singular pairs to the device classification (h2b_near_classify) */
  int skip_sing;
} h2b_nearplan;

/* Vertex -> triangle adjacency plus scratch stamps for the plan builder. */
typedef struct {
  uint32_t nv, nt;
  uint32_t *off, *tri;
  const uint32_t *t;
  uint32_t *vstamp, *tstamp, *tpos;
  int32_t *vloc;
  uint32_t gen;
} h2b_adjacency;

int h2b_adjacency_build(uint32_t vertices, uint32_t triangles, const uint32_t *t,
                        h2b_adjacency *adj);
void h2b_adjacency_free(h2b_adjacency *adj);

void h2b_nearplan_init(h2b_nearplan *p);
void h2b_nearplan_free(h2b_nearplan *p);
int h2b_nearplan_add_block(h2b_nearplan *p, h2b_adjacency *adj, int row_basis, int col_basis,
                           const uint32_t *ridx, uint32_t rows, const uint32_t *cidx,
                           uint32_t cols, uint64_t out_off, uint32_t ld, int ntrans,
                           uint32_t tile);
int h2b_nearplan_finalize(h2b_nearplan *p);
/* Triangle list of an index set (linear: triangles touching the vertices, with local rows;
 * constant: the triangles themselves), appended to p->refs. */
int h2b_nearplan_add_reflist(h2b_nearplan *p, h2b_adjacency *adj, int linear,
                             const uint32_t *idx, uint32_t n, uint32_t *off, uint32_t *len);
uint32_t h2b_pair_code(const uint32_t *tv, const uint32_t *sv);

#ifdef __cplusplus
}
#endif

#endif
