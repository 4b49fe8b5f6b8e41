/* Host-side nearfield plans: cut the requested blocks into output tiles of at most 64 x 64
 * entries, list the triangles each tile touches, and find the singular (vertex-sharing) triangle
 * pairs, bucketed by Sauter-Schwab case.  The device kernels consume the flat arrays.
 *
 * Semantics follow the reference's nearfield callbacks:
 *   constant basis  assemble_cc_near_bem3d   Library/bem3d.c:1151 — one triangle pair per entry;
 *   linear basis    assemble_ll_near_bem3d   Library/bem3d.c:3038 — entry (i, j) sums every pair
 *                   (t, s) with vertex i in t and vertex j in s, using the weight of the local
 *                   basis functions of i in t and j in s; cl / lc mix the two.
 * Classification and vertex permutation restate select_quadrature_singquad2d
 * (Library/singquad2d.c:549): the shared vertices come first, in the row triangle's order.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "h2b200_plan.h"

#define GROW(arr, n, cap, extra, type)                                                   \
  do {                                                                                 \
    if ((n) + (extra) > (cap)) {                                                       \
      size_t nc_ = ((size_t) (n) + (extra)) * 2 + 64;                                  \
      type *p_ = (type *) realloc((arr), sizeof(type) * nc_);                          \
      if (!p_) return H2B_ERR_NOMEM;                                                   \
      (arr) = p_;                                                                      \
      (cap) = nc_;                                                                     \
    }                                                                                  \
  } while (0)

int
h2b_adjacency_build(uint32_t vertices, uint32_t triangles, const uint32_t *t, h2b_adjacency *adj)
{
  uint32_t i, k;
  memset(adj, 0, sizeof(*adj));
  adj->nv = vertices;
  adj->nt = triangles;
  adj->off = (uint32_t *) calloc((size_t) vertices + 1, sizeof(uint32_t));
  adj->tri = (uint32_t *) malloc(sizeof(uint32_t) * 3 * (size_t) (triangles ? triangles : 1));
  adj->vstamp = (uint32_t *) calloc(vertices ? vertices : 1, sizeof(uint32_t));
  adj->vloc = (int32_t *) calloc(vertices ? vertices : 1, sizeof(int32_t));
  adj->tstamp = (uint32_t *) calloc(triangles ? triangles : 1, sizeof(uint32_t));
  adj->tpos = (uint32_t *) calloc(triangles ? triangles : 1, sizeof(uint32_t));
  if (!adj->off || !adj->tri || !adj->vstamp || !adj->vloc || !adj->tstamp || !adj->tpos) {
    h2b_adjacency_free(adj);
    return H2B_ERR_NOMEM;
  }
  for (i = 0; i < triangles; i++)
    for (k = 0; k < 3; k++)
      adj->off[t[3 * (size_t) i + k] + 1]++;
  for (i = 0; i < vertices; i++)
    adj->off[i + 1] += adj->off[i];
  {
    uint32_t *fill = (uint32_t *) malloc(sizeof(uint32_t) * (vertices ? vertices : 1));
    if (!fill) {
      h2b_adjacency_free(adj);
      return H2B_ERR_NOMEM;
    }
    memcpy(fill, adj->off, sizeof(uint32_t) * vertices);
    for (i = 0; i < triangles; i++)
      for (k = 0; k < 3; k++) {
        uint32_t v = t[3 * (size_t) i + k];
        adj->tri[fill[v]++] = i;
      }
    free(fill);
  }
  adj->t = t;
  adj->gen = 0;
  return H2B_OK;
}

void
h2b_adjacency_free(h2b_adjacency *adj)
{
  free(adj->off); free(adj->tri); free(adj->vstamp); free(adj->vloc); free(adj->tstamp);
  free(adj->tpos);
  memset(adj, 0, sizeof(*adj));
}

void
h2b_nearplan_init(h2b_nearplan *p)
{
  memset(p, 0, sizeof(*p));
}

void
h2b_nearplan_free(h2b_nearplan *p)
{
  free(p->tiles); free(p->refs); free(p->sing);
  free((void *) p->lkey); free(p->lkn); free(p->loff); free(p->llen);
  memset(p, 0, sizeof(*p));
}

static size_t
list_slot(const h2b_nearplan *p, const uint32_t *idx, uint32_t kn)
{
  size_t h = ((size_t) (uintptr_t) idx >> 2) * 0x9E3779B97F4A7C15ull ^ (size_t) kn * 0xC2B2AE3D27D4EB4Full;
  size_t m = p->lcap - 1, i = (h >> 17) & m;
  while (p->lkey[i] && !(p->lkey[i] == idx && p->lkn[i] == kn))
    i = (i + 1) & m;
  return i;
}

/* Grow the list table to keep it at most half full. */
static int
list_reserve(h2b_nearplan *p)
{
  size_t i, oc = p->lcap;
  const uint32_t **ok = p->lkey;
  uint32_t *okn = p->lkn, *ooff = p->loff, *olen = p->llen;
  if (2 * (p->lcount + 1) <= p->lcap)
    return H2B_OK;
  p->lcap = oc ? 2 * oc : 1024;
  p->lkey = (const uint32_t **) calloc(p->lcap, sizeof(*p->lkey));
  p->lkn = (uint32_t *) calloc(p->lcap, sizeof(uint32_t));
  p->loff = (uint32_t *) calloc(p->lcap, sizeof(uint32_t));
  p->llen = (uint32_t *) calloc(p->lcap, sizeof(uint32_t));
  if (!p->lkey || !p->lkn || !p->loff || !p->llen)
    return H2B_ERR_NOMEM;
  for (i = 0; i < oc; i++)
    if (ok[i]) {
      size_t j = list_slot(p, ok[i], okn[i]);
      p->lkey[j] = ok[i];
      p->lkn[j] = okn[i];
      p->loff[j] = ooff[i];
      p->llen[j] = olen[i];
    }
  free((void *) ok); free(okn); free(ooff); free(olen);
  return H2B_OK;
}

static uint32_t
next_gen(h2b_adjacency *adj)
{
  if (++adj->gen == 0) {   /* wrapped: reset stamps */
    memset(adj->vstamp, 0, sizeof(uint32_t) * adj->nv);
    memset(adj->tstamp, 0, sizeof(uint32_t) * adj->nt);
    adj->gen = 1;
  }
  return adj->gen;
}

/* Append the triangle list of an index range; returns its offset in p->refs. */
static int
add_reflist(h2b_nearplan *p, h2b_adjacency *adj, int linear, const uint32_t *idx, uint32_t n,
            uint32_t *off, uint32_t *len)
{
  uint32_t i, k;
  *off = p->nrefs;
  if (!linear) {
    GROW(p->refs, p->nrefs, p->crefs, n, h2b_triref);
    for (i = 0; i < n; i++) {
      h2b_triref *r = &p->refs[p->nrefs++];
      r->t = idx[i];
      r->l[0] = r->l[1] = r->l[2] = (int16_t) i;
      r->pad = 0;
    }
  }
  else {
    uint32_t gv = next_gen(adj), gt;
    for (i = 0; i < n; i++) {
      adj->vstamp[idx[i]] = gv;
      adj->vloc[idx[i]] = (int32_t) i;
    }
    gt = next_gen(adj);
    /* vertex stamps of the first generation stay valid: compare against gv below */
    for (i = 0; i < n; i++) {
      uint32_t v = idx[i], a;
      for (a = adj->off[v]; a < adj->off[v + 1]; a++) {
        uint32_t tt = adj->tri[a];
        h2b_triref *r;
        if (adj->tstamp[tt] == gt)
          continue;
        adj->tstamp[tt] = gt;
        GROW(p->refs, p->nrefs, p->crefs, 1, h2b_triref);
        r = &p->refs[p->nrefs++];
        r->t = tt;
        for (k = 0; k < 3; k++) {
          uint32_t w = adj->t[3 * (size_t) tt + k];
          r->l[k] = (adj->vstamp[w] == gv) ? (int16_t) adj->vloc[w] : (int16_t) -1;
        }
        r->pad = 0;
      }
    }
  }
  *len = p->nrefs - *off;
  return H2B_OK;
}

int
h2b_nearplan_add_reflist(h2b_nearplan *p, h2b_adjacency *adj, int linear, const uint32_t *idx,
                         uint32_t n, uint32_t *off, uint32_t *len)
{
  return add_reflist(p, adj, linear, idx, n, off, len);
}

/* Vertex permutation of a pair: returns the number of shared vertices and the packed code
 * case | tp0<<2 | tp1<<4 | tp2<<6 | sp0<<8 | sp1<<10 | sp2<<12. */
uint32_t
h2b_pair_code(const uint32_t *tv, const uint32_t *sv)
{
  uint32_t p = 0, i, j, q, tp[3] = {0, 1, 2}, sp[3] = {0, 1, 2};
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++)
      p += (tv[i] == sv[j]);
  if (p == 1 || p == 2) {
    uint32_t c = 0;
    for (i = 0; i < 3; i++)
      for (j = 0; j < 3; j++)
        if (tv[i] == sv[j]) {
          tp[c] = i;
          sp[c] = j;
          c++;
          break;
        }
    q = c;
    for (i = 0; i < 3; i++) {
      for (j = 0; j < q && tv[i] != tv[tp[j]]; j++)
        ;
      if (j == q)
        tp[q++] = i;
    }
    q = c;
    for (i = 0; i < 3; i++) {
      for (j = 0; j < q && sv[i] != sv[sp[j]]; j++)
        ;
      if (j == q)
        sp[q++] = i;
    }
  }
  if (p > 3)
    p = 3;
  return p | (tp[0] << 2) | (tp[1] << 4) | (tp[2] << 6) | (sp[0] << 8) | (sp[1] << 10)
         | (sp[2] << 12);
}

/* add_reflist, reusing the list of an index range seen before. */
static int
cached_reflist(h2b_nearplan *p, h2b_adjacency *adj, int linear, const uint32_t *idx, uint32_t n,
               uint32_t *off, uint32_t *len)
{
  const uint32_t kn = (n << 1) | (linear ? 1u : 0u);
  size_t i;
  int rc;
  if ((rc = list_reserve(p)) != H2B_OK)
    return rc;
  i = list_slot(p, idx, kn);
  if (p->lkey[i]) {
    *off = p->loff[i];
    *len = p->llen[i];
    return H2B_OK;
  }
  if ((rc = add_reflist(p, adj, linear, idx, n, off, len)) != H2B_OK)
    return rc;
  p->lkey[i] = idx;
  p->lkn[i] = kn;
  p->loff[i] = *off;
  p->llen[i] = *len;
  p->lcount++;
  return H2B_OK;
}

static int
add_tile(h2b_nearplan *p, h2b_adjacency *adj, int row_linear, int col_linear,
         const uint32_t *ridx, uint32_t rows, const uint32_t *cidx, uint32_t cols,
         uint64_t out_off, uint32_t ld, int ntrans, uint32_t reuse_tr_off, uint32_t reuse_tr_len)
{
  h2b_tile *tl;
  uint32_t tr_off, tr_len, sc_off, sc_len, js, i, gt;
  int rc;

  if (reuse_tr_len != UINT32_MAX) {
    tr_off = reuse_tr_off;
    tr_len = reuse_tr_len;
  }
  else if ((rc = cached_reflist(p, adj, row_linear, ridx, rows, &tr_off, &tr_len)) != H2B_OK)
    return rc;
  if ((rc = cached_reflist(p, adj, col_linear, cidx, cols, &sc_off, &sc_len)) != H2B_OK)
    return rc;

  GROW(p->tiles, p->ntiles, p->ctiles, 1, h2b_tile);
  tl = &p->tiles[p->ntiles];
  tl->tr_off = tr_off;
  tl->tr_len = tr_len;
  tl->sc_off = sc_off;
  tl->sc_len = sc_len;
  tl->out_off = out_off;
  tl->ld = ld;
  tl->rows = (uint16_t) rows;
  tl->cols = (uint16_t) cols;
  tl->flags = ntrans ? 1u : 0u;
  tl->pad = 0;

  if (p->skip_sing) {
    p->ntiles++;
    return H2B_OK;
  }
  /* singular pairs: row triangles sharing a vertex with a column triangle */
  gt = next_gen(adj);
  for (i = 0; i < tr_len; i++) {
    uint32_t tt = p->refs[tr_off + i].t;
    adj->tstamp[tt] = gt;
    adj->tpos[tt] = tr_off + i;
  }
  for (js = 0; js < sc_len; js++) {
    uint32_t ss = p->refs[sc_off + js].t, found[24], nf = 0, k, a, f;
    const uint32_t *sv = adj->t + 3 * (size_t) ss;
    for (k = 0; k < 3; k++)
      for (a = adj->off[sv[k]]; a < adj->off[sv[k] + 1]; a++) {
        uint32_t tt = adj->tri[a];
        if (adj->tstamp[tt] != gt)
          continue;
        for (f = 0; f < nf && found[f] != tt; f++)
          ;
        if (f < nf || nf == 24)
          continue;
        found[nf++] = tt;
      }
    for (f = 0; f < nf; f++) {
      h2b_sing *sg;
      uint32_t code = h2b_pair_code(adj->t + 3 * (size_t) found[f], sv);
      GROW(p->sing, p->nsing, p->csing, 1, h2b_sing);
      sg = &p->sing[p->nsing++];
      sg->tile = p->ntiles;
      sg->tr = adj->tpos[found[f]];
      sg->sc = sc_off + js;
      sg->code = code;
    }
  }
  p->ntiles++;
  return H2B_OK;
}

int
h2b_nearplan_add_block(h2b_nearplan *p, h2b_adjacency *adj, int row_basis, int col_basis,
                       const uint32_t *ridx, uint32_t rows, const uint32_t *cidx, uint32_t cols,
                       uint64_t out_off, uint32_t ld, int ntrans, uint32_t tile)
{
  int rl = (row_basis == H2B_BASIS_LINEAR), cl = (col_basis == H2B_BASIS_LINEAR);
  uint32_t r0, c0;
  if (tile == 0 || tile > H2B_TILE_MAX)
    tile = H2B_TILE_MAX;
  for (c0 = 0; c0 < cols; c0 += tile) {
    uint32_t nc = cols - c0 < tile ? cols - c0 : tile;
    for (r0 = 0; r0 < rows; r0 += tile) {
      uint32_t nr = rows - r0 < tile ? rows - r0 : tile;
      uint64_t off = ntrans ? out_off + c0 + (uint64_t) r0 * ld : out_off + r0 + (uint64_t) c0 * ld;
      int rc = add_tile(p, adj, rl, cl, ridx + r0, nr, cidx + c0, nc, off, ld, ntrans, 0,
                        UINT32_MAX);
      if (rc != H2B_OK)
        return rc;
    }
  }
  return H2B_OK;
}

/* Stable counting sort of the singular pairs by case (1 vertex, 2 edge, 3 identical), so that
 * warps meet runs of equal trip counts. */
int
h2b_nearplan_finalize(h2b_nearplan *p)
{
  uint32_t cnt[4] = {0, 0, 0, 0}, start[4], i;
  h2b_sing *tmp;
  if (p->nsing == 0)
    return H2B_OK;
  tmp = (h2b_sing *) malloc(sizeof(h2b_sing) * p->nsing);
  if (!tmp)
    return H2B_ERR_NOMEM;
  for (i = 0; i < p->nsing; i++)
    cnt[p->sing[i].code & 3]++;
  start[0] = 0;
  for (i = 1; i < 4; i++)
    start[i] = start[i - 1] + cnt[i - 1];
  for (i = 0; i < 4; i++)
    p->case_start[i] = start[i];
  p->case_start[4] = p->nsing;
  for (i = 0; i < p->nsing; i++)
    tmp[start[p->sing[i].code & 3]++] = p->sing[i];
  free(p->sing);
  p->sing = tmp;
  p->csing = p->nsing;
  return H2B_OK;
}
