/* C-ABI wrappers of the host-side trees (no GPU involved). */
#include <stdlib.h>
#include <string.h>

#include "h2b200_tree.h"

int h2b_ctree_build(uint32_t vertices, const double *x, uint32_t triangles, const uint32_t *t,
                    int basis, uint32_t clf, h2b_ctree *out);
int h2b_blist_build(const h2b_ctree *rt, const h2b_ctree *ct, double eta, h2b_blist *out);

static int
finish_tree(h2b_tree *tr)
{
  uint32_t i;
  uint64_t near = 0, adm = 0;
  for (i = 0; i < tr->blocks.n; i++) {
    if (tr->blocks.adm[i])
      adm++;
    else
      near += (uint64_t) tr->row.size[tr->blocks.rc[i]] * tr->col.size[tr->blocks.cc[i]];
  }
  tr->near_entries = near;
  tr->admissible = adm;
  return H2B_OK;
}

h2b_tree *
h2b_tree_new(uint32_t vertices, const double *x, uint32_t triangles, const uint32_t *t,
             int row_basis, int col_basis, uint32_t clf, double eta)
{
  h2b_tree *tr;
  if (!x || !t || vertices == 0 || triangles == 0) {
    h2b_set_error("h2b_tree_new: empty mesh");
    return NULL;
  }
  if ((row_basis != H2B_BASIS_CONSTANT && row_basis != H2B_BASIS_LINEAR)
      || (col_basis != H2B_BASIS_CONSTANT && col_basis != H2B_BASIS_LINEAR) || !(eta > 0.0)) {
    h2b_set_error("h2b_tree_new: invalid basis or eta");
    return NULL;
  }
  tr = (h2b_tree *) calloc(1, sizeof(h2b_tree));
  if (!tr) {
    h2b_set_error("h2b_tree_new: out of host memory");
    return NULL;
  }
  tr->row_basis = row_basis;
  tr->col_basis = col_basis;
  if (h2b_ctree_build(vertices, x, triangles, t, row_basis, clf, &tr->row) != H2B_OK
      || h2b_ctree_build(vertices, x, triangles, t, col_basis, clf, &tr->col) != H2B_OK
      || h2b_blist_build(&tr->row, &tr->col, eta, &tr->blocks) != H2B_OK) {
    h2b_tree_del(tr);
    return NULL;
  }
  finish_tree(tr);
  return tr;
}

/* Rebuild son/father/level links of a pre-order tree given only (off, size, sons). */
static int
link_tree(h2b_ctree *t)
{
  uint32_t *stack, sp = 0, i;
  stack = (uint32_t *) malloc(sizeof(uint32_t) * (t->n + 1));
  if (!stack)
    return H2B_ERR_NOMEM;
  t->depth = 0;
  for (i = 0; i < t->n; i++) {
    t->son0[i] = t->son1[i] = UINT32_MAX;
    t->father[i] = UINT32_MAX;
    t->level[i] = 0;
  }
  /* pre-order: the first son of i is i+1; the second son follows the first son's subtree */
  for (i = 0; i < t->n; i++) {
    if (i > 0) {
      /* pop completed fathers: a father is complete when all its sons have been seen */
      while (sp > 0) {
        uint32_t f = stack[sp - 1];
        uint32_t have = (t->son0[f] != UINT32_MAX) + (t->son1[f] != UINT32_MAX);
        if (have < t->sons[f])
          break;
        sp--;
      }
      if (sp == 0) {
        free(stack);
        return H2B_ERR_ARG;
      }
      {
        uint32_t f = stack[sp - 1];
        if (t->son0[f] == UINT32_MAX)
          t->son0[f] = i;
        else
          t->son1[f] = i;
        t->father[i] = f;
        t->level[i] = t->level[f] + 1;
      }
    }
    if (t->level[i] + 1 > t->depth)
      t->depth = t->level[i] + 1;
    if (t->sons[i] > 0) {
      if (t->sons[i] != 2) {
        free(stack);
        return H2B_ERR_ARG;
      }
      stack[sp++] = i;
    }
  }
  free(stack);
  return H2B_OK;
}

static int
copy_flat(h2b_ctree *t, uint32_t nc, const uint32_t *off, const uint32_t *size,
          const uint32_t *sons, const double *box, uint32_t n, const uint32_t *idx)
{
  uint32_t i;
  memset(t, 0, sizeof(*t));
  t->n = nc;
  t->nidx = n;
  t->off = malloc(sizeof(uint32_t) * nc);
  t->size = malloc(sizeof(uint32_t) * nc);
  t->sons = malloc(sizeof(uint32_t) * nc);
  t->son0 = malloc(sizeof(uint32_t) * nc);
  t->son1 = malloc(sizeof(uint32_t) * nc);
  t->father = malloc(sizeof(uint32_t) * nc);
  t->level = malloc(sizeof(uint32_t) * nc);
  t->bmin = malloc(sizeof(double) * 3 * nc);
  t->bmax = malloc(sizeof(double) * 3 * nc);
  t->idx = malloc(sizeof(uint32_t) * (n ? n : 1));
  if (!t->off || !t->size || !t->sons || !t->son0 || !t->son1 || !t->father || !t->level
      || !t->bmin || !t->bmax || !t->idx)
    return H2B_ERR_NOMEM;
  memcpy(t->off, off, sizeof(uint32_t) * nc);
  memcpy(t->size, size, sizeof(uint32_t) * nc);
  memcpy(t->sons, sons, sizeof(uint32_t) * nc);
  memcpy(t->idx, idx, sizeof(uint32_t) * n);
  for (i = 0; i < nc; i++) {
    memcpy(t->bmin + 3 * i, box + 6 * (size_t) i, sizeof(double) * 3);
    memcpy(t->bmax + 3 * i, box + 6 * (size_t) i + 3, sizeof(double) * 3);
    if ((uint64_t) off[i] + size[i] > n)
      return H2B_ERR_ARG;
  }
  return link_tree(t);
}

h2b_tree *
h2b_tree_new_flat(uint32_t row_clusters, const uint32_t *row_off, const uint32_t *row_size,
                  const uint32_t *row_sons, const double *row_box, uint32_t row_n,
                  const uint32_t *row_idx, uint32_t col_clusters, const uint32_t *col_off,
                  const uint32_t *col_size, const uint32_t *col_sons, const double *col_box,
                  uint32_t col_n, const uint32_t *col_idx, uint32_t blocks,
                  const uint32_t *block_rc, const uint32_t *block_cc, const uint8_t *block_adm)
{
  h2b_tree *tr;
  uint32_t i;
  if (!row_clusters || !col_clusters || !blocks || !row_off || !row_size || !row_sons
      || !row_box || !row_idx || !col_off || !col_size || !col_sons || !col_box || !col_idx
      || !block_rc || !block_cc || !block_adm) {
    h2b_set_error("h2b_tree_new_flat: empty tree or NULL array");
    return NULL;
  }
  tr = (h2b_tree *) calloc(1, sizeof(h2b_tree));
  if (!tr) {
    h2b_set_error("h2b_tree_new_flat: out of host memory");
    return NULL;
  }
  tr->row_basis = tr->col_basis = 0;
  if (copy_flat(&tr->row, row_clusters, row_off, row_size, row_sons, row_box, row_n, row_idx)
      || copy_flat(&tr->col, col_clusters, col_off, col_size, col_sons, col_box, col_n,
                   col_idx)) {
    h2b_tree_del(tr);
    h2b_set_error("h2b_tree_new_flat: malformed cluster tree (pre-order, 0 or 2 sons)");
    return NULL;
  }
  tr->blocks.n = blocks;
  tr->blocks.rc = malloc(sizeof(uint32_t) * blocks);
  tr->blocks.cc = malloc(sizeof(uint32_t) * blocks);
  tr->blocks.adm = malloc(blocks);
  if (!tr->blocks.rc || !tr->blocks.cc || !tr->blocks.adm) {
    h2b_tree_del(tr);
    h2b_set_error("h2b_tree_new_flat: out of host memory");
    return NULL;
  }
  for (i = 0; i < blocks; i++) {
    if (block_rc[i] >= row_clusters || block_cc[i] >= col_clusters) {
      h2b_tree_del(tr);
      h2b_set_error("h2b_tree_new_flat: block %u references a missing cluster", i);
      return NULL;
    }
    tr->blocks.rc[i] = block_rc[i];
    tr->blocks.cc[i] = block_cc[i];
    tr->blocks.adm[i] = block_adm[i] ? 1 : 0;
    if (!block_adm[i] && (tr->row.sons[block_rc[i]] || tr->col.sons[block_cc[i]])) {
      /* strict block trees only: nearfield blocks between leaves */
      h2b_tree_del(tr);
      h2b_set_error("h2b_tree_new_flat: inadmissible block %u is not a leaf-leaf block", i);
      return NULL;
    }
  }
  finish_tree(tr);
  return tr;
}

void
h2b_tree_del(h2b_tree *tree)
{
  if (!tree)
    return;
  h2b_ctree_free(&tree->row);
  h2b_ctree_free(&tree->col);
  h2b_blist_free(&tree->blocks);
  free(tree);
}

int
h2b_tree_info(const h2b_tree *tree, uint64_t info[8])
{
  if (!tree || !info) {
    h2b_set_error("h2b_tree_info: NULL argument");
    return H2B_ERR_ARG;
  }
  info[0] = tree->row.n;
  info[1] = tree->col.n;
  info[2] = tree->row.nidx;
  info[3] = tree->col.nidx;
  info[4] = tree->blocks.n;
  info[5] = tree->admissible;
  info[6] = tree->near_entries;
  info[7] = (uint64_t) tree->row.depth | ((uint64_t) tree->col.depth << 32);
  return H2B_OK;
}

int
h2b_tree_export_clusters(const h2b_tree *tree, int which, uint32_t *rec, double *box,
                         uint32_t *idx)
{
  const h2b_ctree *t;
  uint32_t i;
  if (!tree || (which != 0 && which != 1)) {
    h2b_set_error("h2b_tree_export_clusters: bad argument");
    return H2B_ERR_ARG;
  }
  t = which ? &tree->col : &tree->row;
  for (i = 0; i < t->n; i++) {
    if (rec) {
      rec[3 * i] = t->off[i];
      rec[3 * i + 1] = t->size[i];
      rec[3 * i + 2] = t->sons[i];
    }
    if (box) {
      memcpy(box + 6 * (size_t) i, t->bmin + 3 * (size_t) i, sizeof(double) * 3);
      memcpy(box + 6 * (size_t) i + 3, t->bmax + 3 * (size_t) i, sizeof(double) * 3);
    }
  }
  if (idx)
    memcpy(idx, t->idx, sizeof(uint32_t) * t->nidx);
  return H2B_OK;
}

int
h2b_tree_export_blocks(const h2b_tree *tree, uint32_t *rec)
{
  uint32_t i;
  if (!tree || !rec) {
    h2b_set_error("h2b_tree_export_blocks: NULL argument");
    return H2B_ERR_ARG;
  }
  for (i = 0; i < tree->blocks.n; i++) {
    uint32_t r = tree->blocks.rc[i], c = tree->blocks.cc[i];
    rec[5 * i] = tree->row.off[r];
    rec[5 * i + 1] = tree->row.size[r];
    rec[5 * i + 2] = tree->col.off[c];
    rec[5 * i + 3] = tree->col.size[c];
    rec[5 * i + 4] = tree->blocks.adm[i];
  }
  return H2B_OK;
}
