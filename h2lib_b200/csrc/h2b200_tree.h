/* Host tree handle (cluster trees + block leaves) shared by the C and CUDA sources. */
#ifndef H2B200_TREE_H
#define H2B200_TREE_H

#include "h2b200_internal.h"

#ifdef __cplusplus
extern "C" {
#endif

struct h2b_tree {
  int row_basis, col_basis;  /* 0 when built from flat arrays (basis unknown) */
  h2b_ctree row, col;
  h2b_blist blocks;
  uint64_t near_entries, admissible;
};

#ifdef __cplusplus
}
#endif

#endif
