"""The greenhybrid fixture (tests/golden/green.npz, written by the reference's own
setup_h2matrix_aprx_greenhybrid_bem3d through gen_golden.c, on a sphere refined 8 times, scaled and
turned) against the host cluster trees: the reference's cluster tree equals ours on the fixture's
mesh, one rank per cluster in pre-order, every rank within the 12 (m l)^2 = 48 columns of A_t and
the rows of its cluster, and leaf bases and transfer matrices of exactly the sizes those ranks
give."""
import os

import numpy as np
import pytest

from h2lib_b200 import bem3d as hb

GOLD = os.path.join(os.path.dirname(__file__), "golden", "green.npz")
CASES = [("gsll", hb.BASIS_LINEAR_BEM3D), ("gscc", hb.BASIS_CONSTANT_BEM3D),
         ("gdll", hb.BASIS_LINEAR_BEM3D), ("gdcc", hb.BASIS_CONSTANT_BEM3D)]


@pytest.mark.parametrize("prefix,basis", CASES)
def test_green_fixture_matches_tree(prefix, basis):
    d = np.load(GOLD)
    gr = hb.Surface3d(d["green_x"], d["green_t"])
    tree = hb.build_tree(gr, basis, basis, 16, 1.4)
    rec, box, idx = tree.clusters(0)
    np.testing.assert_array_equal(rec, d[f"{prefix}_ctree"])
    np.testing.assert_array_equal(idx, d[f"{prefix}_idx"])
    np.testing.assert_array_equal(tree.block_records(), d[f"{prefix}_blocks"])
    size, sons = rec[:, 1].astype(np.int64), rec[:, 2].astype(np.int64)
    # father of every cluster (pre-order: a father precedes its sons)
    father = np.full(len(rec), -1)
    stack = []
    for i in range(len(rec)):
        while stack and stack[-1][1] == 0:
            stack.pop()
        if stack:
            father[i] = stack[-1][0]
            stack[-1][1] -= 1
        stack.append([i, int(sons[i])])
    for side in ("row", "col"):
        k = d[f"{prefix}_{side}_k"].astype(np.int64)
        assert k.shape == (len(rec),)
        assert np.all(k >= 1) and np.all(k <= 48) and np.all(k <= size)
        leaves = sons == 0
        assert d[f"{prefix}_{side}_V"].size == int(np.sum(size[leaves] * k[leaves]))
        nonroot = father >= 0
        assert d[f"{prefix}_{side}_E"].size == int(np.sum(k[nonroot] * k[father[nonroot]]))
        # a father's A_t has the pivot rows of its sons: its rank is at most their sum
        for i in np.nonzero(sons > 0)[0]:
            assert k[i] <= np.sum(k[father == i])


def test_green_fixture_leaf_bases_are_interpolatory():
    """Each leaf basis is the identity on its pivot rows (V (V[xi])^-1): k of its rows are unit
    vectors, one per column."""
    d = np.load(GOLD)
    for prefix, basis in CASES:
        rec = d[f"{prefix}_ctree"]
        k = d[f"{prefix}_row_k"].astype(np.int64)
        V = d[f"{prefix}_row_V"]
        o = 0
        for i in np.nonzero(rec[:, 2] == 0)[0]:
            n, r = int(rec[i, 1]), int(k[i])
            B = V[o:o + n * r].reshape(r, n).T   # column-major rows x rank
            o += n * r
            unit = [np.nonzero(np.isclose(B[:, j], 1.0, atol=1e-14) &
                               np.all(np.abs(np.delete(B, j, axis=1)) < 1e-14, axis=1))[0]
                    for j in range(r)]
            assert all(len(u) >= 1 for u in unit)
