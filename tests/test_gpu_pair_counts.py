"""Nearfield pair accounting on the B200: the triangle pairs the nearfield tiles evaluate
(h2b_h2matrix_pair_counts) and the distinct ones among them (h2b_h2matrix_unique_pairs), against
a count made here from the exported block tree.  Every inadmissible block evaluates all pairs of
triangles touching its row and column index sets (assemble_ll_near_bem3d,
Library/bem3d.c:3038); with the linear basis neighbouring blocks share triangles, so a pair can
be evaluated more than once.  Also the dense path's kernel timings (h2b_bem_timings)."""
import numpy as np
import pytest

from h2lib_b200 import bem3d as hb

pytestmark = pytest.mark.gpu
L, C = hb.BASIS_LINEAR_BEM3D, hb.BASIS_CONSTANT_BEM3D


def expected_counts(gr, tree, basis):
    """(evaluated, distinct) pair counts by vertices shared, from the block tree."""
    t = np.asarray(gr.t, dtype=np.int64).reshape(-1, 3)
    nt = t.shape[0]
    _, _, ridx = tree.clusters(0)
    _, _, cidx = tree.clusters(1)
    if basis == L:
        # triangles touching each vertex
        touch = [[] for _ in range(gr.vertices)]
        for i, tri in enumerate(t):
            for v in tri:
                touch[v].append(i)

        def tris(idx):
            return np.unique(np.concatenate([touch[v] for v in idx]))
    else:
        def tris(idx):
            return np.asarray(idx, dtype=np.int64)
    # shared vertices of every ordered pair
    shared = np.zeros((nt, nt), dtype=np.int8)
    for i in range(3):
        for j in range(3):
            shared += (t[:, i][:, None] == t[:, j][None, :])
    seen = np.zeros((nt, nt), dtype=bool)
    evaluated = np.zeros(4, dtype=np.int64)
    for ro, rs, co, cs, adm in tree.block_records():
        if adm:
            continue
        tr, sc = tris(ridx[ro:ro + rs]), tris(cidx[co:co + cs])
        evaluated += np.bincount(shared[np.ix_(tr, sc)].ravel(), minlength=4)
        seen[np.ix_(tr, sc)] = True
    distinct = np.bincount(shared[seen], minlength=4)
    return evaluated.tolist(), distinct.tolist()


@pytest.mark.parametrize("basis", [L, C])
def test_pair_counts_and_unique_pairs(basis):
    gr = hb.new_sphere_surface3d(8)
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, basis, basis)
    tree = hb.build_tree(gr, basis, basis, 16, 1.4)
    V = hb.H2Matrix(slp, tree, 3)
    V.assemble()
    ev, un = expected_counts(gr, tree, basis)
    keys = ("distant", "vertex", "edge", "identical")
    pc, up = V.pair_counts(), V.unique_pairs()
    assert [pc[k] for k in keys] == ev
    assert [up[k] for k in keys] == un
    if basis == C:
        # constant basis: the nearfield blocks do not overlap, every pair is evaluated once
        assert un == ev
        assert sum(un) == tree.near_entries
    else:
        assert sum(ev) > sum(un)
    # a second count gives the same numbers (the bitmap is cleared per call)
    assert V.unique_pairs() == up


def test_dense_assembly_timings():
    gr = hb.new_sphere_surface3d(8)
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, C, C)
    assert slp.timings() == {"near_distant": 0.0, "near_singular": 0.0}
    hb.assemble_bem3d_amatrix(slp)
    ms = slp.timings()
    assert ms["near_distant"] > 0.0 and ms["near_singular"] > 0.0
