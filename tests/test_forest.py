"""Forest trees (one cluster/block tree per surface, concatenated): every surface's part of the
forest equals the tree of that surface built alone, shifted by the surface's offsets."""
import numpy as np
import pytest

from h2lib_b200 import bem3d as hb

L, Cb = hb.BASIS_LINEAR_BEM3D, hb.BASIS_CONSTANT_BEM3D


def _surfaces():
    return [hb.new_ellipsoid_surface3d(4, (1.0, 0.7, 1.6)), hb.new_sphere_surface3d(6),
            hb.new_ellipsoid_surface3d(5, (0.5, 2.0, 1.0))]


@pytest.mark.parametrize("basis", [L, Cb])
def test_forest_matches_single_trees(basis):
    surfs = _surfaces()
    gu, voff, toff = hb.union_surface3d(surfs)
    forest = hb.build_forest(gu, voff, toff, basis, basis, 16, 1.4)
    rec_f, box_f, idx_f = forest.clusters(0)
    blocks_f = forest.block_records()
    c0 = b0 = 0
    for m, gr in enumerate(surfs):
        one = hb.build_tree(gr, basis, basis, 16, 1.4)
        rec, box, idx = one.clusters(0)
        ioff = int(voff[m]) if basis == L else int(toff[m])
        n = rec.shape[0]
        part = rec_f[c0:c0 + n].astype(np.int64)
        np.testing.assert_array_equal(part[:, 0] - ioff, rec[:, 0])   # offsets in the index set
        np.testing.assert_array_equal(part[:, 1:], rec[:, 1:])
        np.testing.assert_array_equal(box_f[c0:c0 + n], box)
        np.testing.assert_array_equal(idx_f[ioff:ioff + idx.size].astype(np.int64) - ioff, idx)
        nb = one.blocks
        bf = blocks_f[b0:b0 + nb].astype(np.int64)
        bf[:, 0] -= ioff
        bf[:, 2] -= ioff
        np.testing.assert_array_equal(bf, one.block_records())
        c0 += n
        b0 += nb
    assert c0 == forest.row_clusters and b0 == forest.blocks
    assert forest.near_entries == sum(hb.build_tree(g, basis, basis, 16, 1.4).near_entries
                                      for g in surfs)


def test_forest_rejects_crossing_triangles():
    surfs = _surfaces()[:2]
    gu, voff, toff = hb.union_surface3d(surfs)
    bad = voff.copy()
    bad[1] -= 1   # the first surface's last vertex now belongs to the second
    with pytest.raises(hb.H2BError):
        hb.build_forest(gu, bad, toff, L, L, 16, 1.4)


def test_forest_many_surfaces_mixed_bases():
    """More surfaces than host threads, unequal sizes and constant rows beside linear columns:
    the surfaces are built on several threads and appended in order, so each part of the forest
    (both cluster trees and the blocks) is the tree of its surface alone, shifted."""
    rng = np.random.default_rng(3)
    surfs = [hb.new_ellipsoid_surface3d(int(s), rng.uniform(0.5, 2.0, 3))
             for s in rng.integers(2, 9, 70)]
    gu, voff, toff = hb.union_surface3d(surfs)
    forest = hb.build_forest(gu, voff, toff, Cb, L, 8, 1.2)
    blocks_f = forest.block_records().astype(np.int64)
    for which, offs in ((0, toff), (1, voff)):
        rec_f, box_f, idx_f = forest.clusters(which)
        c0 = 0
        for m, gr in enumerate(surfs):
            rec, box, idx = hb.build_tree(gr, Cb, L, 8, 1.2).clusters(which)
            ioff, n = int(offs[m]), rec.shape[0]
            part = rec_f[c0:c0 + n].astype(np.int64)
            np.testing.assert_array_equal(part[:, 0] - ioff, rec[:, 0])
            np.testing.assert_array_equal(part[:, 1:], rec[:, 1:])
            np.testing.assert_array_equal(box_f[c0:c0 + n], box)
            np.testing.assert_array_equal(idx_f[ioff:ioff + idx.size].astype(np.int64) - ioff,
                                          idx)
            c0 += n
        assert c0 == (forest.row_clusters if which == 0 else forest.col_clusters)
    b0 = 0
    for m, gr in enumerate(surfs):
        one = hb.build_tree(gr, Cb, L, 8, 1.2)
        bf = blocks_f[b0:b0 + one.blocks].copy()
        bf[:, 0] -= int(toff[m])
        bf[:, 2] -= int(voff[m])
        np.testing.assert_array_equal(bf, one.block_records())
        b0 += one.blocks
    assert b0 == forest.blocks


def test_forest_rejects_zero_leaf_size():
    gu, voff, toff = hb.union_surface3d(_surfaces()[:2])
    with pytest.raises(hb.H2BError, match="leaf size"):
        hb.build_forest(gu, voff, toff, L, L, 0, 1.4)
