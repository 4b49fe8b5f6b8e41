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
