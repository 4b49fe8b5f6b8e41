"""Cluster and block trees built on the device (h2b_tree_new_device) equal the host builder's
(h2b_tree_new, index for index with H2Lib's build_adaptive_cluster / build_strict_block, as
tests/test_host.py checks against the reference's own trees): every cluster's offset, size, sons
and bounding box, the index permutation, and the block leaves with their admissibility, for both
bases, several leaf sizes and admissibility parameters, and an index range longer than the
device's shared-memory partition stage (cube, 49152 triangles, constant basis)."""
import time

import numpy as np
import pytest

from h2lib_b200 import bem3d as hb

pytestmark = pytest.mark.gpu
L, C = hb.BASIS_LINEAR_BEM3D, hb.BASIS_CONSTANT_BEM3D


def same_trees(a, b):
    for which in (0, 1):
        ra, ba, ia = a.clusters(which)
        rb, bb, ib = b.clusters(which)
        np.testing.assert_array_equal(ra, rb)
        np.testing.assert_array_equal(ba, bb)
        np.testing.assert_array_equal(ia, ib)
    np.testing.assert_array_equal(a.block_records(), b.block_records())
    assert (a.blocks, a.admissible, a.near_entries) == (b.blocks, b.admissible, b.near_entries)


@pytest.mark.parametrize("mesh,split,rb,cb,clf,eta", [
    ("sphere", 4, L, L, 16, 1.4),
    ("sphere", 8, C, C, 32, 1.0),
    ("sphere", 16, L, C, 24, 1.4),
    ("sphere", 64, L, L, 64, 1.4),
    ("cube", 16, C, L, 8, 0.7),
    ("cube", 64, C, C, 64, 1.4),
])
def test_device_trees_equal_host_trees(mesh, split, rb, cb, clf, eta):
    gr = hb.new_sphere_surface3d(split) if mesh == "sphere" else hb.new_cube_surface3d(split)
    host = hb.build_tree(gr, rb, cb, clf, eta)
    dev = hb.build_tree(gr, rb, cb, clf, eta, device=True)
    same_trees(host, dev)


def test_device_trees_on_an_ellipsoid_and_in_an_h2_matrix():
    gr = hb.new_ellipsoid_surface3d(12, (1.7, 0.6, 1.1))
    host = hb.build_tree(gr, L, L, 32, 1.4)
    dev = hb.build_tree(gr, L, L, 32, 1.4, device=True)
    same_trees(host, dev)
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, L, L)
    x = np.random.default_rng(4).standard_normal(gr.vertices)
    y0 = hb.addeval_h2matrix_avector(1.0, hb.H2Matrix(slp, host, 4).assemble(), x,
                                     np.zeros(gr.vertices))
    y1 = hb.addeval_h2matrix_avector(1.0, hb.H2Matrix(slp, dev, 4).assemble(), x,
                                     np.zeros(gr.vertices))
    assert np.linalg.norm(y1 - y0) <= 1e-14 * np.linalg.norm(y0)


def test_device_tree_rejects_bad_input():
    gr = hb.new_sphere_surface3d(4)
    t = gr.t.copy()
    t[5] = gr.vertices + 3
    from h2lib_b200._lib import lib
    assert not lib.h2b_tree_new_device(gr.vertices, gr.x, gr.triangles, t, L, L, 16, 1.4)
    assert not lib.h2b_tree_new_device(gr.vertices, gr.x, gr.triangles, gr.t, L, L, 0, 1.4)
