"""The launch-shape autotuner (h2b_h2matrix_autotune) on the B200: it picks a shape among the
candidates that fit an SM, the chosen shape gives the same products as the starting one (FP64 and
from the FP32 copies, up to rounding: only the grouping of atomic additions changes), the leaf
split changes the cluster bases by rounding only, the shape is cached for the next matrix of the
same size class, and the cache survives a save / clear / load round trip.  A structure shared
through h2b_h2matrix_new_like keeps its work items while it is shared."""
import os
import tempfile

import numpy as np
import pytest

from h2lib_b200 import bem3d as hb
from h2lib_b200._lib import check, lib

pytestmark = pytest.mark.gpu
L = hb.BASIS_LINEAR_BEM3D


def relerr(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _matrix(split, kind="slp"):
    gr = hb.new_sphere_surface3d(split)
    op = (hb.new_slp_laplace_bem3d(gr, 2, 4, L, L) if kind == "slp"
          else hb.new_dlp_laplace_bem3d(gr, 2, 4, L, L, 0.5))
    tree = hb.build_tree(gr, L, L, 64, 1.4)
    return gr, op, tree, hb.H2Matrix(op, tree, 4).assemble()


def test_autotune_keeps_the_product():
    check(lib.h2b_autotune_clear(), "clear")
    gr, slp, tree, V = _matrix(16)
    V.make_single()
    x = np.random.default_rng(7).standard_normal(V.cols)
    y64 = hb.addeval_h2matrix_avector(1.0, V, x, np.zeros(V.rows))
    y32 = hb.addeval_h2matrix_avector_single(1.0, V, x, np.zeros(V.rows))
    bases = [V.export(p) for p in range(4)]
    res = V.autotune(matvec=True, leaf=True)
    after = V.matvec_shape()
    assert res["matvec_ms"][0] > 0 and 0 < res["matvec_ms"][1] <= res["matvec_ms"][0]
    assert res["bases_ms"][0] > 0 and 0 < res["bases_ms"][1] <= res["bases_ms"][0]
    assert after["panel_kib"] in (12, 16, 24) and 1 <= after["consumer_warps"] <= 4
    assert 1 <= after["ctas_per_sm"] <= 8 and after["leaf_ctas"] in (1, 2, 4, 8)
    assert relerr(hb.addeval_h2matrix_avector(1.0, V, x, np.zeros(V.rows)), y64) < 1e-14
    assert relerr(hb.addeval_h2matrix_avector_single(1.0, V, x, np.zeros(V.rows)), y32) < 1e-14
    for p in range(4):  # leaf bases, transfers: every split sums the same terms
        assert relerr(V.export(p), bases[p]) < 1e-13
    # the next matrix of the class starts from the tuned shape
    _, dlp, _, K = _matrix(16, "dlp")
    assert K.matvec_shape() == after
    check(lib.h2b_autotune_clear(), "clear")


def test_autotune_cache_file_round_trip():
    check(lib.h2b_autotune_clear(), "clear")
    gr, slp, tree, V = _matrix(12)
    V.autotune()
    tuned = V.matvec_shape()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "tune.txt").encode()
        check(lib.h2b_autotune_save(path), "save")
        check(lib.h2b_autotune_clear(), "clear")
        check(lib.h2b_autotune_load(path), "load")
        with open(path, "w") as fh:
            fh.write("0 64 9 1 2 3\n")  # too few entries: rejected
        assert lib.h2b_autotune_load(path) < 0
    _, _, _, W = _matrix(12)
    assert W.matvec_shape() == tuned
    check(lib.h2b_autotune_clear(), "clear")


def test_autotune_shared_structure_keeps_panels():
    check(lib.h2b_autotune_clear(), "clear")
    gr, slp, tree, V = _matrix(12)
    dlp = hb.new_dlp_laplace_bem3d(gr, 2, 4, L, L, 0.5)
    K = hb.H2Matrix(dlp, tree, 4, like=V).assemble()
    x = np.random.default_rng(1).standard_normal(K.cols)
    yk = hb.addeval_h2matrix_avector(1.0, K, x, np.zeros(K.rows))
    yv = hb.addeval_h2matrix_avector(1.0, V, x, np.zeros(V.rows))
    pk = K.matvec_shape()["panel_kib"]
    K.autotune()
    V.autotune()  # the model matrix of a shared structure keeps its panels too
    assert K.matvec_shape()["panel_kib"] == pk and V.matvec_shape()["panel_kib"] == pk
    assert relerr(hb.addeval_h2matrix_avector(1.0, K, x, np.zeros(K.rows)), yk) < 1e-14
    assert relerr(hb.addeval_h2matrix_avector(1.0, V, x, np.zeros(V.rows)), yv) < 1e-14
    check(lib.h2b_autotune_clear(), "clear")


def test_shared_structure_is_fixed_while_shared():
    """The model matrix of h2b_h2matrix_new_like cannot rebuild the work items its sharers read
    (H2B_ERR_STATE) until the last sharer is gone; kernel knobs stay free."""
    gr, slp, tree, V = _matrix(12)
    dlp = hb.new_dlp_laplace_bem3d(gr, 2, 4, L, L, 0.5)
    K = hb.H2Matrix(dlp, tree, 4, like=V).assemble()
    pk = V.matvec_shape()["panel_kib"]
    other = 24 if pk != 24 else 12
    with pytest.raises(hb.H2BError):
        V.set_matvec_shape(panel_kib=other)
    with pytest.raises(hb.H2BError):
        K.set_matvec_shape(panel_kib=other)
    K.set_matvec_shape(ctas_per_sm=2, consumer_warps=2)
    x = np.random.default_rng(2).standard_normal(K.cols)
    y = hb.addeval_h2matrix_avector(1.0, K, x, np.zeros(K.rows))
    assert np.all(np.isfinite(y))
    del K
    V.set_matvec_shape(panel_kib=other)
    assert V.matvec_shape()["panel_kib"] == other
