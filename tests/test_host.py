"""Host-side parts of the library (no GPU): meshes, quadrature tables, cluster and block trees,
the exported C ABI.  Compared with golden vectors from the unmodified H2Lib reference."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from h2lib_b200 import bem3d as hb
from h2lib_b200._lib import LIBPATH, lib

L, C = hb.BASIS_LINEAR_BEM3D, hb.BASIS_CONSTANT_BEM3D


def test_library_exports_every_declared_symbol():
    """Every function declared in include/h2b200.h is exported by libh2b200.so."""
    src = open(os.path.join(ROOT, "include", "h2b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(h2b_[a-z0-9_]+)\s*\(", src))
    assert len(names) > 30
    dll = ctypes.CDLL(LIBPATH)
    missing = [n for n in sorted(names) if not hasattr(dll, n)]
    assert not missing, missing


def test_version_and_error_channel():
    assert b"sm_100a" in lib.h2b_version()
    nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
    assert lib.h2b_macro_mesh_size(7, 4, ctypes.byref(nv), ctypes.byref(nt)) < 0
    assert "unknown mesh kind" in hb.__dict__["check"].__globals__["last_error"]()


@pytest.mark.parametrize("split,key", [(4, "sphere4"), (8, "sphere8")])
def test_sphere_mesh_matches_reference(gold, split, key):
    g = gold(key)
    gr = hb.new_sphere_surface3d(split)
    assert gr.triangles == 8 * split * split
    np.testing.assert_array_equal(gr.t, g[f"{key}_t"])
    np.testing.assert_allclose(gr.x, g[f"{key}_x"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(gr.n, g[f"{key}_n"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(gr.g, g[f"{key}_g"], rtol=1e-13)
    np.testing.assert_allclose([gr.hmin, gr.hmax], g[f"{key}_h"], rtol=1e-13)


def test_config_meshes_match_reference(gold):
    g = gold("config2")
    gr = hb.new_sphere_surface3d(64)
    np.testing.assert_array_equal(gr.t, g["c2mesh_t"])
    np.testing.assert_allclose(gr.x, g["c2mesh_x"], rtol=0, atol=1e-15)
    c = gold("cube")
    cu = hb.new_cube_surface3d(4)
    np.testing.assert_array_equal(cu.t, c["cube4_t"])
    np.testing.assert_allclose(cu.x, c["cube4_x"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(cu.g, c["cube4_g"], rtol=1e-13)
    cu = hb.new_cube_surface3d(64)
    assert cu.triangles == 49152
    np.testing.assert_array_equal(cu.t, c["cube64_t"])
    np.testing.assert_allclose(cu.x, c["cube64_x"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("which,name", [(0, "dist"), (1, "vert"), (2, "edge"), (3, "id")])
def test_quadrature_tables_match_reference(gold, which, name):
    g = gold("quad")
    r = hb.quad_export(2, 4, C, C, which)
    np.testing.assert_allclose(r["x0"], g[f"{name}_x"][0], atol=1e-15)
    np.testing.assert_allclose(r["x1"], g[f"{name}_x"][1], atol=1e-15)
    np.testing.assert_allclose(r["y0"], g[f"{name}_y"][0], atol=1e-15)
    np.testing.assert_allclose(r["y1"], g[f"{name}_y"][1], atol=1e-15)
    np.testing.assert_allclose(r["w"][9], g[f"{name}_w"], rtol=1e-13, atol=1e-18)


def test_basis_weighted_tables_match_reference(gold):
    g = gold("quad")
    r = hb.quad_export(2, 4, L, L, 2)
    np.testing.assert_allclose(r["w"], g["edge_w_ll"], rtol=1e-12, atol=1e-18)
    s = hb.quad_export(2, 4, L, L, 4)
    np.testing.assert_allclose(s["x0"], g["single_x"], atol=1e-15)
    np.testing.assert_allclose(s["x1"], g["single_y"], atol=1e-15)
    np.testing.assert_allclose(s["w"], g["single_w_l"], rtol=1e-13)


@pytest.mark.parametrize("fixture,prefix,basis,clf", [
    ("h2small", "h2ll", L, 16), ("h2small", "h2cc", C, 16), ("config2", "c2", L, 64)])
def test_trees_match_reference(gold, fixture, prefix, basis, clf):
    g = gold(fixture)
    gr = hb.new_sphere_surface3d(64 if prefix == "c2" else 8)
    tr = hb.build_tree(gr, basis, basis, clf, 1.4)
    rec, box, idx = tr.clusters(0)
    np.testing.assert_array_equal(rec, g[f"{prefix}_ctree"])
    np.testing.assert_array_equal(idx, g[f"{prefix}_idx"])
    np.testing.assert_allclose(box, g[f"{prefix}_cbox"], rtol=0, atol=1e-15)
    np.testing.assert_array_equal(tr.block_records(), g[f"{prefix}_blocks"])
    blk = g[f"{prefix}_blocks"]
    near = blk[blk[:, 4] == 0]
    assert tr.near_entries == int(np.sum(near[:, 1].astype(np.int64) * near[:, 3]))


def test_tree_from_flat_arrays_roundtrip(gold):
    g = gold("h2small")
    rec, box, idx = g["h2ll_ctree"], g["h2ll_cbox"], g["h2ll_idx"]
    key = {(int(o), int(s)): i for i, (o, s, _) in enumerate(rec)}
    blk = g["h2ll_blocks"]
    brc = np.array([key[(int(b[0]), int(b[1]))] for b in blk], dtype=np.uint32)
    bcc = np.array([key[(int(b[2]), int(b[3]))] for b in blk], dtype=np.uint32)
    adm = np.ascontiguousarray(blk[:, 4].astype(np.uint8))
    off, size, sons = (np.ascontiguousarray(rec[:, i]) for i in range(3))
    box = np.ascontiguousarray(box)
    h = lib.h2b_tree_new_flat(rec.shape[0], off, size, sons, box, idx.shape[0], idx,
                              rec.shape[0], off, size, sons, box, idx.shape[0], idx,
                              blk.shape[0], brc, bcc, adm)
    assert h
    t = hb.Tree(h)
    np.testing.assert_array_equal(t.block_records(), blk)
    assert t.row_depth == t.col_depth


def test_tree_rejects_bad_input():
    gr = hb.new_sphere_surface3d(2)
    assert not lib.h2b_tree_new(gr.vertices, gr.x, gr.triangles, gr.t, L, L, 16, -1.0)
    assert "eta" in hb.__dict__["check"].__globals__["last_error"]()


def test_server_needs_a_device():
    """Without a CUDA device the server refuses to start (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from h2lib_b200.serve import Server
    with pytest.raises(H2BError):
        Server(slots=2)
from h2lib_b200._lib import H2BError  # noqa: E402
