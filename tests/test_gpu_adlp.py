"""Adjoint double layer operator K' + alpha M on the B200 (new_adlp_laplace_bem3d,
Library/laplacebem3d.c:1180; new_adlp_helmholtz_bem3d, Library/helmholtzbem3d.c:1346) against the
reference's golden vectors: dense nearfield for the four basis pairs, a ragged block and its
transposed write, and the H2 matrix (row basis with normal derivatives, coupling, nearfield,
matvec).  Tolerances as for the other operators: 1e-12 entrywise / relative."""
import numpy as np
import pytest

from conftest import fortran, rel_entry_err
from h2lib_b200 import bem3d as hb

pytestmark = pytest.mark.gpu
L, C = hb.BASIS_LINEAR_BEM3D, hb.BASIS_CONSTANT_BEM3D
TOL = 1e-12


def relerr(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def s4():
    return hb.new_sphere_surface3d(4)


@pytest.fixture(scope="module")
def s8():
    return hb.new_sphere_surface3d(8)


@pytest.mark.parametrize("basis", ["cc", "ll", "cl", "lc"])
def test_adlp_dense(gold, s4, basis):
    g = gold("adlp")
    rb, cb = (L if basis[0] == "l" else C), (L if basis[1] == "l" else C)
    op = hb.new_adlp_laplace_bem3d(s4, 2, 4, rb, cb, 0.5)
    assert rel_entry_err(hb.nearfield(op, None, None), fortran(g[f"ad4{basis}"])) < TOL


def test_adlp_ragged_block_and_transpose(gold, s4):
    g, s4g = gold("adlp"), gold("sphere4")
    ridx, cidx = s4g["block_ridx"], s4g["block_cidx"]
    op = hb.new_adlp_laplace_bem3d(s4, 2, 4, L, L, 0.5)
    assert rel_entry_err(hb.nearfield(op, ridx, cidx), fortran(g["ad4ll_block"])) < TOL
    At = hb.nearfield(op, ridx, cidx, ntrans=True)
    assert rel_entry_err(At, fortran(g["ad4ll_block_trans"])) < TOL


@pytest.mark.parametrize("prefix,basis", [("adh2ll", L), ("adh2cc", C)])
def test_adlp_h2(gold, s8, prefix, basis):
    g = gold("adlp")
    op = hb.new_adlp_laplace_bem3d(s8, 2, 4, basis, basis, 0.5)
    tree = hb.build_tree(s8, basis, basis, 16, 1.4)
    rec, box, idx = tree.clusters(0)
    np.testing.assert_array_equal(rec, g[f"{prefix}_ctree"])
    np.testing.assert_array_equal(idx, g[f"{prefix}_idx"])
    A = hb.H2Matrix(op, tree, 3).assemble()
    assert relerr(A.export(0), g[f"{prefix}_row_V"]) < TOL
    assert relerr(A.export(4, 24), g[f"{prefix}_parts_S"]) < TOL
    assert relerr(A.export(5, 24), g[f"{prefix}_parts_N"]) < TOL
    y = hb.addeval_h2matrix_avector(1.0, A, g[f"{prefix}_x"], np.zeros(A.rows))
    assert relerr(y, g[f"{prefix}_y"]) < TOL
    # FP32 distant-pair quadrature: FP32 accuracy
    A.set_precision(True)
    A.assemble()
    y32 = hb.addeval_h2matrix_avector(1.0, A, g[f"{prefix}_x"], np.zeros(A.rows))
    assert relerr(y32, g[f"{prefix}_y"]) < 1e-6


def test_adlp_helmholtz(gold, s4, s8):
    g = gold("helm_adlp")
    for name, k in (("had4cc", 2.0), ("had4cc_damped", 2.0 + 0.5j)):
        op = hb.new_adlp_helmholtz_bem3d(k, s4, 2, 4, C, C, 0.5)
        assert rel_entry_err(hb.nearfield(op, None, None), fortran(g[name])) < TOL
    op = hb.new_adlp_helmholtz_bem3d(2.0, s8, 2, 4, C, C, 0.5)
    tree = hb.build_tree(s8, C, C, 16, 1.4)
    A = hb.H2Matrix(op, tree, 3).assemble()
    assert relerr(A.export(0), g["hadh2cc_row_V"].real) < TOL
    assert relerr(A.export(5, 24), g["hadh2cc_parts_N"]) < TOL
    x = np.ascontiguousarray(g["hadh2cc_x"])
    y = hb.addeval_h2matrix_avector(1.0, A, x, np.zeros(A.rows, dtype=np.complex128))
    assert relerr(y, g["hadh2cc_y"]) < TOL
