"""Mixed precision on the B200: FP32 copies of the H2 matrix (products within FP32 rounding of
the FP64 product) and GMRES with FP32 Arnoldi steps and FP64 residuals, whose result meets the
FP64 stopping tolerance of the reference's solver (Library/krylovsolvers.c:183) on the FP64
operator."""
import numpy as np
import pytest

from h2lib_b200 import bem3d as hb

pytestmark = pytest.mark.gpu
L = hb.BASIS_LINEAR_BEM3D
Z = (1.2, 1.2, 1.2)


def relerr(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _dirichlet(split):
    gr = hb.new_sphere_surface3d(split)
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, L, L)
    dlp = hb.new_dlp_laplace_bem3d(gr, 2, 4, L, L, 0.5)
    tree = hb.build_tree(gr, L, L, 64, 1.4)
    V = hb.H2Matrix(slp, tree, 4).assemble()
    K = hb.H2Matrix(dlp, tree, 4).assemble()
    gD = hb.project_l2_harmonic(dlp, Z)
    b = hb.addeval_h2matrix_avector(1.0, K, gD, np.zeros(K.rows))
    return gr, slp, V, b


def test_single_copy_matvec():
    gr, slp, V, b = _dirichlet(16)
    V.make_single()
    x = np.random.default_rng(3).standard_normal(V.cols)
    y64 = hb.addeval_h2matrix_avector(1.0, V, x, np.zeros(V.rows))
    y32 = hb.addeval_h2matrix_avector_single(1.0, V, x, np.zeros(V.rows))
    assert 1e-10 < relerr(y32, y64) < 2e-6


def test_single_copy_dropped_on_reassembly():
    gr, slp, V, b = _dirichlet(8)
    V.make_single()
    V.assemble()
    x = np.ones(V.cols)
    with pytest.raises(hb.H2BError):
        hb.addeval_h2matrix_avector_single(1.0, V, x, np.zeros(V.rows))


def test_mixed_solve_meets_fp64_tolerance():
    gr, slp, V, b = _dirichlet(24)
    u64 = np.zeros(V.rows)
    it64 = hb.solve_gmres_h2matrix_avector(V, b, u64, 1e-8, 1000, 50)
    V.make_single()
    u = np.zeros(V.rows)
    it = hb.solve_gmres_mixed([V], [1.0], b, u, 1e-8, 1000, 50)
    assert hb.residual_norm([V], [1.0], b, u) <= 1e-8 * 1.0001
    assert relerr(u, u64) < 1e-6
    assert it <= 1.3 * it64 + 5
    err, nrm = hb.l2_error_harmonic(slp, Z, u)
    err64, _ = hb.l2_error_harmonic(slp, Z, u64)
    assert abs(err - err64) < 1e-6 * nrm


def test_batched_mixed_multi_rhs():
    ss = [hb.new_ellipsoid_surface3d(6, (1.0, 0.7, 1.6)), hb.new_sphere_surface3d(9)]
    gu, voff, toff = hb.union_surface3d(ss)
    slp = hb.new_slp_laplace_bem3d(gu, 2, 4, L, L)
    V = hb.H2Matrix(slp, hb.build_forest(gu, voff, toff, L, L, 32, 1.4), 4).assemble()
    V.make_single()
    n = gu.vertices
    rng = np.random.default_rng(11)
    B = rng.standard_normal((2, n))
    X = np.zeros((2, n))
    its = hb.solve_gmres_batch([V], [1.0], voff, B, X, 1e-8, 1000, 40, nrhs=2, mixed=True)
    assert its.shape == (2, 2)
    for r in range(2):
        for m in range(2):
            lo, hi = int(voff[m]), int(voff[m + 1])
            # FP64 residual of each system on its own block
            y = hb.addeval_h2matrix_avector(1.0, V, np.where(np.arange(n) >= lo, 1.0, 0.0) *
                                            np.where(np.arange(n) < hi, 1.0, 0.0) * X[r],
                                            np.zeros(n))
            res = np.linalg.norm(B[r, lo:hi] - y[lo:hi]) / np.linalg.norm(B[r, lo:hi])
            assert res <= 1.0001e-8


def test_fp32_quadrature_operator():
    """FP32 distant-pair quadrature: entries within FP32 accuracy of the FP64 ones, and the
    mixed solve on that operator meets the FP64 tolerance with a solution close to the FP64
    one and the same analytic error."""
    gr = hb.new_sphere_surface3d(16)
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, L, L)
    dlp = hb.new_dlp_laplace_bem3d(gr, 2, 4, L, L, 0.5)
    tree = hb.build_tree(gr, L, L, 64, 1.4)
    V64 = hb.H2Matrix(slp, tree, 4).assemble()
    K64 = hb.H2Matrix(dlp, tree, 4).assemble()
    V32 = hb.H2Matrix(slp, tree, 4).set_precision(True).assemble()
    K32 = hb.H2Matrix(dlp, tree, 4).set_precision(True).assemble()
    for a, b in ((V32, V64), (K32, K64)):
        n32, n64 = a.export(5), b.export(5)
        d = relerr(n32, n64)
        assert 1e-11 < d < 1e-6
        np.testing.assert_array_equal(a.export(4), b.export(4))  # coupling stays FP64
    gD = hb.project_l2_harmonic(dlp, Z)
    b64 = hb.addeval_h2matrix_avector(1.0, K64, gD, np.zeros(K64.rows))
    b32 = hb.addeval_h2matrix_avector(1.0, K32, gD, np.zeros(K32.rows))
    assert relerr(b32, b64) < 1e-6
    u64 = np.zeros(V64.rows)
    hb.solve_gmres_h2matrix_avector(V64, b64, u64, 1e-8, 1000, 50)
    V32.make_single()
    u = np.zeros(V32.rows)
    hb.solve_gmres_mixed([V32], [1.0], b32, u, 1e-8, 1000, 50)
    assert hb.residual_norm([V32], [1.0], b32, u) <= 1.0001e-8
    assert relerr(u, u64) < 1e-5
    e32, nrm = hb.l2_error_harmonic(slp, Z, u)
    e64, _ = hb.l2_error_harmonic(slp, Z, u64)
    assert abs(e32 - e64) < 1e-4 * nrm
