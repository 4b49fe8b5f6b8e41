"""Forest H2 matrices and batched GMRES on the B200: an H2 matrix on the forest of several
surfaces is block diagonal with exactly the H2 matrices of the single surfaces as blocks, and
the batched solver gives every system the result of its own solve."""
import numpy as np
import pytest

from h2lib_b200 import bem3d as hb

pytestmark = pytest.mark.gpu
L = hb.BASIS_LINEAR_BEM3D


def relerr(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _surfaces():
    return [hb.new_ellipsoid_surface3d(6, (1.0, 0.7, 1.6)), hb.new_sphere_surface3d(8),
            hb.new_ellipsoid_surface3d(5, (0.5, 2.0, 1.0))]


def test_forest_matvec_and_batched_solve():
    ss = _surfaces()
    gu, voff, toff = hb.union_surface3d(ss)
    slp_u = hb.new_slp_laplace_bem3d(gu, 2, 4, L, L)
    forest = hb.build_forest(gu, voff, toff, L, L, 32, 1.4)
    Vf = hb.H2Matrix(slp_u, forest, 4).assemble()
    rng = np.random.default_rng(7)
    x = rng.standard_normal(gu.vertices)
    yf = hb.addeval_h2matrix_avector(1.0, Vf, x, np.zeros(gu.vertices))
    singles = []
    for m, g in enumerate(ss):
        slp = hb.new_slp_laplace_bem3d(g, 2, 4, L, L)
        V = hb.H2Matrix(slp, hb.build_tree(g, L, L, 32, 1.4), 4).assemble()
        lo, hi = int(voff[m]), int(voff[m + 1])
        ys = hb.addeval_h2matrix_avector(1.0, V, x[lo:hi].copy(), np.zeros(g.vertices))
        assert relerr(yf[lo:hi], ys) < 1e-13
        singles.append(V)
    b = rng.standard_normal(gu.vertices)
    u = np.zeros(gu.vertices)
    its = hb.solve_gmres_batch([Vf], [1.0], voff, b, u, 1e-8, 1000, 50)[0]
    for m, V in enumerate(singles):
        lo, hi = int(voff[m]), int(voff[m + 1])
        us = np.zeros(hi - lo)
        it = hb.solve_gmres_h2matrix_avector(V, b[lo:hi].copy(), us, 1e-8, 1000, 50)
        assert abs(int(its[m]) - it) <= 1
        assert relerr(u[lo:hi], us) < 1e-7
        assert hb.residual_norm([V], [1.0], b[lo:hi].copy(), u[lo:hi].copy()) < 1.05e-8


def test_batched_solve_rejects_bad_segments():
    g = hb.new_sphere_surface3d(4)
    slp = hb.new_slp_laplace_bem3d(g, 2, 4, L, L)
    V = hb.H2Matrix(slp, hb.build_tree(g, L, L, 32, 1.4), 4).assemble()
    b = np.ones(g.vertices)
    u = np.zeros(g.vertices)
    with pytest.raises(hb.H2BError):
        hb.solve_gmres_batch([V], [1.0], [0, g.vertices - 1], b, u, 1e-8, 100, 20)
    with pytest.raises(hb.H2BError):
        hb.solve_gmres_batch([V], [1.0], [0, 10, 10, g.vertices], b, u, 1e-8, 100, 20)
