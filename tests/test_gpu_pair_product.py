"""The product of a double layer beside its single layer on one structure (K + c V, as in the
Brakhage-Werner and Laplace Dirichlet systems) reads the shared coupling matrices and row basis
once; its result must equal the two products taken apart (tolerance 1e-12 relative), for real and
complex operators."""
import numpy as np
import pytest

from h2lib_b200 import bem3d as hb

pytestmark = pytest.mark.gpu
L, C = hb.BASIS_LINEAR_BEM3D, hb.BASIS_CONSTANT_BEM3D


def separate_residual(ops, coefs, b, x):
    y = np.zeros_like(b)
    for op, c in zip(ops, coefs):
        y += c * hb.addeval_h2matrix_avector(1.0, op, x, np.zeros_like(b))
    return np.linalg.norm(b - y) / np.linalg.norm(b)


@pytest.mark.parametrize("pde", ["laplace", "helmholtz"])
def test_pair_product_equals_separate_products(pde):
    rng = np.random.default_rng(11)
    if pde == "laplace":
        gr = hb.new_sphere_surface3d(8)
        basis = L
        slp = hb.new_slp_laplace_bem3d(gr, 2, 4, basis, basis)
        dlp = hb.new_dlp_laplace_bem3d(gr, 2, 4, basis, basis, 0.5)
        coefs = [1.0, -0.7]
        m = 3
    else:
        gr = hb.new_cube_surface3d(6)
        basis = C
        k = 4.0
        slp = hb.new_slp_helmholtz_bem3d(k, gr, 2, 4, basis, basis)
        dlp = hb.new_dlp_helmholtz_bem3d(k, gr, 2, 4, basis, basis, 0.5)
        coefs = [1.0, -1j * k]
        m = 4
    tree = hb.build_tree(gr, basis, basis, 16, 1.4)
    V = hb.H2Matrix(slp, tree, m)
    K = hb.H2Matrix(dlp, tree, m, like=V)
    V.assemble()
    K.assemble()
    n = V.rows
    if pde == "laplace":
        x, b = rng.standard_normal(n), rng.standard_normal(n)
    else:
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = separate_residual([K, V], coefs, b, x)
    for _ in range(2):  # the fused product's work vectors are reused
        got = hb.residual_norm([K, V], coefs, b, x)
        assert abs(got - ref) <= 1e-12 * ref
    # the other order of the two terms (the single layer's plan first)
    got = hb.residual_norm([V, K], coefs[::-1], b, x)
    assert abs(got - ref) <= 1e-12 * ref


def test_pair_mixed_solve_meets_fp64_tolerance():
    """Brakhage-Werner system solved with FP32 Arnoldi products of the pair (FP32 copies of both
    matrices) and FP64 residuals: the FP64 residual meets eps and the solution is the FP64 one to
    FP32-level accuracy."""
    k = 2.0
    gr = hb.new_cube_surface3d(6)
    slp = hb.new_slp_helmholtz_bem3d(k, gr, 2, 4, C, C)
    dlp = hb.new_dlp_helmholtz_bem3d(k, gr, 2, 4, C, C, 0.5)
    tree = hb.build_tree(gr, C, C, 16, 1.4)
    V = hb.H2Matrix(slp, tree, 4)
    K = hb.H2Matrix(dlp, tree, 4, like=V)
    V.assemble()
    K.assemble()
    V.make_single()
    K.make_single()
    d = np.ones(3) / np.sqrt(3.0)
    b = hb.integrate_plane_wave(slp, k * d, coef=-1.0)
    coefs = [1.0, -1j * k]
    u64 = np.zeros(V.rows, dtype=np.complex128)
    it64 = hb.solve_gmres([K, V], coefs, b, u64, 1e-8, 1000, 80)
    u32 = np.zeros(V.rows, dtype=np.complex128)
    it32 = hb.solve_gmres_mixed([K, V], coefs, b, u32, 1e-8, 1000, 80)
    assert hb.residual_norm([K, V], coefs, b, u32) <= 1.01e-8
    assert abs(it32 - it64) <= 6
    assert np.linalg.norm(u32 - u64) / np.linalg.norm(u64) < 1e-6


@pytest.mark.parametrize("basis", [C, L])
def test_helmholtz_nearfield_pair_equals_separate(basis):
    """The fused single + double layer nearfield pass of Helmholtz (one sine and cosine per
    quadrature point for both kernels) against the two operators assembled apart, for a complex
    wavenumber too (relative to the largest entry, 1e-13)."""
    from h2lib_b200._lib import check, lib
    gr = hb.new_sphere_surface3d(8)
    tree = hb.build_tree(gr, basis, basis, 16, 1.4)
    for k in (3.0, 3.0 + 0.5j):
        slp = hb.new_slp_helmholtz_bem3d(k, gr, 2, 4, basis, basis)
        dlp = hb.new_dlp_helmholtz_bem3d(k, gr, 2, 4, basis, basis, 0.5)
        V = hb.H2Matrix(slp, tree, 3)
        K = hb.H2Matrix(dlp, tree, 3, like=V)
        check(lib.h2b_h2matrix_assemble_nearfield_pair(V.handle, K.handle), "nearfield pair")
        V2 = hb.H2Matrix(slp, tree, 3)
        K2 = hb.H2Matrix(dlp, tree, 3, like=V2)
        check(lib.h2b_h2matrix_assemble_nearfield(V2.handle), "nearfield V")
        check(lib.h2b_h2matrix_assemble_nearfield(K2.handle), "nearfield K")
        for a, b in ((V, V2), (K, K2)):
            na, nb = a.export(5), b.export(5)
            assert np.max(np.abs(na - nb)) <= 1e-13 * np.max(np.abs(nb))
