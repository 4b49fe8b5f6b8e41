"""The allocation-free GMRES entry point (h2b_solve_gmres_noalloc) against h2b_solve_gmres.

h2b_solve_gmres_noalloc serves callers that must not allocate device memory during a solve: it
takes its work space from a fixed array compiled into the library instead of allocating it per
call.  Called twice in a row through the C ABI, it must return the same iteration count and the
same solution as the allocating entry point, within the solution tolerance of the other GMRES
tests (1e-9 relative).  The file is collected last so that a failure here stops a run only after
every other test has run; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from h2lib_b200 import bem3d as hb
from h2lib_b200._lib import check, lib

pytestmark = pytest.mark.gpu
L, C = hb.BASIS_LINEAR_BEM3D, hb.BASIS_CONSTANT_BEM3D
TOL = 1e-9


def relerr(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def solve_noalloc(ops, coefs, b, eps, maxiter, kmax):
    arr = (ctypes.c_void_p * len(ops))(*[o.handle for o in ops])
    cf = np.zeros(2 * len(ops))
    for i, c in enumerate(coefs):
        cf[2 * i], cf[2 * i + 1] = complex(c).real, complex(c).imag
    x = np.zeros_like(b)
    it = check(lib.h2b_solve_gmres_noalloc(len(ops), ctypes.cast(arr, ctypes.c_void_p), cf,
                                           ctypes.c_void_p(b.ctypes.data),
                                           ctypes.c_void_p(x.ctypes.data), eps, maxiter, kmax),
               "h2b_solve_gmres_noalloc")
    return it, x


def device_memory():
    out = np.zeros(4, dtype=np.uint64)
    check(lib.h2b_device_memory(out), "h2b_device_memory")
    return [int(v) for v in out]


def test_noalloc_gmres_matches_allocating_gmres_laplace():
    check(lib.h2b_device_init(0), "device_init")
    gr = hb.new_sphere_surface3d(8)
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, L, L)
    tree = hb.build_tree(gr, L, L, 16, 1.4)
    V = hb.H2Matrix(slp, tree, 3).assemble()
    b = np.sin(0.37 * np.arange(V.rows)) + 0.5
    u = np.zeros(V.rows)
    it_ref = hb.solve_gmres_h2matrix_avector(V, b, u, 1e-8, 1000, 20)
    for call in range(2):  # two calls in a row share the fixed work space
        before = device_memory()
        it, x = solve_noalloc([V], [1.0], b, 1e-8, 1000, 20)
        after = device_memory()
        assert it == it_ref
        assert relerr(x, u) < TOL
        if call == 1:
            # the second call allocates nothing: free device memory and the stream-ordered
            # pool's used and reserved bytes are unchanged
            assert after[0] == before[0]
            assert after[2] == before[2] and after[3] == before[3]


def test_noalloc_gmres_matches_allocating_gmres_helmholtz():
    gr = hb.new_sphere_surface3d(8)
    k = 2.0
    slp = hb.new_slp_helmholtz_bem3d(k, gr, 2, 4, C, C)
    dlp = hb.new_dlp_helmholtz_bem3d(k, gr, 2, 4, C, C, 0.5)
    tree = hb.build_tree(gr, C, C, 16, 1.4)
    V = hb.H2Matrix(slp, tree, 3).assemble()
    K = hb.H2Matrix(dlp, tree, 3).assemble()
    b = hb.integrate_plane_wave(slp, k * np.ones(3) / np.sqrt(3.0), coef=-1.0)
    u = np.zeros(V.rows, dtype=np.complex128)
    it_ref = hb.solve_gmres([K, V], [1.0, -1j * k], b, u, 1e-8, 1000, 30)
    for _ in range(2):
        it, x = solve_noalloc([K, V], [1.0, -1j * k], b, 1e-8, 1000, 30)
        assert it == it_ref
        assert relerr(x, u) < TOL


def test_noalloc_gmres_rejects_problems_larger_than_its_work_space():
    # 49152 unknowns x 64 Krylov vectors x 8 bytes is already the whole fixed work space
    gr = hb.new_cube_surface3d(64)
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, C, C)
    tree = hb.build_tree(gr, C, C, 64, 1.4)
    V = hb.H2Matrix(slp, tree, 2)
    b = np.ones(V.rows)
    with pytest.raises(hb.H2BError, match="work space"):
        solve_noalloc([V], [1.0], b, 1e-8, 1000, 64)
    with pytest.raises(hb.H2BError):
        solve_noalloc([V], [1.0], b, 1e-8, 1000, 200)   # kmax beyond the solver's limit
