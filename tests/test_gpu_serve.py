"""Solve server on the B200: requests admitted while others run give the same results as alone
(and as the direct API), meet the FP64 tolerance, and complete under a budget that admits only
one request at a time."""
import numpy as np
import pytest

from h2lib_b200 import bem3d as hb
from h2lib_b200.serve import HELMHOLTZ, LAPLACE, Server

pytestmark = pytest.mark.gpu
L, Cb = hb.BASIS_LINEAR_BEM3D, hb.BASIS_CONSTANT_BEM3D
Z = (1.2, 1.2, 1.2)
D = np.ones(3) / np.sqrt(3.0)


def relerr(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def direct_laplace(gr, z):
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, L, L)
    dlp = hb.new_dlp_laplace_bem3d(gr, 2, 4, L, L, 0.5)
    tree = hb.build_tree(gr, L, L, 64, 1.4)
    V = hb.H2Matrix(slp, tree, 4).assemble()
    K = hb.H2Matrix(dlp, tree, 4).assemble()
    b = hb.addeval_h2matrix_avector(1.0, K, hb.project_l2_harmonic(dlp, z), np.zeros(K.rows))
    u = np.zeros(V.rows)
    it = hb.solve_gmres_h2matrix_avector(V, b, u, 1e-8, 1000, 50)
    return u, it


def direct_helmholtz(gr, k):
    slp = hb.new_slp_helmholtz_bem3d(k, gr, 2, 4, Cb, Cb)
    dlp = hb.new_dlp_helmholtz_bem3d(k, gr, 2, 4, Cb, Cb, 0.5)
    tree = hb.build_tree(gr, Cb, Cb, 64, 1.4)
    V = hb.H2Matrix(slp, tree, 5).assemble()
    K = hb.H2Matrix(dlp, tree, 5).assemble()
    b = hb.integrate_plane_wave(slp, k * D, coef=-1.0)
    u = np.zeros(V.rows, dtype=np.complex128)
    it = hb.solve_gmres([K, V], [1.0, -1j * k], b, u, 1e-8, 1000, 80)
    return u, it


def test_same_alone_and_in_the_mix():
    ga = hb.new_sphere_surface3d(12)
    gb = hb.new_cube_surface3d(6)
    gc = hb.new_ellipsoid_surface3d(10, (1.5, 0.8, 1.0))
    gd = hb.new_sphere_surface3d(16)
    srv = Server(slots=4)
    try:
        a_alone, ra = srv.wait(srv.submit(ga, LAPLACE, Z))
        ids = [srv.submit(gb, HELMHOLTZ, D, k=3.0), srv.submit(gc, LAPLACE, (0.0, 0.0, 3.5)),
               srv.submit(ga, LAPLACE, Z), srv.submit(gd, LAPLACE, (2.0, -1.0, 0.5)),
               srv.submit(gb, HELMHOLTZ, D, k=3.0)]
        out = [srv.wait(i) for i in ids]
    finally:
        srv.close()
    a_mix, rm = out[2]
    assert ra["status"] == 0 and rm["status"] == 0
    assert abs(int(ra["iterations"]) - int(rm["iterations"])) <= 1
    assert relerr(a_mix, a_alone) < 1e-6
    for sol, res in out:
        assert res["rel_residual"] <= 1.05e-8
        assert res["t_submit"] <= res["t_start"] <= res["t_done"]
    # the two identical Helmholtz requests agree, and both match the direct API
    assert relerr(out[0][0], out[4][0]) < 1e-6
    u, it = direct_helmholtz(gb, 3.0)
    assert relerr(out[0][0], u) < 1e-6
    u, it = direct_laplace(ga, Z)
    assert relerr(a_alone, u) < 1e-6 and abs(it - int(ra["iterations"])) <= 1


def test_mixed_precision_requests_meet_tolerance():
    srv = Server(slots=2)
    try:
        g = hb.new_ellipsoid_surface3d(14, (1.0, 1.3, 0.7))
        sol, res = srv.wait(srv.submit(g, LAPLACE, (0.5, 3.0, 0.0), mixed=True))
        gh = hb.new_cube_surface3d(5)
        solh, resh = srv.wait(srv.submit(gh, HELMHOLTZ, D, k=2.0, mixed=True))
    finally:
        srv.close()
    assert res["rel_residual"] <= 1.0001e-8 and resh["rel_residual"] <= 1.0001e-8
    # mixed requests also assemble the distant pairs in FP32 (entries ~1e-7 from FP64)
    u, _ = direct_laplace(g, (0.5, 3.0, 0.0))
    assert relerr(sol, u) < 1e-5


def test_tiny_budget_serialises():
    srv = Server(slots=3, hbm_budget=1)
    try:
        gs = [hb.new_sphere_surface3d(s) for s in (6, 8, 10)]
        ids = [srv.submit(g, LAPLACE, Z) for g in gs]
        res = [srv.wait(i)[1] for i in ids]
    finally:
        srv.close()
    # every request is larger than the budget, so each ran alone: no overlap in time
    spans = sorted((r["t_start"], r["t_done"]) for r in res)
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0 - 1e-6
    assert all(r["rel_residual"] <= 1.05e-8 for r in res)


def test_batched_requests_match_alone():
    """Laplace requests queued behind a running one are solved as one batch (forest H2 matrix,
    batched GMRES): each result matches the request solved alone through the direct API."""
    gh = hb.new_cube_surface3d(6)
    gs = [hb.new_sphere_surface3d(10), hb.new_ellipsoid_surface3d(8, (1.4, 0.9, 1.1)),
          hb.new_cube_surface3d(5)]
    zs = [(1.2, 1.2, 1.2), (0.0, 3.0, 0.5), (2.5, -2.5, 1.0)]
    srv = Server(slots=1)
    try:
        first = srv.submit(gh, HELMHOLTZ, D, k=2.0)  # keeps the only worker busy meanwhile
        ids = [srv.submit(g, LAPLACE, z) for g, z in zip(gs, zs)]
        srv.wait(first)
        out = [srv.wait(i) for i in ids]
    finally:
        srv.close()
    starts = {r["t_start"] for _, r in out}
    assert len(starts) == 1  # one admission took all three
    for (sol, res), g, z in zip(out, gs, zs):
        u, it = direct_laplace(g, z)
        assert res["status"] == 0 and res["rel_residual"] <= 1.05e-8
        assert abs(int(res["iterations"]) - it) <= 1
        assert relerr(sol, u) < 1e-6
