"""L2 projection of the harmonic Dirichlet datum on a union of surfaces with one source per
(right-hand side, surface) -- the batched solves' right-hand sides -- against the projection on
each surface alone (projectL2_bem3d_l_avector, Library/bem3d.c:9009), to 1e-12 relative.  The
surfaces differ in refinement, so the stacked mass system is badly scaled without its diagonal."""
import numpy as np
import pytest

from h2lib_b200 import bem3d as hb

pytestmark = pytest.mark.gpu
L = hb.BASIS_LINEAR_BEM3D


def test_multi_projection_equals_projection_per_surface():
    specs = [(4, (1.0, 1.0, 1.0)), (12, (0.6, 1.4, 0.9)), (24, (1.8, 0.7, 1.1))]
    surfs = [hb.new_ellipsoid_surface3d(s, ax) for s, ax in specs]
    gu, voff, toff = hb.union_surface3d(surfs)
    dlp = hb.new_dlp_laplace_bem3d(gu, 2, 4, L, L, 0.5)
    rng = np.random.default_rng(5)
    nrhs = 2
    zs = np.zeros((nrhs, len(surfs), 3))
    for m, (_, ax) in enumerate(specs):
        for r in range(nrhs):
            d = rng.standard_normal(3)
            zs[r, m] = 3.0 * max(ax) * d / np.linalg.norm(d)
    w = hb.project_l2_harmonic_multi(dlp, toff, zs)
    for m, gr in enumerate(surfs):
        op = hb.new_dlp_laplace_bem3d(gr, 2, 4, L, L, 0.5)
        for r in range(nrhs):
            ref = hb.project_l2_harmonic(op, zs[r, m])
            got = w[r, int(voff[m]):int(voff[m + 1])]
            assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
