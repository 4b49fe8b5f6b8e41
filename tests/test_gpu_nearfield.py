"""Nearfield quadrature on the B200 through the C ABI, against the oracle and the reference's
golden vectors.  Tolerance: |a - b| <= 1e-12 * max(|b_ij|, max_j |b_ij|) per entry (FP64 path)."""
import numpy as np
import pytest

from conftest import fortran, rel_entry_err
from h2lib_b200 import bem3d as hb
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
L, C = hb.BASIS_LINEAR_BEM3D, hb.BASIS_CONSTANT_BEM3D
TOL = 1e-12


def omesh(gr):
    return orc.Mesh(gr.x, gr.t, gr.n, gr.g)


@pytest.fixture(scope="module")
def s4():
    return hb.new_sphere_surface3d(4)


@pytest.fixture(scope="module")
def s8():
    return hb.new_sphere_surface3d(8)


def test_config1_dense_slp_dlp(gold, s8):
    """Config 1: 512 x 512 cc SLP (and DLP, alpha = 1/2) on the sphere refined x8, q = 2 / 4."""
    g = gold("sphere8")
    slp = hb.new_slp_laplace_bem3d(s8, 2, 4, C, C)
    G = hb.assemble_bem3d_amatrix(slp)
    assert rel_entry_err(G, fortran(g["c1_slp"])) < TOL
    dlp = hb.new_dlp_laplace_bem3d(s8, 2, 4, C, C, 0.5)
    K = hb.assemble_bem3d_amatrix(dlp)
    ncol = g["c1_dlp"].shape[0]
    assert rel_entry_err(K[:, :ncol], fortran(g["c1_dlp"])) < TOL
    ref = orc.nearfield(omesh(s8), orc.LAPLACE, orc.DLP, C, C, alpha=0.5)
    assert rel_entry_err(K, ref) < TOL


@pytest.mark.parametrize("basis", ["cc", "ll", "cl", "lc"])
@pytest.mark.parametrize("layer", ["slp", "dlp"])
def test_sphere4_all_bases(gold, s4, basis, layer):
    g = gold("sphere4")
    rb, cb = (L if basis[0] == "l" else C), (L if basis[1] == "l" else C)
    if layer == "slp":
        bem = hb.new_slp_laplace_bem3d(s4, 2, 4, rb, cb)
    else:
        bem = hb.new_dlp_laplace_bem3d(s4, 2, 4, rb, cb, 0.5)
    A = hb.nearfield(bem, None, None)
    assert rel_entry_err(A, fortran(g[f"s4{basis}_{layer}"])) < TOL


def test_ll_ragged_block_and_transpose(gold, s4):
    g = gold("sphere4")
    ridx, cidx = g["block_ridx"], g["block_cidx"]
    slp = hb.new_slp_laplace_bem3d(s4, 2, 4, L, L)
    assert rel_entry_err(hb.nearfield(slp, ridx, cidx), fortran(g["s4ll_slp_block"])) < TOL
    dlp = hb.new_dlp_laplace_bem3d(s4, 2, 4, L, L, 0.5)
    assert rel_entry_err(hb.nearfield(dlp, ridx, cidx), fortran(g["s4ll_dlp_block"])) < TOL
    At = hb.nearfield(dlp, ridx, cidx, ntrans=True)
    assert rel_entry_err(At, fortran(g["s4ll_dlp_block_trans"])) < TOL


@pytest.mark.parametrize("name,layer,k,alpha", [
    ("hs4cc_slp", "slp", 2.0, 0.0), ("hs4cc_dlp", "dlp", 2.0, 0.5),
    ("hs4cc_slp_damped", "slp", 2.0 + 0.5j, 0.0)])
def test_helmholtz_cc(gold, s4, name, layer, k, alpha):
    if layer == "slp":
        bem = hb.new_slp_helmholtz_bem3d(k, s4, 2, 4, C, C)
    else:
        bem = hb.new_dlp_helmholtz_bem3d(k, s4, 2, 4, C, C, alpha)
    A = hb.nearfield(bem, None, None)
    assert rel_entry_err(A, fortran(gold("helm_sphere4")[name])) < TOL


def test_helmholtz_ll_against_oracle(s4):
    bem = hb.new_dlp_helmholtz_bem3d(3.0, s4, 2, 4, L, L, 0.5)
    A = hb.nearfield(bem, None, None)
    ref = orc.nearfield(omesh(s4), orc.HELMHOLTZ, orc.DLP, L, L, k=3.0, alpha=0.5)
    assert rel_entry_err(A, ref) < TOL


def test_larger_ll_blocks_against_oracle():
    """Sphere refined x16 (2048 triangles): several 64 x 64 tiles, interior vertices."""
    gr = hb.new_sphere_surface3d(16)
    rng = np.random.default_rng(7)
    ridx = rng.permutation(gr.vertices)[:150].astype(np.uint32)
    cidx = rng.permutation(gr.vertices)[:130].astype(np.uint32)
    for layer in ("slp", "dlp"):
        bem = (hb.new_slp_laplace_bem3d(gr, 2, 4, L, L) if layer == "slp"
               else hb.new_dlp_laplace_bem3d(gr, 2, 4, L, L, -0.5))
        A = hb.nearfield(bem, ridx, cidx)
        ref = orc.nearfield(omesh(gr), orc.LAPLACE, orc.SLP if layer == "slp" else orc.DLP, L, L,
                            ridx, cidx, alpha=0.0 if layer == "slp" else -0.5)
        assert rel_entry_err(A, ref) < TOL


def test_device_output_matches_host_output(s8):
    torch = pytest.importorskip("torch")
    slp = hb.new_slp_laplace_bem3d(s8, 2, 4, C, C)
    host = hb.assemble_bem3d_amatrix(slp)
    dev = torch.zeros((512, 512), dtype=torch.float64, device="cuda")  # row-major = transposed
    hb.assemble_bem3d_amatrix(slp, dev)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy().T, host)


def test_leading_dimension_padding(s4):
    """ld > rows: entries outside the block are left untouched (host output)."""
    slp = hb.new_slp_laplace_bem3d(s4, 2, 4, C, C)
    out = np.full((140, 128), 7.0, order="F")
    hb.nearfield(slp, None, None, out=out)
    assert np.all(out[128:] == 7.0)
    ref = hb.nearfield(slp, None, None)
    assert np.array_equal(out[:128], ref)


def test_invalid_arguments_fail_loudly(s4):
    slp = hb.new_slp_laplace_bem3d(s4, 2, 4, C, C)
    with pytest.raises(hb.H2BError):
        hb.nearfield(slp, np.array([0, 0], dtype=np.uint32), None)   # repeated index
    with pytest.raises(hb.H2BError):
        hb.nearfield(slp, np.array([4096], dtype=np.uint32), None)   # out of range


@pytest.mark.parametrize("q,q2", [(1, 2), (3, 3), (4, 5)])
def test_other_quadrature_orders_against_oracle(s4, q, q2):
    """Orders other than the default 2 / 4: the generic distant kernel, the full common-vertex
    rule (no tensor or merged form) and the reduced edge / identical rules for other q2."""
    for rb, cb in ((L, L), (C, C), (L, C)):
        for layer in ("slp", "dlp"):
            bem = (hb.new_slp_laplace_bem3d(s4, q, q2, rb, cb) if layer == "slp"
                   else hb.new_dlp_laplace_bem3d(s4, q, q2, rb, cb, 0.5))
            A = hb.nearfield(bem, None, None)
            ref = orc.nearfield(omesh(s4), orc.LAPLACE, orc.SLP if layer == "slp" else orc.DLP,
                                rb, cb, q=q, q2=q2, alpha=0.0 if layer == "slp" else 0.5)
            assert rel_entry_err(A, ref) < TOL, (q, q2, rb, cb, layer)
    bem = hb.new_dlp_helmholtz_bem3d(2.0 + 0.5j, s4, q, q2, C, C, 0.5)
    A = hb.nearfield(bem, None, None)
    ref = orc.nearfield(omesh(s4), orc.HELMHOLTZ, orc.DLP, C, C, q=q, q2=q2, k=2.0 + 0.5j,
                        alpha=0.5)
    assert rel_entry_err(A, ref) < TOL
