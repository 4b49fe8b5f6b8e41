"""The H2Lib drop-in layer (h2lib_b200/shim) on the B200: one unchanged H2Lib program
(tests/h2lib_app/h2lib_app.c) runs once against H2Lib alone and once with the shim linked in front
of it, and the two runs must agree.

Compared (the tolerances of the other GPU parity tests):
  * the dense constant-basis single layer matrix (assemble_bem3d_amatrix), entrywise at 1e-12 with
    the row-scaled rule;
  * H2 products with the linear single and double layer operators (assemble_bem3d_h2matrix_* then
    addeval_h2matrix_avector), 1e-12 relative, and y += alpha A x accumulating;
  * H2Lib's own CPU product on the host H2 matrix the shim filled (bases, transfers, coupling and
    nearfield blocks written back into H2Lib's structures), 1e-12 relative;
  * solve_gmres_h2matrix_avector and solve_gmres_avector with addeval_h2matrix_avector: iteration
    count within one (the device GMRES applies the Householder reflectors in another order) and
    solution to 1e-6;
  * greenhybrid single and double layer products on a turned ellipsoid (1e-10), from the device
    and from H2Lib's CPU code on the bases, transfers and couplings with per-cluster ranks that
    the shim wrote back;
  * the Helmholtz build: a single-layer block through the bem->nearfield plugin point, the dense
    double layer matrix, the products and a GMRES solve of the single layer operator;
and the shim's counters show that the device did the work.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import rel_entry_err

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFOUT = os.path.join(ROOT, "oracle", "_ref")
DT = {"f8": np.float64, "c16": np.complex128}


def run_app(name):
    exe = os.path.join(REFOUT, name)
    if not os.path.exists(exe):
        pytest.skip(f"{name} not built (the H2Lib sources were absent at build time)")
    with tempfile.TemporaryDirectory() as tmp:
        res = subprocess.run([exe, tmp], capture_output=True, text=True, timeout=600)
        assert res.returncode == 0, res.stderr[-2000:]
        out = {}
        with open(os.path.join(tmp, "manifest.txt")) as fh:
            for line in fh:
                key, dt, n = line.split()
                out[key] = np.fromfile(os.path.join(tmp, key + ".bin"), dtype=DT[dt])
                assert out[key].size == int(n)
        return out


def relerr(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("field", ["real", "complex"])
def test_h2lib_program_through_the_shim(field):
    cpu = run_app(f"h2lib_app_{field}_cpu")
    gpu = run_app(f"h2lib_app_{field}_gpu")
    counts = gpu["shim_counts"]
    if field == "real":
        n = int(np.sqrt(cpu["dense_slp_cc"].size))
        a = gpu["dense_slp_cc"].reshape(n, n).T
        b = cpu["dense_slp_cc"].reshape(n, n).T
        assert rel_entry_err(a, b) < 1e-12
        assert counts[1] >= 1  # dense matrix on the device
        assert relerr(gpu["b"], cpu["b"]) < 1e-12
        assert abs(gpu["gmres_iter2"][0] - cpu["gmres_iter2"][0]) <= 1
        assert relerr(gpu["u2"], cpu["u2"]) < 1e-6
        # greenhybrid (setup_h2matrix_aprx_greenhybrid_bem3d): the device's products, and H2Lib's
        # own product on the per-cluster-rank bases and couplings the shim wrote back
        for op in ("Vg", "Kg"):
            assert relerr(gpu[f"y{op}"], cpu[f"y{op}"]) < 1e-10
            assert relerr(gpu[f"y{op}_acc"], cpu[f"y{op}_acc"]) < 1e-10
            assert relerr(gpu[f"y{op}_host"], cpu[f"y{op}"]) < 1e-10
    else:
        b = cpu["block_slp"].reshape(5, 7).T
        assert rel_entry_err(gpu["block_slp"].reshape(5, 7).T, b) < 1e-12
        assert counts[0] >= 1  # the nearfield callback ran on the device
        n = int(np.sqrt(cpu["dense_dlp_cc"].size))
        a = gpu["dense_dlp_cc"].reshape(n, n).T
        assert rel_entry_err(a, cpu["dense_dlp_cc"].reshape(n, n).T) < 1e-12
    for op in ("V", "K"):
        assert relerr(gpu[f"y{op}"], cpu[f"y{op}"]) < 1e-12
        assert relerr(gpu[f"y{op}_acc"], cpu[f"y{op}_acc"]) < 1e-12
        assert relerr(gpu[f"y{op}_host"], cpu[f"y{op}"]) < 1e-12
    assert abs(gpu["gmres_iter"][0] - cpu["gmres_iter"][0]) <= 1
    assert relerr(gpu["u"], cpu["u"]) < 1e-6
    assert counts[2] >= 4 and counts[3] >= 2  # bases and H2 matrices assembled on the device
    assert counts[4] >= 4 and counts[5] >= 1  # products and solves on the device
