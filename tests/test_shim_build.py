"""The H2Lib drop-in layer builds and exports H2Lib's own entry points (no GPU needed): the shim
libraries define the names an H2Lib program binds, and the test program linked with the shim
binds them to the shim rather than to H2Lib."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "h2lib_b200", "shim")

COMMON = ["assemble_bem3d_amatrix", "assemble_bem3d_h2matrix",
          "assemble_bem3d_nearfield_h2matrix", "assemble_bem3d_farfield_h2matrix",
          "assemble_bem3d_h2matrix_row_clusterbasis", "assemble_bem3d_h2matrix_col_clusterbasis",
          "setup_h2matrix_aprx_inter_bem3d", "addeval_h2matrix_avector",
          "solve_gmres_h2matrix_avector", "solve_gmres_avector", "del_h2matrix", "del_surface3d",
          "h2b_shim_set_bypass", "h2b_shim_counts"]
NAMES = {
    "real": COMMON + ["new_slp_laplace_bem3d", "new_dlp_laplace_bem3d", "new_adlp_laplace_bem3d",
                      "del_laplace_bem3d"],
    "complex": COMMON + ["new_slp_helmholtz_bem3d", "new_dlp_helmholtz_bem3d",
                         "new_adlp_helmholtz_bem3d", "del_helmholtz_bem3d"],
}


def defined_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


@pytest.mark.parametrize("field", ["real", "complex"])
def test_shim_exports_h2lib_names(field):
    lib = os.path.join(SHIM, f"libh2b_h2lib_{field}.so")
    if not os.path.exists(lib):
        pytest.skip("shim not built (the H2Lib sources were absent at build time)")
    missing = [n for n in NAMES[field] if n not in defined_symbols(lib)]
    assert not missing, missing


def test_program_binds_h2lib_names_to_the_shim():
    exe = os.path.join(ROOT, "oracle", "_ref", "h2lib_app_real_gpu")
    if not os.path.exists(exe):
        pytest.skip("shim test program not built")
    needed = subprocess.run(["readelf", "-d", exe], capture_output=True, text=True,
                            check=True).stdout
    libs = [line.split("[")[1].rstrip("]") for line in needed.splitlines() if "(NEEDED)" in line]
    # the shim precedes H2Lib in the search order, so its definitions win
    assert libs.index("libh2b_h2lib_real.so") < libs.index("libh2ref_real.so")
