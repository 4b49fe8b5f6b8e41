"""Regenerate the golden fixtures in this directory from the unmodified H2Lib reference.

Builds oracle/_ref/libh2ref_{real,complex}.so from the reference sources (oracle/Makefile), compiles
gen_golden.c against them, runs the requested sections and packs each section's raw arrays into
``<section>.npz``.  Needs the reference tree (REF, default /root/reference); the tests themselves only
read the committed .npz files.

    python tests/golden/make_golden.py [section ...]

Sections: quad sphere8 sphere4 h2small config2 cube adlp green helm_sphere4 helm_h2small config3
config3_k8 helm_gmres helm_adlp helm_point
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("REF", "/root/reference")
REFOUT = os.path.join(ROOT, "oracle", "_ref")

REAL_SECTIONS = ["quad", "sphere8", "sphere4", "h2small", "config2", "cube", "adlp", "green"]
COMPLEX_SECTIONS = ["helm_sphere4", "helm_h2small", "config3", "config3_k8", "helm_gmres",
                    "helm_adlp", "helm_point"]
DTYPES = {"f8": np.float64, "u4": np.uint32, "c16": np.complex128}
# Arrays stored only in part, to keep the fixtures small: name -> number of leading columns kept
# (matrices are written column-major, i.e. shape (cols, rows)).
CROP = {"c1_dlp": 128}
# Arrays not stored: the adjoint double layer's transfer matrices and column bases equal the single
# layer's, which other fixtures pin already.
DROP = {f"{p}_{part}" for p in ("adh2ll", "adh2cc", "hadh2cc")
        for part in ("row_E", "col_E", "col_V")}


def build():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref",
                           f"REF={REF}", f"-j{os.cpu_count()}"])
    exes = {}
    for variant, flags in (("real", []), ("complex", ["-DUSE_COMPLEX"])):
        exe = os.path.join(REFOUT, f"gen_golden_{variant}")
        # the complex build links the reference's Helmholtz test for its exterior-field
        # evaluation (eval_brakhage_werner_c/_l, max_rel_outer_error), its main renamed
        extra = []
        if variant == "complex":
            obj = os.path.join(REFOUT, "test_helmholtzbem3d.o")
            subprocess.check_call(["gcc", "-O2", "-w", "-c", *flags, f"-I{REF}/Library",
                                   "-Dmain=h2lib_test_helmholtzbem3d_main",
                                   f"{REF}/Tests/test_helmholtzbem3d.c", "-o", obj])
            extra = [obj]
        subprocess.check_call(["gcc", "-O2", "-w", *flags, f"-I{REF}/Library",
                               os.path.join(HERE, "gen_golden.c"), *extra, "-o", exe,
                               f"-L{REFOUT}", f"-lh2ref_{variant}",
                               f"-Wl,-rpath,{REFOUT}", "-lm"])
        exes[variant] = exe
    return exes


def run_section(exe, section):
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.check_call([exe, tmp, section])
        arrays = {}
        with open(os.path.join(tmp, "manifest.txt")) as fh:
            for line in fh:
                parts = line.split()
                name, dt, shape = parts[0], DTYPES[parts[1]], tuple(int(s) for s in parts[2:])
                if name in DROP:
                    continue
                data = np.fromfile(os.path.join(tmp, name + ".bin"), dtype=dt)
                data = data.reshape(shape)
                if name in CROP:
                    data = data[:CROP[name]].copy()
                arrays[name] = data
    out = os.path.join(HERE, f"{section}.npz")
    np.savez_compressed(out, **arrays)
    print(f"{section}: {len(arrays)} arrays -> {os.path.relpath(out, ROOT)}")


def main(argv):
    sections = argv or REAL_SECTIONS + COMPLEX_SECTIONS
    exes = build()
    for s in sections:
        run_section(exes["complex" if s in COMPLEX_SECTIONS else "real"], s)


if __name__ == "__main__":
    main(sys.argv[1:])
