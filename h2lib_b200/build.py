"""Build libh2b200.so in-tree (h2lib_b200/libh2b200.so) for sm_100a.

Host sources (*.c) are compiled with gcc, device sources (*.cu) with nvcc
(-gencode arch=compute_100a,code=sm_100a), objects go to h2lib_b200/_build/ and are rebuilt when a
source or header is newer than its object.  nvcc cross-compiles, so no GPU is needed.

    python -m h2lib_b200.build [--force]
"""
import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libh2b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O2", "-fPIC", "-std=gnu11", "-Wall", "-fno-fast-math", f"-I{CSRC}", f"-I{INCLUDE}"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-O3",
                  "--expt-relaxed-constexpr", f"-I{CSRC}", f"-I{INCLUDE}"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the sm_100a library cannot be built")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(src, obj, newest_header):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or newest_header > t


def _compile(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    return res.stderr


def build(force=False, verbose=False, defines=(), lib=LIB, build_dir=BUILD):
    """Compile and link; `defines` (e.g. ["-DH2B_FOO=1"]) build a variant into `lib`,
    with objects in `build_dir`."""
    os.makedirs(build_dir, exist_ok=True)
    nvcc = _nvcc()
    newest_header = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    jobs, objs = [], []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.c"))):
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(src, obj, newest_header):
            jobs.append(["gcc", *CFLAGS, *defines, "-c", src, "-o", obj])
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(src, obj, newest_header):
            jobs.append([nvcc, *NVFLAGS, *defines, "-c", src, "-o", obj])
    if jobs:
        with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
            for out in ex.map(_compile, jobs):
                if verbose and out:
                    print(out, file=sys.stderr)
    if jobs or force or not os.path.exists(lib) or \
            any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        tmp = lib + ".tmp"
        _compile([nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcuda", "-lpthread", "-lm"])
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
