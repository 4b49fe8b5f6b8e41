"""ctypes wrapper of the C oracle (oracle/_build/liboracle.so) — TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker of
the CUDA library.  Builds the oracle with gcc on first use if the shared object is missing
(gcc is available wherever the tests run).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
vp = C.c_void_p

_dll = None


def _load():
    global _dll
    if _dll is None:
        src = os.path.join(HERE, "bem3d_oracle.c")
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
        d = C.CDLL(LIB)
        d.orc_gauss01.argtypes = [C.c_uint32, _f64p, _f64p]
        d.orc_rule.argtypes = [C.c_uint32, C.c_uint32, C.c_int, C.POINTER(C.c_uint32), vp, vp,
                               vp, vp, vp]
        d.orc_nearfield.argtypes = [C.c_uint32, _f64p, C.c_uint32, _u32p, _f64p, _f64p, C.c_int,
                                    C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_uint32,
                                    C.c_double, C.c_double, C.c_double, C.c_double, vp,
                                    C.c_uint32, vp, C.c_uint32, C.c_int, vp, C.c_uint64]
        d.orc_h2_new.restype = vp
        d.orc_h2_new.argtypes = [C.c_uint32, _f64p, C.c_uint32, _u32p, _f64p, _f64p, C.c_int,
                                 C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_uint32, C.c_double,
                                 C.c_double, C.c_double, C.c_double, C.c_uint32,
                                 C.c_uint32, _u32p, _f64p, C.c_uint32, _u32p,
                                 C.c_uint32, _u32p, _f64p, C.c_uint32, _u32p,
                                 C.c_uint32, _u32p, _u32p, _u8p]
        d.orc_h2_del.argtypes = [vp]
        d.orc_h2_export.argtypes = [vp, C.c_int, C.c_uint32, vp, C.POINTER(C.c_uint64)]
        d.orc_h2_addeval.argtypes = [vp, C.c_double, C.c_double, vp, vp]
        d.orc_gmres.argtypes = [C.c_uint32, vp, _f64p, vp, vp, C.c_double, C.c_uint32,
                                C.c_uint32]
        d.orc_gmres_unitary.argtypes = [C.c_uint32, vp, _f64p, vp, vp, C.c_double,
                                        C.c_uint32, C.c_uint32]
        d.orc_project_l2_harmonic.argtypes = [C.c_uint32, _f64p, C.c_uint32, _u32p, _f64p,
                                              C.c_uint32, _f64p, _f64p]
        d.orc_l2_error_harmonic.argtypes = [C.c_uint32, _f64p, C.c_uint32, _u32p, _f64p, _f64p,
                                            C.c_uint32, _f64p, _f64p, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]
        d.orc_integrate_point_source.argtypes = [C.c_uint32, _f64p, C.c_uint32, _u32p, _f64p,
                                                 C.c_uint32, C.c_int, _f64p, C.c_double, vp]
        d.orc_eval_brakhage_werner.argtypes = [C.c_uint32, _f64p, C.c_uint32, _u32p, _f64p,
                                               _f64p, C.c_uint32, C.c_int, C.c_double,
                                               C.c_double, C.c_double, C.c_double, vp,
                                               C.c_uint32, _f64p, vp]
        _dll = d
    return _dll


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def gauss01(m):
    x, w = np.zeros(m), np.zeros(m)
    assert _load().orc_gauss01(m, x, w) == 0
    return x, w


def rule(q, q2, which):
    n = C.c_uint32()
    d = _load()
    assert d.orc_rule(q, q2, which, C.byref(n), None, None, None, None, None) == 0
    arr = [np.zeros(n.value) for _ in range(5)]
    assert d.orc_rule(q, q2, which, C.byref(n), *[_p(a) for a in arr]) == 0
    return dict(zip(("x0", "x1", "y0", "y1", "w"), arr))


class Mesh:
    def __init__(self, x, t, n, g):
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.t = np.ascontiguousarray(t, dtype=np.uint32)
        self.n = np.ascontiguousarray(n, dtype=np.float64)
        self.g = np.ascontiguousarray(g, dtype=np.float64)
        self.nv, self.nt = self.x.shape[0], self.t.shape[0]


LAPLACE, HELMHOLTZ, SLP, DLP, ADLP = 0, 1, 0, 1, 2


def nearfield(mesh, pde, layer, rb, cb, ridx=None, cidx=None, q=2, q2=4, k=0.0, alpha=0.0,
              ntrans=False):
    rl, cl = rb == ord("l"), cb == ord("l")
    rows = (mesh.nv if rl else mesh.nt) if ridx is None else len(ridx)
    cols = (mesh.nv if cl else mesh.nt) if cidx is None else len(cidx)
    ri = None if ridx is None else np.ascontiguousarray(ridx, dtype=np.uint32)
    ci = None if cidx is None else np.ascontiguousarray(cidx, dtype=np.uint32)
    shape = (cols, rows) if ntrans else (rows, cols)
    cx = pde == HELMHOLTZ
    out = np.zeros(shape, dtype=np.complex128 if cx else np.float64, order="F")
    k, alpha = complex(k), complex(alpha)
    rc = _load().orc_nearfield(mesh.nv, mesh.x, mesh.nt, mesh.t, mesh.n, mesh.g, pde, layer, rb,
                               cb, q, q2, k.real, k.imag, alpha.real, alpha.imag, _p(ri), rows,
                               _p(ci), cols, int(ntrans), _p(out), shape[0])
    assert rc == 0
    return out


class H2:
    """Oracle H2 matrix on flattened trees (rec: (off,size,sons) per cluster, box: 6 per
    cluster, idx; blocks: (row cluster id, col cluster id, adm))."""

    def __init__(self, mesh, pde, layer, rb, cb, m, rtree, ctree, blocks, q=2, q2=4, k=0.0,
                 alpha=0.0):
        (rrec, rbox, ridx), (crec, cbox, cidx) = rtree, ctree
        # the C side keeps pointers to the index arrays: hold the converted copies
        self._keep = [np.ascontiguousarray(a, dtype=dt) for a, dt in (
            (rrec, np.uint32), (rbox, np.float64), (ridx, np.uint32), (crec, np.uint32),
            (cbox, np.float64), (cidx, np.uint32))]
        rrec, rbox, ridx, crec, cbox, cidx = self._keep
        brc = np.ascontiguousarray(blocks[0], dtype=np.uint32)
        bcc = np.ascontiguousarray(blocks[1], dtype=np.uint32)
        badm = np.ascontiguousarray(blocks[2], dtype=np.uint8)
        self._keep += [brc, bcc, badm, mesh]
        k, alpha = complex(k), complex(alpha)
        self.cx = pde == HELMHOLTZ
        self.handle = _load().orc_h2_new(
            mesh.nv, mesh.x, mesh.nt, mesh.t, mesh.n, mesh.g, pde, layer, rb, cb, q, q2, k.real,
            k.imag, alpha.real, alpha.imag, m, rrec.shape[0], rrec, rbox, ridx.shape[0], ridx,
            crec.shape[0], crec, cbox, cidx.shape[0], cidx, brc.shape[0], brc, bcc, badm)
        assert self.handle
        self.rows, self.cols = ridx.shape[0], cidx.shape[0]

    def export(self, part, count=0xFFFFFFFF):
        n = C.c_uint64()
        d = _load()
        assert d.orc_h2_export(self.handle, part, count, None, C.byref(n)) == 0
        out = np.zeros(n.value)
        assert d.orc_h2_export(self.handle, part, count, _p(out), C.byref(n)) == 0
        return out.view(np.complex128) if self.cx else out

    def addeval(self, alpha, x, y):
        alpha = complex(alpha)
        x = np.ascontiguousarray(x)
        assert _load().orc_h2_addeval(self.handle, alpha.real, alpha.imag, _p(x), _p(y)) == 0
        return y

    def __del__(self):
        if getattr(self, "handle", None):
            _load().orc_h2_del(self.handle)
            self.handle = None


def gmres(ops, coefs, b, x, eps, maxiter, kmax, unitary=False):
    """unitary: complex Givens rotations in unitary form (the reference's form otherwise)."""
    arr = (C.c_void_p * len(ops))(*[o.handle for o in ops])
    cf = np.zeros(2 * len(ops))
    for i, c in enumerate(coefs):
        cf[2 * i], cf[2 * i + 1] = complex(c).real, complex(c).imag
    fn = _load().orc_gmres_unitary if unitary else _load().orc_gmres
    return fn(len(ops), C.cast(arr, C.c_void_p), cf, _p(np.ascontiguousarray(b)), _p(x), eps,
              maxiter, kmax)


def project_l2_harmonic(mesh, z, q=2):
    w = np.zeros(mesh.nv)
    assert _load().orc_project_l2_harmonic(mesh.nv, mesh.x, mesh.nt, mesh.t, mesh.g, q,
                                           np.asarray(z, dtype=np.float64), w) == 0
    return w


def l2_error_harmonic(mesh, z, u, q=2):
    e, n = C.c_double(), C.c_double()
    assert _load().orc_l2_error_harmonic(mesh.nv, mesh.x, mesh.nt, mesh.t, mesh.n, mesh.g, q,
                                         np.asarray(z, dtype=np.float64),
                                         np.ascontiguousarray(u, dtype=np.float64),
                                         C.byref(e), C.byref(n)) == 0
    return e.value, n.value


def integrate_point_source(mesh, z, k, linear, q=2):
    """Point-source Dirichlet datum tested with the constant / linear basis (complex)."""
    b = np.zeros(mesh.nv if linear else mesh.nt, dtype=np.complex128)
    assert _load().orc_integrate_point_source(mesh.nv, mesh.x, mesh.nt, mesh.t, mesh.g, q,
                                              1 if linear else 0,
                                              np.asarray(z, dtype=np.float64), k, _p(b)) == 0
    return b


def eval_brakhage_werner(mesh, w, points, k, eta, linear, q=2):
    """Brakhage-Werner potential of the density w at the points (complex)."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    w = np.ascontiguousarray(w, dtype=np.complex128)
    u = np.zeros(len(pts), dtype=np.complex128)
    k, eta = complex(k), complex(eta)
    assert _load().orc_eval_brakhage_werner(mesh.nv, mesh.x, mesh.nt, mesh.t, mesh.n, mesh.g, q,
                                            1 if linear else 0, k.real, k.imag, eta.real,
                                            eta.imag, _p(w), len(pts), pts.ravel(), _p(u)) == 0
    return u
