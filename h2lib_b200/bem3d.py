"""Python mirror of H2Lib's bem3d / h2matrix / krylovsolvers interface for the B200 path.

Function names, argument order and meaning follow H2Lib (file:line of the reference given per
function); every compute call goes through the C ABI of libh2b200.so (include/h2b200.h).
Arrays may be numpy arrays (host) or CUDA tensors exposing data_ptr() (device).
"""
import ctypes as C
import sys

import numpy as np

from ._lib import (ADLP, BASIS_CONSTANT, BASIS_LINEAR, DLP, HELMHOLTZ, LAPLACE, MESH_CUBE,
                   MESH_SPHERE, SLP, H2BError, check, checkp, lib)

__all__ = [
    "BASIS_CONSTANT_BEM3D", "BASIS_LINEAR_BEM3D", "Surface3d", "new_sphere_surface3d",
    "new_cube_surface3d", "new_slp_laplace_bem3d", "new_dlp_laplace_bem3d",
    "new_slp_helmholtz_bem3d", "new_dlp_helmholtz_bem3d", "new_adlp_laplace_bem3d",
    "new_adlp_helmholtz_bem3d", "assemble_bem3d_amatrix",
    "nearfield", "Tree", "build_tree", "H2Matrix", "addeval_h2matrix_avector",
    "solve_gmres_h2matrix_avector", "solve_gmres", "quad_export",
]

BASIS_CONSTANT_BEM3D = BASIS_CONSTANT
BASIS_LINEAR_BEM3D = BASIS_LINEAR


def _ptr(a):
    """Raw pointer of a numpy array or a CUDA tensor."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"] and not a.flags["F_CONTIGUOUS"]:
            raise ValueError("array must be contiguous")
        return C.c_void_p(a.ctypes.data)
    raise TypeError(f"unsupported array type {type(a)}")


class Surface3d:
    """Mesh arrays of H2Lib's struct _surface3d (Library/surface3d.h:45) plus the device copy."""

    def __init__(self, x, t):
        self.x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        self.t = np.ascontiguousarray(t, dtype=np.uint32).reshape(-1, 3)
        self.vertices = self.x.shape[0]
        self.triangles = self.t.shape[0]
        self.n = np.zeros((self.triangles, 3))
        self.g = np.zeros(self.triangles)
        h = np.zeros(2)
        check(lib.h2b_prepare_surface(self.vertices, self.x, self.triangles, self.t, self.n,
                                      self.g, h), "prepare_surface3d")
        self.hmin, self.hmax = h
        self._dev = None

    @property
    def handle(self):
        if self._dev is None:
            self._dev = checkp(lib.h2b_surface_new(self.vertices, self.x, self.triangles, self.t,
                                                   self.n, self.g), "h2b_surface_new")
        return self._dev

    def __del__(self):
        # at interpreter exit the handles are left to the process teardown: the garbage
        # collector may finalise an object after the surface or structure it depends on
        if getattr(self, "_dev", None) and not sys.is_finalizing():
            try:
                lib.h2b_surface_del(self._dev)
            except Exception:  # interpreter shutdown
                pass
            self._dev = None


def _macro(kind, split):
    nv, nt = C.c_uint32(), C.c_uint32()
    check(lib.h2b_macro_mesh_size(kind, split, C.byref(nv), C.byref(nt)), "macro_mesh_size")
    x = np.zeros((nv.value, 3))
    t = np.zeros((nt.value, 3), dtype=np.uint32)
    check(lib.h2b_macro_mesh_build(kind, split, x, t), "macro_mesh_build")
    return x, t


def new_sphere_surface3d(split):
    """new_sphere_macrosurface3d + build_from_macrosurface3d_surface3d(mg, split)
    (Library/macrosurface3d.c:81, :707): 8*split^2 triangles on the unit sphere."""
    return Surface3d(*_macro(MESH_SPHERE, split))


def new_cube_surface3d(split):
    """new_cube_macrosurface3d + build_from_macrosurface3d_surface3d (Library/macrosurface3d.c:390,
    :707): 12*split^2 triangles on the surface of [-1,1]^3."""
    return Surface3d(*_macro(MESH_CUBE, split))


def new_ellipsoid_surface3d(split, axes):
    """Sphere refined `split` times, scaled per axis (semi-axes `axes`)."""
    x, t = _macro(MESH_SPHERE, split)
    check(lib.h2b_scale_vertices(x.shape[0], x, np.asarray(axes, dtype=np.float64)), "scale")
    return Surface3d(x, t)


def union_surface3d(surfaces):
    """One Surface3d holding several disjoint surfaces (vertices and triangles concatenated, the
    triangles' vertex ids shifted).  Returns (surface, vertex_off, triangle_off): surface m owns
    vertices [vertex_off[m], vertex_off[m+1]) and triangles [triangle_off[m], triangle_off[m+1])."""
    voff = np.zeros(len(surfaces) + 1, dtype=np.uint32)
    toff = np.zeros(len(surfaces) + 1, dtype=np.uint32)
    for m, gr in enumerate(surfaces):
        voff[m + 1] = voff[m] + gr.vertices
        toff[m + 1] = toff[m] + gr.triangles
    x = np.concatenate([gr.x for gr in surfaces])
    t = np.concatenate([gr.t.astype(np.uint64) + int(voff[m])
                        for m, gr in enumerate(surfaces)]).astype(np.uint32)
    return Surface3d(x, t), voff, toff


class Bem3d:
    """Operator handle: the counterpart of H2Lib's pbem3d (Library/bem3d.h:290)."""

    def __init__(self, gr, pde, layer, q_regular, q_singular, row_basis, col_basis, k=0.0,
                 alpha=0.0):
        self.gr = gr
        self.pde, self.layer = pde, layer
        self.row_basis, self.col_basis = row_basis, col_basis
        self.k = complex(k)
        self.alpha = complex(alpha)
        self.q_regular, self.q_singular = q_regular, q_singular
        self.handle = checkp(lib.h2b_bem_new(gr.handle, pde, layer, row_basis, col_basis,
                                             q_regular, q_singular, self.k.real, self.k.imag,
                                             self.alpha.real, self.alpha.imag), "h2b_bem_new")
        self.rows = gr.vertices if row_basis == BASIS_LINEAR else gr.triangles
        self.cols = gr.vertices if col_basis == BASIS_LINEAR else gr.triangles
        self.dtype = np.complex128 if pde == HELMHOLTZ else np.float64

    def timings(self):
        """Device ms of the distant and singular kernels of the last nearfield or dense
        assembly call on this operator."""
        ms = np.zeros(2)
        check(lib.h2b_bem_timings(self.handle, ms), "timings")
        return dict(zip(("near_distant", "near_singular"), ms.tolist()))

    def __del__(self):
        # at interpreter exit the handles are left to the process teardown: the garbage
        # collector may finalise an object after the surface or structure it depends on
        if getattr(self, "handle", None) and not sys.is_finalizing():
            try:
                lib.h2b_bem_del(self.handle)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None


def new_slp_laplace_bem3d(gr, q_regular, q_singular, row_basis, col_basis):
    """Library/laplacebem3d.c:844"""
    return Bem3d(gr, LAPLACE, SLP, q_regular, q_singular, row_basis, col_basis)


def new_dlp_laplace_bem3d(gr, q_regular, q_singular, row_basis, col_basis, alpha):
    """Library/laplacebem3d.c:1012"""
    return Bem3d(gr, LAPLACE, DLP, q_regular, q_singular, row_basis, col_basis, alpha=alpha)


def new_slp_helmholtz_bem3d(k, gr, q_regular, q_singular, row_basis, col_basis):
    """Library/helmholtzbem3d.c:1008"""
    return Bem3d(gr, HELMHOLTZ, SLP, q_regular, q_singular, row_basis, col_basis, k=k)


def new_dlp_helmholtz_bem3d(k, gr, q_regular, q_singular, row_basis, col_basis, alpha):
    """Library/helmholtzbem3d.c:1177"""
    return Bem3d(gr, HELMHOLTZ, DLP, q_regular, q_singular, row_basis, col_basis, k=k,
                 alpha=alpha)


def new_adlp_laplace_bem3d(gr, q_regular, q_singular, row_basis, col_basis, alpha):
    """Adjoint double layer K' + alpha M (Library/laplacebem3d.c:1180)"""
    return Bem3d(gr, LAPLACE, ADLP, q_regular, q_singular, row_basis, col_basis, alpha=alpha)


def new_adlp_helmholtz_bem3d(k, gr, q_regular, q_singular, row_basis, col_basis, alpha):
    """Library/helmholtzbem3d.c:1346"""
    return Bem3d(gr, HELMHOLTZ, ADLP, q_regular, q_singular, row_basis, col_basis, k=k,
                 alpha=alpha)


def nearfield(bem, ridx, cidx, ntrans=False, out=None):
    """bem->nearfield(ridx, cidx, bem, ntrans, N) (Library/bem3d.h:380).  Returns N as a
    column-major (Fortran-ordered) numpy array of shape (rows, cols) (transposed if ntrans)."""
    rows = bem.rows if ridx is None else len(ridx)
    cols = bem.cols if cidx is None else len(cidx)
    ri = None if ridx is None else np.ascontiguousarray(ridx, dtype=np.uint32)
    ci = None if cidx is None else np.ascontiguousarray(cidx, dtype=np.uint32)
    shape = (cols, rows) if ntrans else (rows, cols)
    if out is None:
        out = np.zeros(shape, dtype=bem.dtype, order="F")
    ld = out.shape[0] if isinstance(out, np.ndarray) else shape[0]
    check(lib.h2b_bem_nearfield(bem.handle, _ptr(ri), rows, _ptr(ci), cols, int(ntrans),
                                _ptr(out), ld), "nearfield")
    return out


def assemble_bem3d_amatrix(bem, G=None):
    """Library/bem3d.c:9988: dense matrix of the operator (square)."""
    if G is None:
        G = np.zeros((bem.rows, bem.rows), dtype=bem.dtype, order="F")
    ld = G.shape[0] if isinstance(G, np.ndarray) else bem.rows
    check(lib.h2b_bem_assemble_amatrix(bem.handle, _ptr(G), ld), "assemble_bem3d_amatrix")
    return G


class Tree:
    """Cluster trees + block leaves (build_bem3d_cluster, Library/bem3d.c:932;
    build_strict_block + admissible_max_cluster, Library/block.c:258/52)."""

    def __init__(self, handle):
        self.handle = handle
        info = np.zeros(8, dtype=np.uint64)
        check(lib.h2b_tree_info(handle, info), "tree_info")
        self.row_clusters, self.col_clusters = int(info[0]), int(info[1])
        self.row_n, self.col_n = int(info[2]), int(info[3])
        self.blocks, self.admissible, self.near_entries = int(info[4]), int(info[5]), int(info[6])
        self.row_depth, self.col_depth = int(info[7]) & 0xFFFFFFFF, int(info[7]) >> 32

    def clusters(self, which=0):
        n = self.row_clusters if which == 0 else self.col_clusters
        m = self.row_n if which == 0 else self.col_n
        rec = np.zeros((n, 3), dtype=np.uint32)
        box = np.zeros((n, 6))
        idx = np.zeros(m, dtype=np.uint32)
        check(lib.h2b_tree_export_clusters(self.handle, which, _ptr(rec), _ptr(box), _ptr(idx)),
              "export_clusters")
        return rec, box, idx

    def block_records(self):
        rec = np.zeros((self.blocks, 5), dtype=np.uint32)
        check(lib.h2b_tree_export_blocks(self.handle, rec), "export_blocks")
        return rec

    def __del__(self):
        # at interpreter exit the handles are left to the process teardown: the garbage
        # collector may finalise an object after the surface or structure it depends on
        if getattr(self, "handle", None) and not sys.is_finalizing():
            try:
                lib.h2b_tree_del(self.handle)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None


def build_tree(gr, row_basis, col_basis, clf, eta, device=False):
    """Cluster and block trees, built on the host (h2b_tree_new) or on the device
    (h2b_tree_new_device); both give the same trees."""
    fn = lib.h2b_tree_new_device if device else lib.h2b_tree_new
    return Tree(checkp(fn(gr.vertices, gr.x, gr.triangles, gr.t, row_basis, col_basis, clf, eta),
                       "h2b_tree_new_device" if device else "h2b_tree_new"))


def build_forest(gr, vertex_off, triangle_off, row_basis, col_basis, clf, eta):
    """Cluster and block trees of every surface of a union (union_surface3d), side by side: the
    H2 matrix on this forest is block diagonal, one block per surface."""
    return Tree(checkp(lib.h2b_tree_new_forest(len(vertex_off) - 1,
                                               np.ascontiguousarray(vertex_off, dtype=np.uint32),
                                               np.ascontiguousarray(triangle_off, dtype=np.uint32),
                                               gr.x, gr.t, row_basis, col_basis, clf, eta),
                       "h2b_tree_new_forest"))


class H2Matrix:
    """Device H2 matrix with Chebyshev interpolation (setup_h2matrix_aprx_inter_bem3d,
    Library/bem3d.c:9658)."""

    def __init__(self, bem, tree, m, like=None, green=None):
        """like: an H2Matrix on the same surface, trees, bases and quadrature whose device
        structure this one shares (h2b_h2matrix_new_like); it is kept alive by this object.
        green: (l, delta, accur) for the greenhybrid farfield with m Gauss points on each of l
        parts per box-face axis (setup_h2matrix_aprx_greenhybrid_bem3d, Library/bem3d.c:9689);
        a matrix made like a greenhybrid one is greenhybrid too."""
        self.bem, self.tree, self.m, self._like = bem, tree, m, like
        self.green = green if like is None else like.green
        if like is not None:
            self.handle = checkp(lib.h2b_h2matrix_new_like(bem.handle, like.handle),
                                 "h2matrix_new_like")
        elif green is not None:
            l, delta, accur = green
            self.handle = checkp(lib.h2b_h2matrix_new_greenhybrid(bem.handle, tree.handle, m, l,
                                                                  delta, accur),
                                 "h2matrix_new_greenhybrid")
        else:
            self.handle = checkp(lib.h2b_h2matrix_new(bem.handle, tree.handle, m),
                                 "h2matrix_new")
        self.rows, self.cols, self.dtype = bem.rows, bem.cols, bem.dtype

    def assemble(self):
        """assemble_bem3d_h2matrix_row/col_clusterbasis + assemble_bem3d_h2matrix."""
        check(lib.h2b_h2matrix_assemble_all(self.handle), "h2matrix_assemble_all")
        return self

    def set_precision(self, fp32):
        """FP32 (True) or FP64 (False, default) distant-pair quadrature for later assembly."""
        check(lib.h2b_h2matrix_set_precision(self.handle, 1 if fp32 else 0), "set_precision")
        return self

    def make_single(self):
        """FP32 copies of N, S and the flattened bases for mixed-precision products."""
        check(lib.h2b_h2matrix_make_single(self.handle), "h2matrix_make_single")
        return self

    SHAPE_NAMES = ("fwd_rows", "back_rows", "ctas_per_sm", "stages_per_warp", "panel_kib",
                   "leaf_ctas", "consumer_warps")

    def matvec_shape(self):
        """The launch shape of the matvec and leaf-basis kernels (h2b_h2matrix_get_matvec_shape)."""
        sh = np.zeros(7, dtype=np.uint32)
        check(lib.h2b_h2matrix_get_matvec_shape(self.handle, sh), "get_matvec_shape")
        return dict(zip(self.SHAPE_NAMES, (int(v) for v in sh)))

    def set_matvec_shape(self, **kw):
        """Sets entries of the launch shape by name (see matvec_shape); the others are kept."""
        sh = np.zeros(7, dtype=np.uint32)
        for k, v in kw.items():
            sh[self.SHAPE_NAMES.index(k)] = v
        check(lib.h2b_h2matrix_set_matvec_shape(self.handle, sh), "set_matvec_shape")
        return self

    def autotune(self, matvec=True, leaf=False):
        """h2b_h2matrix_autotune: the chosen shape and the costs (device ms) before and after."""
        flags = (1 if matvec else 0) | (2 if leaf else 0)
        sh = np.zeros(7, dtype=np.uint32)
        ms = np.zeros(4)
        check(lib.h2b_h2matrix_autotune(self.handle, flags, sh, ms), "autotune")
        return dict(shape=self.matvec_shape(), matvec_ms=(float(ms[0]), float(ms[1])),
                    bases_ms=(float(ms[2]), float(ms[3])))

    def info(self):
        info = np.zeros(8, dtype=np.uint64)
        check(lib.h2b_h2matrix_info(self.handle, info), "h2matrix_info")
        return dict(near_entries=int(info[0]), coupling_entries=int(info[1]),
                    leaf_entries=int(info[2]), transfer_entries=int(info[3]),
                    bytes=int(info[4]), admissible=int(info[5]), near_blocks=int(info[6]),
                    rank=int(info[7]))

    def timings(self):
        """Device ms of the last row basis, column basis, coupling, nearfield distant,
        nearfield singular and matvec runs."""
        ms = np.zeros(6)
        check(lib.h2b_h2matrix_timings(self.handle, ms), "timings")
        return dict(zip(("row_basis", "col_basis", "coupling", "near_distant", "near_singular",
                         "matvec"), ms.tolist()))

    def pair_counts(self):
        c = np.zeros(4, dtype=np.uint64)
        check(lib.h2b_h2matrix_pair_counts(self.handle, c), "pair_counts")
        return dict(zip(("distant", "vertex", "edge", "identical"), (int(v) for v in c)))

    def green_ranks(self, side=0):
        """Ranks of the greenhybrid cluster bases (0 row, 1 column), tree pre-order."""
        n = self.tree.row_clusters if side == 0 else self.tree.col_clusters
        out = np.zeros(n, dtype=np.uint32)
        check(lib.h2b_h2matrix_green_ranks(self.handle, side, _ptr(out)), "green_ranks")
        return out

    def export_green(self, part):
        """Greenhybrid parts with their per-cluster ranks (h2b_h2matrix_export_green): 0 / 2 row /
        column leaf bases, 1 / 3 transfers, 4 couplings, concatenated in H2Lib's layouts."""
        n = np.zeros(1, dtype=np.uint64)
        check(lib.h2b_h2matrix_export_green(self.handle, part, None, _ptr(n)), "export_green")
        out = np.zeros(int(n[0]))
        check(lib.h2b_h2matrix_export_green(self.handle, part, _ptr(out), _ptr(n)),
              "export_green")
        return out

    def unique_pairs(self):
        """Distinct triangle pairs among pair_counts(), by the same cases (device bitmap)."""
        c = np.zeros(4, dtype=np.uint64)
        check(lib.h2b_h2matrix_unique_pairs(self.handle, c), "unique_pairs")
        return dict(zip(("distant", "vertex", "edge", "identical"), (int(v) for v in c)))

    def export(self, part, count=0xFFFFFFFF):
        n = C.c_uint64()
        check(lib.h2b_h2matrix_export(self.handle, part, count, None, C.byref(n)), "export")
        # cluster bases and transfer matrices (parts 0-3) are real for every operator
        if self.dtype == np.complex128 and part >= 4:
            out = np.zeros(n.value // 2, dtype=np.complex128)
        else:
            out = np.zeros(n.value)
        check(lib.h2b_h2matrix_export(self.handle, part, count, _ptr(out), C.byref(n)), "export")
        return out

    def __del__(self):
        # at interpreter exit the handles are left to the process teardown: the garbage
        # collector may finalise an object after the surface or structure it depends on
        if getattr(self, "handle", None) and not sys.is_finalizing():
            try:
                lib.h2b_h2matrix_del(self.handle)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None


def addeval_h2matrix_avector_single(alpha, h2, x, y):
    """y += alpha * A x from the FP32 copies of the matrix (H2Matrix.make_single)."""
    alpha = complex(alpha)
    check(lib.h2b_h2matrix_addeval_single(alpha.real, alpha.imag, h2.handle, _ptr(x), _ptr(y)),
          "addeval_h2matrix_avector_single")
    return y


def addeval_h2matrix_avector(alpha, h2, x, y):
    """y += alpha * A x (Library/h2matrix.c:1269)."""
    alpha = complex(alpha)
    check(lib.h2b_h2matrix_addeval(alpha.real, alpha.imag, h2.handle, _ptr(x), _ptr(y)),
          "addeval_h2matrix_avector")
    return y


def solve_gmres(ops, coefs, b, x, eps, maxiter, kmax, unitary=False):
    """GMRES on sum_i coefs[i] * ops[i] (solve_gmres_avector, Library/krylovsolvers.c:183).
    unitary: complex Givens rotations in unitary form (H2B_SOLVE_UNITARY), so that the stop at
    eps holds for the true residual of a complex system; the default keeps the reference's
    rotations and iteration counts."""
    if unitary:
        n = ops[0].rows
        it = solve_gmres_batch(ops, coefs, [0, n], b, x, eps, maxiter, kmax, unitary=True)
        return int(it[0, 0])
    arr = (C.c_void_p * len(ops))(*[o.handle for o in ops])
    cf = np.zeros(2 * len(ops))
    for i, c in enumerate(coefs):
        cf[2 * i], cf[2 * i + 1] = complex(c).real, complex(c).imag
    return check(lib.h2b_solve_gmres(len(ops), C.cast(arr, C.c_void_p), cf, _ptr(b), _ptr(x),
                                     eps, maxiter, kmax), "solve_gmres")


SOLVE_MIXED = 1
SOLVE_UNITARY = 2


def _coefs(ops, coefs):
    arr = (C.c_void_p * len(ops))(*[o.handle for o in ops])
    cf = np.zeros(2 * len(ops))
    for i, c in enumerate(coefs):
        cf[2 * i], cf[2 * i + 1] = complex(c).real, complex(c).imag
    return C.cast(arr, C.c_void_p), cf, arr


def solve_gmres_batch(ops, coefs, system_off, b, x, eps, maxiter, kmax, nrhs=1, mixed=False,
                      unitary=False):
    """Independent GMRES solves of the diagonal blocks [system_off[s], system_off[s+1]) of a block
    diagonal operator (an H2 matrix on a forest), all in one device loop; with nrhs > 1, b and x
    hold nrhs columns.  mixed: FP32 Arnoldi steps, FP64 residuals (make_single first; implies
    unitary).  unitary: unitary complex Givens rotations.  Returns the iteration counts, shape
    (nrhs, systems)."""
    ptr, cf, _keep = _coefs(ops, coefs)
    off = np.ascontiguousarray(system_off, dtype=np.uint32)
    iters = np.zeros(nrhs * (off.size - 1), dtype=np.uint32)
    check(lib.h2b_solve_gmres_batch(len(ops), ptr, cf, off.size - 1, off, nrhs, _ptr(b),
                                    _ptr(x), eps, maxiter, kmax,
                                    (SOLVE_MIXED if mixed else 0) |
                                    (SOLVE_UNITARY if unitary else 0), iters),
          "solve_gmres_batch")
    return iters.reshape(nrhs, off.size - 1)


def solve_gmres_mixed(ops, coefs, b, x, eps, maxiter, kmax):
    """solve_gmres with FP32 Arnoldi steps and FP64 residuals (iterative refinement); the
    operators need their FP32 copies (H2Matrix.make_single)."""
    ptr, cf, _keep = _coefs(ops, coefs)
    return check(lib.h2b_solve_gmres_mixed(len(ops), ptr, cf, _ptr(b), _ptr(x), eps, maxiter,
                                           kmax), "solve_gmres_mixed")


def solve_gmres_h2matrix_avector(A, b, x, eps, maxiter, kmax):
    """Library/krylovsolvers.c:254"""
    return solve_gmres([A], [1.0], b, x, eps, maxiter, kmax)


def residual_norm(ops, coefs, b, x):
    arr = (C.c_void_p * len(ops))(*[o.handle for o in ops])
    cf = np.zeros(2 * len(ops))
    for i, c in enumerate(coefs):
        cf[2 * i], cf[2 * i + 1] = complex(c).real, complex(c).imag
    r = C.c_double()
    check(lib.h2b_residual_norm(len(ops), C.cast(arr, C.c_void_p), cf, _ptr(b), _ptr(x),
                                C.byref(r)), "residual_norm")
    return r.value


def project_l2_harmonic(bem, z, w=None):
    """projectL2_bem3d_l_avector with eval_dirichlet_fundamental_laplacebem3d
    (Library/bem3d.c:9009, Library/laplacebem3d.c:1391)."""
    if w is None:
        w = np.zeros(bem.gr.vertices)
    check(lib.h2b_project_l2_harmonic(bem.handle, np.asarray(z, dtype=np.float64), _ptr(w)),
          "project_l2_harmonic")
    return w


def l2_error_harmonic(bem, z, u):
    """(normL2diff_l_bem3d, normL2_bem3d) against the Neumann trace of 1/|x - z|."""
    e, n = C.c_double(), C.c_double()
    check(lib.h2b_l2_error_harmonic(bem.handle, np.asarray(z, dtype=np.float64), _ptr(u),
                                    C.byref(e), C.byref(n)), "l2_error_harmonic")
    return e.value, n.value


def project_l2_harmonic_multi(bem, triangle_off, zs, w=None):
    """project_l2_harmonic on a union of surfaces with one source per (column, surface):
    zs has shape (nrhs, surfaces, 3); returns w of shape (nrhs, vertices)."""
    zs = np.ascontiguousarray(zs, dtype=np.float64)
    nrhs, nseg = zs.shape[0], zs.shape[1]
    if w is None:
        w = np.zeros((nrhs, bem.gr.vertices))
    check(lib.h2b_project_l2_harmonic_multi(bem.handle, nseg,
                                            np.ascontiguousarray(triangle_off, dtype=np.uint32),
                                            nrhs, zs.reshape(-1), _ptr(w)),
          "project_l2_harmonic_multi")
    return w


def l2_error_harmonic_multi(bem, triangle_off, zs, u):
    """l2_error_harmonic per (column, surface); returns (err, norm), each (nrhs, surfaces)."""
    zs = np.ascontiguousarray(zs, dtype=np.float64)
    nrhs, nseg = zs.shape[0], zs.shape[1]
    err = np.zeros(nrhs * nseg)
    nrm = np.zeros(nrhs * nseg)
    check(lib.h2b_l2_error_harmonic_multi(bem.handle, nseg,
                                          np.ascontiguousarray(triangle_off, dtype=np.uint32),
                                          nrhs, zs.reshape(-1), _ptr(u), err, nrm),
          "l2_error_harmonic_multi")
    return err.reshape(nrhs, nseg), nrm.reshape(nrhs, nseg)


def integrate_plane_wave(bem, kvec, src=(0.0, 0.0, 0.0), coef=1.0, b=None):
    """b_t = coef * int_t exp(i kvec.(x - src)) (integrate_bem3d_c_avector with
    rhs_dirichlet_plane_helmholtzbem3d, Library/bem3d.c:8579, Library/helmholtzbem3d.c:1611)."""
    if b is None:
        b = np.zeros(bem.gr.triangles, dtype=np.complex128)
    coef = complex(coef)
    check(lib.h2b_integrate_plane_wave(bem.handle, np.asarray(kvec, dtype=np.float64),
                                       np.asarray(src, dtype=np.float64), coef.real, coef.imag,
                                       _ptr(b)), "integrate_plane_wave")
    return b


def integrate_point_source(bem, src, k, coef=1.0, b=None):
    """b_i = coef * int e^{ik|x - src|} / |x - src| phi_i(x) dx with the row basis
    (integrate_bem3d_c/l_avector with rhs_dirichlet_point_helmholtzbem3d, Library/bem3d.c:8579,
    :8631, Library/helmholtzbem3d.c:1521)."""
    if b is None:
        b = np.zeros(bem.rows, dtype=np.complex128)
    coef = complex(coef)
    check(lib.h2b_integrate_point_source(bem.handle, np.asarray(src, dtype=np.float64), float(k),
                                         coef.real, coef.imag, _ptr(b)), "integrate_point_source")
    return b


def eval_brakhage_werner(bem, w, points, eta):
    """Brakhage-Werner potential of the density w at the points (n x 3) outside the surface
    (eval_brakhage_werner_c / _l, Tests/test_helmholtzbem3d.c:68 / :134)."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    w = np.ascontiguousarray(w, dtype=np.complex128)
    u = np.zeros(len(pts), dtype=np.complex128)
    eta = complex(eta)
    check(lib.h2b_eval_brakhage_werner(bem.handle, len(pts), pts.ravel(), _ptr(w), eta.real,
                                       eta.imag, _ptr(u)), "eval_brakhage_werner")
    return u


def outer_points(n=20, half=10.0):
    """The evaluation points of the reference's exterior test (max_rel_outer_error,
    Tests/test_helmholtzbem3d.c:224): an n x n grid of the plane y = 0 over [-half, half]^2,
    the points with x^2 + z^2 > 1."""
    pts = []
    for j in range(n):
        for i in range(n):
            p = (-half + (2 * half / (n - 1)) * i, 0.0, -half + (2 * half / (n - 1)) * j)
            if p[0] ** 2 + p[2] ** 2 > 1:
                pts.append(p)
    return np.array(pts)


def point_source_field(points, src, k):
    """e^{ik|x - src|} / |x - src| (rhs_dirichlet_point_helmholtzbem3d)."""
    r = np.linalg.norm(np.asarray(points) - np.asarray(src), axis=1)
    return np.exp(1j * k * r) / r


def quad_export(q, q2, row_basis, col_basis, which):
    """Quadrature rule tables (Library/singquad2d.c:25-320): dict of arrays."""
    n = C.c_uint32()
    check(lib.h2b_quad_export(q, q2, row_basis, col_basis, which, C.byref(n), None, None, None,
                              None, None), "quad_export")
    n = n.value
    x0, x1, y0, y1 = (np.zeros(n) for _ in range(4))
    w = np.zeros((4 if which == 4 else 10) * n)
    check(lib.h2b_quad_export(q, q2, row_basis, col_basis, which, C.byref(C.c_uint32()),
                              _ptr(x0), _ptr(x1), _ptr(y0), _ptr(y1), _ptr(w)), "quad_export")
    return dict(n=n, x0=x0, x1=x1, y0=y0, y1=y1, w=w.reshape(-1, n))
