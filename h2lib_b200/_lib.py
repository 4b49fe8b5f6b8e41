"""ctypes binding of libh2b200.so (the C ABI declared in include/h2b200.h).

The shared library is built in-tree by h2lib_b200.build; importing this module never compiles and
never substitutes another implementation: if the library is missing, every call raises.
"""
import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
# H2B_LIBRARY selects another build of the same library (e.g. a variant compiled with different
# kernel options); by default the in-tree libh2b200.so is used.
LIBPATH = os.environ.get("H2B_LIBRARY") or os.path.join(PKG, "libh2b200.so")

H2B_OK = 0
BASIS_CONSTANT = ord("c")
BASIS_LINEAR = ord("l")
LAPLACE, HELMHOLTZ = 0, 1
SLP, DLP, ADLP = 0, 1, 2
MESH_SPHERE, MESH_CUBE = 0, 1

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
vp = C.c_void_p

# name: (restype, argtypes)
_SIGS = {
    "h2b_last_error": (C.c_char_p, []),
    "h2b_version": (C.c_char_p, []),
    "h2b_device_init": (C.c_int, [C.c_int]),
    "h2b_device_memory": (C.c_int, [_u64p]),
    "h2b_launch_count": (C.c_int, [C.POINTER(C.c_uint64)]),
    "h2b_macro_mesh_size": (C.c_int, [C.c_int, C.c_uint32, C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_uint32)]),
    "h2b_macro_mesh_build": (C.c_int, [C.c_int, C.c_uint32, _f64p, _u32p]),
    "h2b_prepare_surface": (C.c_int, [C.c_uint32, _f64p, C.c_uint32, _u32p, _f64p, _f64p, _f64p]),
    "h2b_scale_vertices": (C.c_int, [C.c_uint32, _f64p, _f64p]),
    "h2b_quad_export": (C.c_int, [C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(C.c_uint32), vp, vp, vp, vp, vp]),
    "h2b_tree_new": (vp, [C.c_uint32, _f64p, C.c_uint32, _u32p, C.c_int, C.c_int, C.c_uint32,
                          C.c_double]),
    "h2b_tree_new_device": (vp, [C.c_uint32, _f64p, C.c_uint32, _u32p, C.c_int, C.c_int,
                                 C.c_uint32, C.c_double]),
    "h2b_tree_new_flat": (vp, [C.c_uint32, _u32p, _u32p, _u32p, _f64p, C.c_uint32, _u32p,
                               C.c_uint32, _u32p, _u32p, _u32p, _f64p, C.c_uint32, _u32p,
                               C.c_uint32, _u32p, _u32p, _u8p]),
    "h2b_tree_new_forest": (vp, [C.c_uint32, _u32p, _u32p, _f64p, _u32p, C.c_int, C.c_int,
                                 C.c_uint32, C.c_double]),
    "h2b_tree_del": (None, [vp]),
    "h2b_tree_info": (C.c_int, [vp, _u64p]),
    "h2b_tree_export_clusters": (C.c_int, [vp, C.c_int, vp, vp, vp]),
    "h2b_tree_export_blocks": (C.c_int, [vp, _u32p]),
    "h2b_surface_new": (vp, [C.c_uint32, _f64p, C.c_uint32, _u32p, _f64p, _f64p]),
    "h2b_surface_del": (None, [vp]),
    "h2b_bem_new": (vp, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_uint32,
                         C.c_double, C.c_double, C.c_double, C.c_double]),
    "h2b_bem_del": (None, [vp]),
    "h2b_bem_nearfield": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, C.c_int, vp,
                                    C.c_uint64]),
    "h2b_bem_assemble_amatrix": (C.c_int, [vp, vp, C.c_uint64]),
    "h2b_bem_timings": (C.c_int, [vp, _f64p]),
    "h2b_h2matrix_new": (vp, [vp, vp, C.c_uint32]),
    "h2b_h2matrix_new_like": (vp, [vp, vp]),
    "h2b_h2matrix_new_greenhybrid": (vp, [vp, vp, C.c_uint32, C.c_uint32, C.c_double, C.c_double]),
    "h2b_h2matrix_green_ranks": (C.c_int, [vp, C.c_int, vp]),
    "h2b_h2matrix_export_green": (C.c_int, [vp, C.c_int, vp, vp]),
    "h2b_h2matrix_del": (None, [vp]),
    "h2b_h2matrix_assemble_row_clusterbasis": (C.c_int, [vp]),
    "h2b_h2matrix_assemble_col_clusterbasis": (C.c_int, [vp]),
    "h2b_h2matrix_assemble_nearfield": (C.c_int, [vp]),
    "h2b_h2matrix_assemble_farfield": (C.c_int, [vp]),
    "h2b_h2matrix_assemble": (C.c_int, [vp]),
    "h2b_h2matrix_assemble_all": (C.c_int, [vp]),
    "h2b_h2matrix_assemble_nearfield_pair": (C.c_int, [vp, vp]),
    "h2b_h2matrix_info": (C.c_int, [vp, _u64p]),
    "h2b_h2matrix_timings": (C.c_int, [vp, _f64p]),
    "h2b_h2matrix_pair_counts": (C.c_int, [vp, _u64p]),
    "h2b_h2matrix_unique_pairs": (C.c_int, [vp, _u64p]),
    "h2b_h2matrix_export": (C.c_int, [vp, C.c_int, C.c_uint32, vp, C.POINTER(C.c_uint64)]),
    "h2b_h2matrix_export_async": (C.c_int, [vp, C.c_int, C.c_uint32, vp]),
    "h2b_h2matrix_export_wait": (C.c_int, [vp]),
    "h2b_h2matrix_addeval": (C.c_int, [C.c_double, C.c_double, vp, vp, vp]),
    "h2b_h2matrix_addeval_multi": (C.c_int, [C.c_double, C.c_double, vp, C.c_uint32, vp,
                                             C.c_uint64, vp, C.c_uint64]),
    "h2b_solve_gmres": (C.c_int, [C.c_uint32, vp, _f64p, vp, vp, C.c_double, C.c_uint32,
                                  C.c_uint32]),
    "h2b_solve_gmres_batch": (C.c_int, [C.c_uint32, vp, _f64p, C.c_uint32, _u32p, C.c_uint32,
                                        vp, vp, C.c_double, C.c_uint32, C.c_uint32, C.c_uint32,
                                        _u32p]),
    "h2b_solve_gmres_mixed": (C.c_int, [C.c_uint32, vp, _f64p, vp, vp, C.c_double, C.c_uint32,
                                        C.c_uint32]),
    "h2b_h2matrix_make_single": (C.c_int, [vp]),
    "h2b_h2matrix_set_precision": (C.c_int, [vp, C.c_int]),
    "h2b_h2matrix_set_matvec_shape": (C.c_int, [vp, _u32p]),
    "h2b_h2matrix_get_matvec_shape": (C.c_int, [vp, _u32p]),
    "h2b_h2matrix_autotune": (C.c_int, [vp, C.c_uint32, _u32p, _f64p]),
    "h2b_autotune_save": (C.c_int, [C.c_char_p]),
    "h2b_autotune_load": (C.c_int, [C.c_char_p]),
    "h2b_autotune_clear": (C.c_int, []),
    "h2b_h2matrix_addeval_single": (C.c_int, [C.c_double, C.c_double, vp, vp, vp]),
    "h2b_residual_norm": (C.c_int, [C.c_uint32, vp, _f64p, vp, vp, C.POINTER(C.c_double)]),
    "h2b_solve_gmres_noalloc": (C.c_int, [C.c_uint32, vp, _f64p, vp, vp, C.c_double,
                                          C.c_uint32, C.c_uint32]),
    "h2b_project_l2_harmonic": (C.c_int, [vp, _f64p, vp]),
    "h2b_l2_error_harmonic": (C.c_int, [vp, _f64p, vp, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]),
    "h2b_server_new": (vp, [C.c_int, C.c_uint32, C.c_uint64]),
    "h2b_server_submit": (C.c_int64, [vp, vp]),
    "h2b_server_wait": (C.c_int, [vp, C.c_int64, vp, vp]),
    "h2b_server_stats": (C.c_int, [vp, _u64p]),
    "h2b_server_set_batching": (C.c_int, [vp, C.c_uint32]),
    "h2b_server_del": (None, [vp]),
    "h2b_project_l2_harmonic_multi": (C.c_int, [vp, C.c_uint32, _u32p, C.c_uint32, _f64p, vp]),
    "h2b_l2_error_harmonic_multi": (C.c_int, [vp, C.c_uint32, _u32p, C.c_uint32, _f64p, vp,
                                              _f64p, _f64p]),
    "h2b_integrate_plane_wave": (C.c_int, [vp, _f64p, _f64p, C.c_double, C.c_double, vp]),
    "h2b_integrate_point_source": (C.c_int, [vp, _f64p, C.c_double, C.c_double, C.c_double,
                                             vp]),
    "h2b_eval_brakhage_werner": (C.c_int, [vp, C.c_uint32, _f64p, vp, C.c_double, C.c_double,
                                           vp]),
}


class H2BError(RuntimeError):
    pass


class _Lib:
    def __init__(self):
        self._dll = None

    def _load(self):
        if self._dll is None:
            if not os.path.exists(LIBPATH):
                raise H2BError(f"{LIBPATH} is missing: build it with `python -m h2lib_b200.build`"
                               " (the CUDA library is required; there is no CPU fallback)")
            self._dll = C.CDLL(LIBPATH)
        return self._dll

    def __getattr__(self, name):
        if name not in _SIGS:
            raise AttributeError(name)
        dll = self._load()
        try:
            fn = getattr(dll, name)
        except AttributeError as e:
            raise H2BError(f"{name} is not exported by {LIBPATH}") from e
        fn.restype, fn.argtypes = _SIGS[name]
        setattr(self, name, fn)
        return fn

    def exported(self):
        dll = self._load()
        return [n for n in _SIGS if hasattr(dll, n)]


lib = _Lib()


def last_error():
    return lib.h2b_last_error().decode()


def check(rc, what=""):
    if rc < 0:
        raise H2BError(f"{what}: error {rc}: {last_error()}")
    return rc


def checkp(p, what=""):
    if not p:
        raise H2BError(f"{what}: {last_error()}")
    return p
