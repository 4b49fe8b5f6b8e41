"""h2lib_b200: B200-native BEM quadrature, H2 matrix-vector product and GMRES behind H2Lib's API.

The compute path is the CUDA library libh2b200.so (sm_100a) reached through its C ABI
(include/h2b200.h); this package holds the ctypes binding and a Python mirror of the H2Lib
functions the path replaces (h2lib_b200.bem3d).
"""
from ._lib import LIBPATH, H2BError, last_error, lib  # noqa: F401
from . import bem3d  # noqa: F401

__version__ = "0.1.0"
