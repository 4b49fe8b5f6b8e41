"""Python binding of the solve server (h2b_server_* in include/h2b200.h).

A Server admits Dirichlet BEM solve requests continuously: requests wait in arrival order until
a worker slot is free and their device-memory estimate fits the HBM budget, then run on their
own CUDA streams, overlapping on the device with the other running requests.  Queued Laplace
requests with equal settings are batched: a worker solves them together as one forest H2 matrix
with a batched GMRES (each request keeps its own Krylov space and stop).
"""
import ctypes as C

import numpy as np

from ._lib import HELMHOLTZ, LAPLACE, H2BError, check, checkp, last_error, lib

SOLVE_MIXED = 1


class Request(C.Structure):
    _fields_ = [("vertices", C.c_uint32), ("triangles", C.c_uint32),
                ("x", C.c_void_p), ("t", C.c_void_p), ("pde", C.c_int), ("k", C.c_double),
                ("src", C.c_double * 3), ("eps", C.c_double), ("maxiter", C.c_uint32),
                ("kmax", C.c_uint32), ("flags", C.c_uint32)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_uint32), ("unknowns", C.c_uint32),
                ("rel_residual", C.c_double), ("t_submit", C.c_double), ("t_start", C.c_double),
                ("t_done", C.c_double), ("bytes_reserved", C.c_uint64),
                ("t_setup", C.c_double), ("t_assembly", C.c_double), ("t_rhs", C.c_double),
                ("t_solve", C.c_double)]


class Server:
    def __init__(self, slots=8, hbm_budget=150 << 30, device=0, batching=64):
        """batching: most queued Laplace requests with equal settings one worker solves together
        (one forest H2 matrix, one batched GMRES); 1 solves every request alone."""
        self.handle = checkp(lib.h2b_server_new(device, slots, hbm_budget), "h2b_server_new")
        check(lib.h2b_server_set_batching(self.handle, batching), "server_set_batching")
        self._sizes = {}

    def submit(self, gr, pde, src, k=0.0, eps=1e-8, maxiter=1000, kmax=None, mixed=False):
        """Queue a Laplace (src = point source outside the surface) or Helmholtz (src = unit
        wave direction, wavenumber k) Dirichlet solve on surface `gr`; returns its id."""
        x = np.ascontiguousarray(gr.x, dtype=np.float64)
        t = np.ascontiguousarray(gr.t, dtype=np.uint32)
        r = Request(gr.vertices, gr.triangles, x.ctypes.data, t.ctypes.data, pde, float(k),
                    (C.c_double * 3)(*[float(v) for v in src]), eps, maxiter,
                    kmax if kmax is not None else (80 if pde == HELMHOLTZ else 50),
                    SOLVE_MIXED if mixed else 0)
        rid = lib.h2b_server_submit(self.handle, C.byref(r))
        if rid < 0:
            raise H2BError(f"h2b_server_submit: error {rid}: {last_error()}")
        self._sizes[rid] = 2 * gr.triangles if pde == HELMHOLTZ else gr.vertices
        return rid

    def wait(self, rid):
        """(solution, result) of request rid; blocks until it is done."""
        n = self._sizes.pop(rid)
        out = np.zeros(n)
        res = Result()
        check(lib.h2b_server_wait(self.handle, rid, out.ctypes.data, C.byref(res)),
              f"request {rid}")
        if n and res.unknowns and 2 * res.unknowns == n:
            out = out.view(np.complex128)
        return out, {f: getattr(res, f) for f, _ in Result._fields_}

    def stats(self):
        s = np.zeros(4, dtype=np.uint64)
        check(lib.h2b_server_stats(self.handle, s), "server_stats")
        return dict(queued=int(s[0]), running=int(s[1]), done=int(s[2]), reserved=int(s[3]))

    def close(self):
        if getattr(self, "handle", None):
            lib.h2b_server_del(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass


__all__ = ["Server", "LAPLACE", "HELMHOLTZ", "SOLVE_MIXED"]
