"""ctypes binding of the oracle (test infrastructure only).

The oracle is the CPU restatement of the reference's dd_pcg path that the CUDA
product is checked against.  It is loaded only by tests, the smoke check and the
benchmark's CPU-baseline leg.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_DIR = os.path.join(os.path.dirname(_HERE), "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle_hdd.so")
_lib = None


def build_oracle() -> str:
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return ORACLE_SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        vp, ip, up, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_uint32), C.POINTER(C.c_double)
        L.hddo_create.restype = vp
        L.hddo_create.argtypes = [ip, ip, up] + [C.c_int] * 8 + [C.c_char_p, C.c_int]
        L.hddo_create_ml.restype = vp
        L.hddo_create_ml.argtypes = [ip, ip, up] + [C.c_int] * 9 + [C.c_char_p, C.c_int]
        L.hddo_num_second_level.argtypes = [vp]
        L.hddo_second_level_interface.argtypes = [vp, C.c_int]
        L.hddo_velocity_divergence.argtypes = [ip, up, vp, vp, vp, C.c_float, up, vp]
        L.hddo_sl_num_interface.argtypes = [vp, C.c_int, C.c_int]
        L.hddo_sl_interface_map.argtypes = [vp, C.c_int, ip]
        L.hddo_sl_num_subdomains.argtypes = [vp, C.c_int]
        L.hddo_sl_matrix_shape.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, ip]
        L.hddo_sl_matrix_get.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, dp]
        L.hddo_destroy.argtypes = [vp]
        L.hddo_num_levels.argtypes = [vp]
        L.hddo_level_dims.argtypes = [vp, C.c_int, ip]
        L.hddo_level_flags.argtypes = [vp, C.c_int, up]
        L.hddo_num_subdomains.argtypes = [vp]
        L.hddo_num_interface.argtypes = [vp, C.c_int]
        L.hddo_interface_map.argtypes = [vp, ip]
        L.hddo_matrix_shape.argtypes = [vp, C.c_int, C.c_int, C.c_int, ip, ip, ip]
        L.hddo_matrix_get.argtypes = [vp, C.c_int, C.c_int, C.c_int, ip, ip, dp]
        L.hddo_vcycle.argtypes = [vp, vp, vp, vp]
        L.hddo_apply_preconditioner.argtypes = [vp, vp, vp]
        L.hddo_multiply.argtypes = [vp, vp, vp]
        L.hddo_laplace_ri.argtypes = [vp, vp, vp]
        L.hddo_laplace_subdomain.argtypes = [vp, C.c_int, vp, vp]
        L.hddo_sigma_vcycle.argtypes = [vp, vp, vp]
        L.hddo_sigma_smooth.argtypes = [vp, C.c_int, vp, vp]
        L.hddo_solve.restype = C.c_int
        L.hddo_solve.argtypes = [vp, vp, vp, C.c_double, C.c_int, C.c_int, C.c_int, dp, dp, C.c_int]
        try:
            L.hddo_solve_timed.restype = C.c_int
            L.hddo_solve_timed.argtypes = [vp, vp, vp, C.c_double, C.c_int, C.c_int, C.c_int, dp, dp, C.c_int, dp]
        except AttributeError:  # a library built before it existed: solve_timed() raises
            pass
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def velocity_divergence(fluid_flags, u, v, w, dx):
    """The oracle's velocity -> divergence right-hand side and converted flags
    (the Test_Bench "velocity" mode on a uniform grid): (flags, rhs)."""
    ff = np.ascontiguousarray(fluid_flags, np.uint32)
    f32 = [np.ascontiguousarray(a, np.float32) for a in (u, v, w)]
    flags = np.zeros(ff.shape, np.uint32)
    rhs = np.zeros(ff.shape, np.float32)
    size = (C.c_int * 3)(*ff.shape)
    lib().hddo_velocity_divergence(size, _p(ff, C.c_uint32), f32[0].ctypes.data, f32[1].ctypes.data,
                                   f32[2].ctypes.data, float(dx), _p(flags, C.c_uint32), rhs.ctypes.data)
    return flags, rhs


class Oracle:
    """CPU dd_pcg restatement for one domain (float32 or float64 arithmetic)."""

    def __init__(self, size, sub_size, flags, vlevels=3, nVcycles=1, interior_smoothing=1,
                 boundary_smoothing=3, sigma_levels=3, sigma_smoothing=3, sigma_mg=1,
                 dtype=np.float32, multilevel=False):
        L = lib()
        self.size = tuple(int(s) for s in size)
        self.dtype = np.dtype(dtype)
        self.sigma_levels = sigma_levels
        flags = np.ascontiguousarray(flags, np.uint32)
        sz = (C.c_int * 3)(*self.size)
        sb = (C.c_int * 3)(*[int(s) for s in sub_size])
        err = C.create_string_buffer(512)
        self.h = L.hddo_create_ml(sz, sb, _p(flags, C.c_uint32), vlevels, nVcycles, interior_smoothing,
                                  boundary_smoothing, sigma_levels, sigma_smoothing, sigma_mg,
                                  1 if self.dtype == np.float64 else 0, 1 if multilevel else 0, err, 512)
        if not self.h:
            raise RuntimeError("oracle setup failed: " + err.value.decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().hddo_destroy(self.h)
            self.h = None

    def _vec(self, a=None):
        if a is None:
            return np.zeros(self.size, self.dtype)
        return np.ascontiguousarray(a, self.dtype).copy()

    def level_flags(self, l):
        d = (C.c_int * 3)()
        lib().hddo_level_dims(self.h, l, d)
        out = np.zeros(tuple(d), np.uint32)
        lib().hddo_level_flags(self.h, l, _p(out, C.c_uint32))
        return out

    @property
    def num_levels(self):
        return lib().hddo_num_levels(self.h)

    @property
    def num_subdomains(self):
        return lib().hddo_num_subdomains(self.h)

    def num_interface(self, level=0):
        return lib().hddo_num_interface(self.h, level)

    def second_level_sizes(self):
        """Level-0 interface sizes of a two-level solver's per-subdomain systems."""
        return [lib().hddo_second_level_interface(self.h, i) for i in range(lib().hddo_num_second_level(self.h))]

    def second_level_map(self, i):
        """Level-0 interface cells (global) of second-level system i."""
        n = lib().hddo_sl_num_interface(self.h, i, 0)
        out = np.zeros((n, 3), np.int32)
        lib().hddo_sl_interface_map(self.h, i, _p(out, C.c_int))
        return out

    def second_level_matrix(self, i, kind, level, sub=0):
        """Matrix of second-level system i, as matrix()."""
        import scipy.sparse as sp
        k = {"Arr": 0, "Aii": 1, "Air": 2, "Prr": 3}[kind]
        r, c, nnz = C.c_int(), C.c_int(), C.c_int()
        lib().hddo_sl_matrix_shape(self.h, i, k, level, sub, C.byref(r), C.byref(c), C.byref(nnz))
        ptr = np.zeros(r.value + 1, np.int32)
        col = np.zeros(nnz.value, np.int32)
        val = np.zeros(nnz.value, np.float64)
        lib().hddo_sl_matrix_get(self.h, i, k, level, sub, _p(ptr, C.c_int), _p(col, C.c_int), _p(val, C.c_double))
        return sp.csr_matrix((val, col, ptr), shape=(r.value, c.value))

    def interface_map(self):
        n = self.num_interface(0)
        out = np.zeros((n, 3), np.int32)
        lib().hddo_interface_map(self.h, _p(out, C.c_int))
        return out

    def matrix(self, kind, level, sub=0):
        """kind: 'Arr', 'Aii', 'Air' or 'Prr'.  Returns a scipy CSR matrix."""
        import scipy.sparse as sp
        k = {"Arr": 0, "Aii": 1, "Air": 2, "Prr": 3}[kind]
        r, c, nnz = C.c_int(), C.c_int(), C.c_int()
        lib().hddo_matrix_shape(self.h, k, level, sub, C.byref(r), C.byref(c), C.byref(nnz))
        ptr = np.zeros(r.value + 1, np.int32)
        col = np.zeros(nnz.value, np.int32)
        val = np.zeros(nnz.value, np.float64)
        lib().hddo_matrix_get(self.h, k, level, sub, _p(ptr, C.c_int), _p(col, C.c_int), _p(val, C.c_double))
        return sp.csr_matrix((val, col, ptr), shape=(r.value, c.value))

    def vcycle(self, u, r, b):
        u = self._vec(u); r = self._vec(r); b = self._vec(b)
        lib().hddo_vcycle(self.h, u.ctypes.data, r.ctypes.data, b.ctypes.data)
        return u, r

    def laplace_ri(self, u, lu):
        """lu after Laplace_ri(u) (the interface right-hand side step)."""
        u = self._vec(u)
        lu = self._vec(lu)
        lib().hddo_laplace_ri(self.h, u.ctypes.data, lu.ctypes.data)
        return lu

    def laplace_subdomain(self, which, u, lu):
        """lu after Laplace_ri_Subdomain ("ri") or Laplace_ir_Subdomain ("ir") of u."""
        u = self._vec(u)
        lu = self._vec(lu)
        lib().hddo_laplace_subdomain(self.h, {"ri": 0, "ir": 1}[which], u.ctypes.data, lu.ctypes.data)
        return lu

    def apply_preconditioner(self, rhs):
        rhs = self._vec(rhs)
        z = self._vec()
        lib().hddo_apply_preconditioner(self.h, rhs.ctypes.data, z.ctypes.data)
        return z

    def multiply(self, x):
        x = self._vec(x)
        y = self._vec()
        lib().hddo_multiply(self.h, x.ctypes.data, y.ctypes.data)
        return y

    def sigma_vcycle(self, b0):
        b0 = np.ascontiguousarray(b0, self.dtype).copy()
        u0 = np.zeros_like(b0)
        lib().hddo_sigma_vcycle(self.h, b0.ctypes.data, u0.ctypes.data)
        return u0

    def sigma_smooth(self, level, u, b):
        u = np.ascontiguousarray(u, self.dtype).copy()
        b = np.ascontiguousarray(b, self.dtype).copy()
        lib().hddo_sigma_smooth(self.h, level, u.ctypes.data, b.ctypes.data)
        return u

    def solve(self, rhs, tol=1e-6, relative=True, max_it=500, min_it=0):
        """PCG solve.  Returns (x, iterations, info dict)."""
        b = self._vec(rhs)
        x = self._vec()
        norms = np.zeros(5, np.float64)
        hist = np.zeros(max_it + 1, np.float64)
        it = lib().hddo_solve(self.h, b.ctypes.data, x.ctypes.data, tol, 1 if relative else 0, min_it, max_it,
                              _p(norms, C.c_double), _p(hist, C.c_double), max_it + 1)
        info = dict(final_norm=norms[0], b_inf=norms[1], true_res_inf=norms[2], true_res_l2=norms[3],
                    b_l2=norms[4], history=hist[:it + 1].copy())
        return x, it, info

    def solve_timed(self, rhs, tol=1e-6, relative=True, max_it=500, min_it=0):
        """solve() that also returns the wall seconds (from the start of the
        solve) at the end of every PCG iteration: (x, iterations, info, times)."""
        b = self._vec(rhs)
        x = self._vec()
        norms = np.zeros(5, np.float64)
        hist = np.zeros(max_it + 1, np.float64)
        times = np.zeros(max_it + 1, np.float64)
        it = lib().hddo_solve_timed(self.h, b.ctypes.data, x.ctypes.data, tol, 1 if relative else 0, min_it, max_it,
                                    _p(norms, C.c_double), _p(hist, C.c_double), max_it + 1,
                                    _p(times, C.c_double))
        info = dict(final_norm=norms[0], b_inf=norms[1], true_res_inf=norms[2], true_res_l2=norms[3],
                    b_l2=norms[4], history=hist[:it + 1].copy())
        return x, it, info, times[:it].copy()
