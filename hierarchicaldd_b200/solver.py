"""Host-side mirror of the reference solver API over the C ABI.

``SPGrid_Domain_Decomposition_Solver`` keeps the method names, argument order
and meaning of the reference class
(demos/Domain_Decomposition_CPU_Only/SPGrid_Domain_Decomposition_Solver/
SPGrid_Domain_Decomposition_Solver.h): ``Read_SPGrid``, ``Initialize_Preconditioner``
and ``Solve``.  Errors surface as ``HddError`` carrying the C status code
instead of the reference's ``abort()``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import HddError, hdd_options, hdd_result


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class SPGrid_Domain_Decomposition_Solver:
    def __init__(self, number_of_threads: int = 0, device: int = 0):
        self.lib = _lib.load()
        self.number_of_threads = number_of_threads  # host setup threads come from OpenMP
        self.device = device
        self.h = None
        self.size = None
        self.flags = None
        self.rhs = None
        self.spgrid_dir = None
        self.spgrid_size = None
        self.pages = None
        self.velocity = None
        self.last_result = None
        self.options = None

    # -- domain input --------------------------------------------------------
    def Read_SPGrid(self, base_dir: str):
        """Reference Read_SPGrid: size, block_offset, flags and data files."""
        size = np.fromfile(os.path.join(base_dir, "size"), dtype=np.int32)
        if size.size != 3:
            raise HddError(5, "only 3D SPGrid directories are supported")
        # The file holds the allocator's padded size; the grid size proper is
        # the `size` given to Initialize_Preconditioner (at most this).
        self.spgrid_size = tuple(int(v) for v in size)
        self.size = None
        self.spgrid_dir = base_dir
        self.flags = self.rhs = None
        self.pages = None
        self.velocity = None

    def Set_Domain_Pages(self, page_origin: np.ndarray, flags: np.ndarray, rhs: np.ndarray):
        """SPGrid pages of 4x8x8 cells, as Convert/Copy read them from an SPGrid
        allocator: page_origin (n, 3) cell index of each page's first cell,
        flags / rhs (n, 256) with cell (x, y, z) of a page at (x*8 + y)*8 + z.
        The grid size is the ``size`` given to Initialize_Preconditioner."""
        origin = np.ascontiguousarray(page_origin, np.int32).reshape(-1, 3)
        n = origin.shape[0]
        self.pages = (origin, np.ascontiguousarray(flags, np.uint32).reshape(n, 256),
                      np.ascontiguousarray(rhs, np.float32).reshape(n, 256))
        self.size = None
        self.spgrid_dir = None
        self.flags = self.rhs = None
        self.velocity = None

    def Set_Domain(self, flags: np.ndarray, rhs: np.ndarray):
        """Dense flags (uint32, reference bits) and right-hand side (float32)."""
        self.size = tuple(int(v) for v in flags.shape)
        self.flags = np.ascontiguousarray(flags, np.uint32)
        self.rhs = np.ascontiguousarray(rhs, np.float32)
        self.spgrid_dir = None
        self.pages = None
        self.velocity = None

    def Set_Domain_Velocity(self, fluid_flags: np.ndarray, u: np.ndarray, v: np.ndarray, w: np.ndarray,
                            dx: float):
        """The Test_Bench "velocity" mode on a uniform grid (Test_Bench_3D/main.cpp:317-324):
        the right-hand side is the divergence of the face velocities (u on each
        cell's -x face, v, w likewise) and the flags are converted from the
        SPGrid_Fluids bits, on the GPU when Initialize_Preconditioner loads the
        domain (hdd_set_domain_velocity_dense)."""
        self.size = tuple(int(x) for x in fluid_flags.shape)
        f32 = lambda a: np.ascontiguousarray(a, np.float32)
        self.velocity = (np.ascontiguousarray(fluid_flags, np.uint32), f32(u), f32(v), f32(w), float(dx))
        self.flags = self.rhs = None
        self.spgrid_dir = None
        self.pages = None

    # -- setup ------------------------------------------------------------------
    def Initialize_Preconditioner(self, v_cycle_levels, size, subdomain_size, sigma_levels, nVcycles,
                                  interior_smoothing, boundary_smoothing, sigma_smoothing, n_sigma_mg,
                                  tol=1e-6, relative_tol=True, max_iters=5000, min_iters=0,
                                  precision_mode=_lib.PRECISION_REFERENCE, true_residual_every=20,
                                  iomode="neither", dump_directory="matrices_dump",
                                  coarse_solve=_lib.COARSE_REFERENCE, solve_share=0, multilevel=False):
        """Setup with the reference's arguments (SPGrid_Domain_Decomposition_Solver.h:121).
        ``iomode`` "output" writes the interface matrices to ``dump_directory`` in the
        reference's dump layout, "input" reads them from there instead of assembling
        (the reference defaults to "output"; this mirror to "neither").  ``multilevel``
        is the two-level demo's last argument (Domain_Decomposition_CPU_Only_Two_Levels,
        SPGrid_Domain_Decomposition_Solver.h:124): every subdomain is solved by a DD
        at subdomain_size/2 instead of by V-cycles."""
        if iomode not in _lib.IOMODES:
            raise HddError(1, f"iomode must be one of {sorted(_lib.IOMODES)}, not {iomode!r}")
        o = hdd_options()
        self.lib.hdd_options_default(C.byref(o))
        size = tuple(int(s) for s in (size if np.ndim(size) else (size,) * 3))
        sub = tuple(int(s) for s in (subdomain_size if np.ndim(subdomain_size) else (subdomain_size,) * 3))
        if self.spgrid_dir is not None:
            if any(a > b for a, b in zip(size, self.spgrid_size)):
                raise HddError(1, f"size {size} exceeds the SPGrid directory's size {self.spgrid_size}")
            self.size = tuple(size)
        elif self.pages is not None:
            self.size = tuple(size)
        elif self.size is not None and tuple(size) != tuple(self.size):
            raise HddError(1, f"size {size} differs from the loaded domain {self.size}")
        for a in range(3):
            o.size[a] = size[a]
            o.sub_size[a] = sub[a]
        o.vlevels, o.nVcycles = int(v_cycle_levels), int(nVcycles)
        o.interior_smoothing, o.boundary_smoothing = int(interior_smoothing), int(boundary_smoothing)
        o.sigma_levels, o.sigma_smoothing, o.sigma_mg = int(sigma_levels), int(sigma_smoothing), int(n_sigma_mg)
        o.tol, o.relative_tol = float(tol), 1 if relative_tol else 0
        o.max_iters, o.min_iters = int(max_iters), int(min_iters)
        o.precision_mode, o.true_residual_every = int(precision_mode), int(true_residual_every)
        o.coarse_solve = int(coarse_solve)
        o.solve_share = int(solve_share)
        o.multilevel = 1 if multilevel else 0
        o.device = self.device
        self.options = o
        self.close()
        h = C.c_void_p()
        self._check(self.lib.hdd_create(C.byref(o), C.byref(h)), None)
        self.h = h
        if self.spgrid_dir is not None:
            self._check(self.lib.hdd_load_spgrid_dir(self.h, self.spgrid_dir.encode()))
        elif self.pages is not None:
            origin, flags, rhs = self.pages
            self._check(self.lib.hdd_set_domain_pages(self.h, origin.shape[0], _ip(origin),
                                                      flags.ctypes.data_as(C.POINTER(C.c_uint32)), _fp(rhs)))
        elif self.velocity is not None:
            ff, u, v, w, dx = self.velocity
            self._check(self.lib.hdd_set_domain_velocity_dense(self.h, ff.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                               _fp(u), _fp(v), _fp(w), dx))
        else:
            self._check(self.lib.hdd_set_domain_dense(self.h, self.flags.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                      _fp(self.rhs)))
        self._check(self.lib.hdd_set_iomode(self.h, _lib.IOMODES[iomode], str(dump_directory).encode()))
        self._check(self.lib.hdd_initialize_preconditioner(self.h))

    # -- solve --------------------------------------------------------------------
    def Set_RHS(self, rhs: np.ndarray):
        rhs = np.ascontiguousarray(rhs, np.float32)
        self._check(self.lib.hdd_set_rhs_dense(self.h, _fp(rhs)))

    def Set_RHS_Pages(self, page_origin: np.ndarray, rhs: np.ndarray):
        origin = np.ascontiguousarray(page_origin, np.int32).reshape(-1, 3)
        rhs = np.ascontiguousarray(rhs, np.float32).reshape(origin.shape[0], 256)
        self._check(self.lib.hdd_set_rhs_pages(self.h, origin.shape[0], _ip(origin), _fp(rhs)))

    def Setup_Timing(self) -> dict:
        """Host wall seconds of the last Initialize_Preconditioner by phase."""
        ms = (C.c_double * 4)()
        self._check(self.lib.hdd_get_setup_timing(self.h, ms))
        return {"layout": ms[0] / 1e3, "interface_system": ms[1] / 1e3, "interface_solver": ms[2] / 1e3,
                "total": ms[3] / 1e3}

    def Solve(self, allow_not_converged: bool = False) -> dict:
        res = hdd_result()
        st = self.lib.hdd_solve(self.h, C.byref(res))
        if st != 0 and not (allow_not_converged and st == 6):
            self._check(st)
        self.last_result = {f: getattr(res, f) for f, _ in hdd_result._fields_}
        self.last_result["status"] = st
        return self.last_result

    def Solution_F64(self) -> np.ndarray:
        """The FP64 iterate of the precision form (the FP32 solution widened otherwise)."""
        x = np.zeros(self.size, np.float64)
        self._check(self.lib.hdd_get_solution_dense_f64(self.h, x.ctypes.data_as(C.POINTER(C.c_double))))
        return x

    def Residual_History(self) -> np.ndarray:
        """max|r| at the start of every PCG iteration of the last solve (entry 0: r = b)."""
        n = C.c_int()
        self._check(self.lib.hdd_get_residual_history(self.h, None, 0, C.byref(n)))
        out = np.zeros(n.value, np.float64)
        self._check(self.lib.hdd_get_residual_history(self.h, out.ctypes.data_as(C.POINTER(C.c_double)),
                                                      n.value, C.byref(n)))
        return out

    def PCG_Coefficients(self):
        """(alpha, beta) of every PCG iteration of the last solve (beta[0] = 0)."""
        n = C.c_int()
        dp = C.POINTER(C.c_double)
        self._check(self.lib.hdd_get_pcg_coefficients(self.h, dp(), dp(), 0, C.byref(n)))
        a = np.zeros(n.value, np.float64)
        b = np.zeros(n.value, np.float64)
        self._check(self.lib.hdd_get_pcg_coefficients(self.h, a.ctypes.data_as(dp), b.ctypes.data_as(dp), n.value,
                                                      C.byref(n)))
        return a, b

    def Solution(self) -> np.ndarray:
        x = np.zeros(self.size, np.float32)
        self._check(self.lib.hdd_get_solution_dense(self.h, _fp(x)))
        return x

    def Solution_Pages(self, page_origin: np.ndarray) -> np.ndarray:
        origin = np.ascontiguousarray(page_origin, np.int32).reshape(-1, 3)
        x = np.zeros((origin.shape[0], 256), np.float32)
        self._check(self.lib.hdd_get_solution_pages(self.h, origin.shape[0], _ip(origin), _fp(x)))
        return x

    # -- seams mirroring the reference's internal entry points ---------------------
    def Apply_Preconditioner(self, r: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float32)
        z = np.zeros(self.size, np.float32)
        self._check(self.lib.hdd_apply_preconditioner_dense(self.h, _fp(r), _fp(z)))
        return z

    def V_Cycle(self, u: np.ndarray, b: np.ndarray, n_vcycles: int = 1) -> np.ndarray:
        u = np.ascontiguousarray(u, np.float32).copy()
        b = np.ascontiguousarray(b, np.float32)
        self._check(self.lib.hdd_vcycle_dense(self.h, _fp(u), _fp(b), int(n_vcycles)))
        return u

    def Multiply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros(self.size, np.float32)
        self._check(self.lib.hdd_multiply_dense(self.h, _fp(x), _fp(y)))
        return y

    def Sigma_V_Cycle(self, b0: np.ndarray) -> np.ndarray:
        b0 = np.ascontiguousarray(b0, np.float32)
        u0 = np.zeros_like(b0)
        self._check(self.lib.hdd_sigma_vcycle(self.h, _fp(b0), _fp(u0)))
        return u0

    def Interface_Size(self, level: int = 0) -> int:
        n = C.c_int()
        self._check(self.lib.hdd_interface_size(self.h, level, C.byref(n)))
        return n.value

    def Interface_Map(self) -> np.ndarray:
        n = self.Interface_Size(0)
        out = np.zeros((n, 3), np.int32)
        self._check(self.lib.hdd_interface_map(self.h, out.ctypes.data_as(C.POINTER(C.c_int))))
        return out

    def Interface_Matrix(self, kind: str, level: int, sub: int = 0):
        import scipy.sparse as sp
        k = {"Arr": 0, "Aii": 1, "Air": 2, "Prr": 3}[kind]
        r, c, nnz = C.c_int(), C.c_int(), C.c_int()
        null = C.POINTER(C.c_int)()
        self._check(self.lib.hdd_interface_matrix(self.h, k, level, sub, C.byref(r), C.byref(c), C.byref(nnz),
                                                  null, null, C.POINTER(C.c_double)()))
        ptr = np.zeros(r.value + 1, np.int32)
        col = np.zeros(max(nnz.value, 1), np.int32)
        val = np.zeros(max(nnz.value, 1), np.float64)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        self._check(self.lib.hdd_interface_matrix(self.h, k, level, sub, None, None, None, ip(ptr), ip(col),
                                                  val.ctypes.data_as(C.POINTER(C.c_double))))
        return sp.csr_matrix((val[:nnz.value], col[:nnz.value], ptr), shape=(r.value, c.value))

    def Kernel_Launches(self) -> int:
        n = C.c_longlong()
        self._check(self.lib.hdd_kernel_launch_count(self.h, C.byref(n)))
        return n.value

    # -- lifetime -----------------------------------------------------------------
    def _check(self, st, h="self"):
        if st != 0:
            msg = ""
            if h == "self" and self.h is not None:
                msg = (self.lib.hdd_last_error(self.h) or b"").decode()
            raise HddError(st, msg or (self.lib.hdd_status_string(st) or b"").decode())

    def close(self):
        if self.h is not None:
            self.lib.hdd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
