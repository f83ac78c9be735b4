"""ctypes binding of the C ABI in include/hdd.h (libhdd_b200.so, built in-tree).

There is no CPU fallback: if the library is missing or cannot be loaded the
import fails with the reason.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhdd_b200.so")

HDD_OK = 0
STATUS_NAMES = {
    0: "HDD_OK", 1: "HDD_ERR_INVALID_ARGUMENT", 2: "HDD_ERR_CUDA", 3: "HDD_ERR_OUT_OF_MEMORY",
    4: "HDD_ERR_NOT_INITIALIZED", 5: "HDD_ERR_UNSUPPORTED", 6: "HDD_ERR_NOT_CONVERGED",
    7: "HDD_ERR_BREAKDOWN", 8: "HDD_ERR_TIMEOUT", 9: "HDD_ERR_IO", 10: "HDD_ERR_BUSY",
    11: "HDD_ERR_NOT_FOUND", 12: "HDD_ERR_INTERNAL",
}
PRECISION_REFERENCE = 0
PRECISION_MIXED = 1
COARSE_REFERENCE = 0
COARSE_EXACT = 1
# Initialize_Preconditioner's iomode (reference Test_Bench -iomode).
IOMODES = {"neither": 0, "output": 1, "input": 2}


class hdd_options(C.Structure):
    _fields_ = [
        ("size", C.c_int * 3), ("sub_size", C.c_int * 3), ("vlevels", C.c_int), ("nVcycles", C.c_int),
        ("interior_smoothing", C.c_int), ("boundary_smoothing", C.c_int), ("sigma_levels", C.c_int),
        ("sigma_smoothing", C.c_int), ("sigma_mg", C.c_int), ("tol", C.c_double), ("relative_tol", C.c_int),
        ("max_iters", C.c_int), ("min_iters", C.c_int), ("precision_mode", C.c_int),
        ("true_residual_every", C.c_int), ("device", C.c_int), ("coarse_solve", C.c_int),
        ("solve_share", C.c_int), ("multilevel", C.c_int),
    ]


class hdd_result(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("converged", C.c_int), ("final_norm", C.c_double), ("b_inf", C.c_double),
        ("true_residual_inf", C.c_double), ("true_residual_l2", C.c_double), ("solve_ms", C.c_double),
        ("setup_ms", C.c_double),
    ]


class HddError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class hdd_server_options(C.Structure):
    _fields_ = [("slots", C.c_int), ("hbm_budget_bytes", C.c_longlong), ("device", C.c_int),
                ("setup_threads", C.c_int), ("batch", C.c_int)]


# Every symbol declared in include/hdd.h: name -> (restype, argtypes).
_vp = C.c_void_p
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
SIGNATURES = {
    "hdd_options_default": (None, [C.POINTER(hdd_options)]),
    "hdd_create": (C.c_int, [C.POINTER(hdd_options), C.POINTER(C.c_void_p)]),
    "hdd_set_domain_dense": (C.c_int, [_vp, C.POINTER(C.c_uint32), _fp]),
    "hdd_velocity_divergence_dense": (C.c_int, [_vp, C.POINTER(C.c_uint32), _fp, _fp, _fp, C.c_float,
                                                C.POINTER(C.c_uint32), _fp]),
    "hdd_set_domain_velocity_dense": (C.c_int, [_vp, C.POINTER(C.c_uint32), _fp, _fp, _fp, C.c_float]),
    "hdd_load_spgrid_dir": (C.c_int, [_vp, C.c_char_p]),
    "hdd_set_domain_pages": (C.c_int, [_vp, C.c_longlong, _ip, C.POINTER(C.c_uint32), _fp]),
    "hdd_set_rhs_pages": (C.c_int, [_vp, C.c_longlong, _ip, _fp]),
    "hdd_get_solution_pages": (C.c_int, [_vp, C.c_longlong, _ip, _fp]),
    "hdd_set_iomode": (C.c_int, [_vp, C.c_int, C.c_char_p]),
    "hdd_initialize_preconditioner": (C.c_int, [_vp]),
    "hdd_set_rhs_dense": (C.c_int, [_vp, _fp]),
    "hdd_solve": (C.c_int, [_vp, C.POINTER(hdd_result)]),
    "hdd_get_solution_dense": (C.c_int, [_vp, _fp]),
    "hdd_get_solution_dense_f64": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "hdd_get_residual_history": (C.c_int, [_vp, C.POINTER(C.c_double), C.c_int, _ip]),
    "hdd_apply_preconditioner_dense": (C.c_int, [_vp, _fp, _fp]),
    "hdd_vcycle_dense": (C.c_int, [_vp, _fp, _fp, C.c_int]),
    "hdd_multiply_dense": (C.c_int, [_vp, _fp, _fp]),
    "hdd_multiply_dot_dense_device_noalloc": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "hdd_sigma_vcycle": (C.c_int, [_vp, _fp, _fp]),
    "hdd_interface_solve": (C.c_int, [_vp, C.c_int, C.c_int, _fp, _fp, _ip]),
    "hdd_interface_solve_batch": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _fp, _fp, _ip]),
    "hdd_interface_size": (C.c_int, [_vp, C.c_int, _ip]),
    "hdd_interface_map": (C.c_int, [_vp, _ip]),
    "hdd_interface_matrix": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _ip, _ip,
                                       C.POINTER(C.c_double)]),
    "hdd_kernel_launch_count": (C.c_int, [_vp, C.POINTER(C.c_longlong)]),
    "hdd_get_pcg_coefficients": (C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, _ip]),
    "hdd_set_wait_limit": (C.c_int, [_vp, C.c_longlong]),
    "hdd_test_stall_dependency": (C.c_int, [_vp, C.c_int]),
    "hdd_get_setup_timing": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "hdd_set_kernel_timing": (C.c_int, [_vp, C.c_int]),
    "hdd_get_kernel_timing": (C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    "hdd_get_kernel_bytes": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "hdd_status_string": (C.c_char_p, [C.c_int]),
    "hdd_last_error": (C.c_char_p, [_vp]),
    "hdd_destroy": (None, [_vp]),
    "hdd_server_options_default": (None, [C.POINTER(hdd_server_options)]),
    "hdd_server_create": (C.c_int, [C.POINTER(hdd_server_options), C.POINTER(C.c_void_p)]),
    "hdd_server_add_domain": (C.c_int, [_vp, C.POINTER(hdd_options), C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_longlong)]),
    "hdd_server_domain_status": (C.c_int, [_vp, C.c_longlong, C.c_int]),
    "hdd_server_domain_error": (C.c_int, [_vp, C.c_longlong, C.c_char_p, C.c_int]),
    "hdd_server_submit": (C.c_int, [_vp, C.c_longlong, _fp, C.POINTER(C.c_longlong)]),
    "hdd_server_poll": (C.c_int, [_vp, C.c_longlong, C.c_int, C.POINTER(hdd_result), _fp,
                                  C.POINTER(C.c_double)]),
    "hdd_server_remove_domain": (C.c_int, [_vp, C.c_longlong]),
    "hdd_server_memory": (C.c_int, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "hdd_server_destroy": (None, [_vp]),
}

_lib = None


def load():
    """Load libhdd_b200.so (raises OSError with the reason if it cannot)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing; build it with `python -m hierarchicaldd_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
