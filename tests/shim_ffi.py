"""ctypes binding of the host-code test shim (tests/host_shim.cpp): the CUDA
library's host-side setup sources (layout, interface assembly, supernodal
Cholesky, solve plans) compiled with g++ on their own, for checks that need no
GPU and as a host reference for the GPU tests."""
import ctypes as C
import os
import subprocess

from conftest import ROOT

CSRC = os.path.join(ROOT, "hierarchicaldd_b200", "csrc")
BUILD = os.path.join(ROOT, "hierarchicaldd_b200", "_build")
SHIM = os.path.join(BUILD, "libhost_shim.so")


def load_shim():
    """Build (if stale) and load the host-code test shim."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(ROOT, "tests", "host_shim.cpp")] + [
        os.path.join(CSRC, f) for f in ("host_setup.cpp", "host_interface.cpp", "host_cholesky.cpp", "host_interface_io.cpp",
                                        "sn_plan.cpp")]
    if not os.path.exists(SHIM) or any(os.path.getmtime(f) > os.path.getmtime(SHIM) for f in srcs):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
                        "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                        "-o", SHIM] + srcs, check=True)
    L = C.CDLL(SHIM)
    ip = C.POINTER(C.c_int)
    L.shim_build.restype = C.c_void_p
    L.shim_build.argtypes = [ip, ip, C.c_int, C.c_int, C.POINTER(C.c_uint32), C.c_char_p, C.c_int]
    L.shim_free.argtypes = [C.c_void_p]
    L.shim_build_second_level.restype = C.c_void_p
    L.shim_build_second_level.argtypes = [ip, ip, C.c_int, C.POINTER(C.c_uint32), C.c_char_p, C.c_int]
    L.shim_num_interface.argtypes = [C.c_void_p, C.c_int]
    L.shim_global_vcycle.argtypes = [C.c_void_p]
    L.shim_num_subdomains.argtypes = [C.c_void_p]
    L.shim_matrix_shape.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, ip]
    L.shim_matrix_get.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, ip, ip, C.POINTER(C.c_double)]
    cp = C.c_char_p
    L.shim_write_interface.argtypes = [C.c_void_p, cp, cp, C.c_int]
    L.shim_read_interface.restype = C.c_void_p
    L.shim_read_interface.argtypes = [cp, cp, C.c_int]
    L.shim_check_interface.argtypes = [C.c_void_p, C.c_void_p, C.c_int, cp, C.c_int]
    L.shim_positions.restype = C.c_longlong
    L.shim_positions.argtypes = [C.c_void_p, C.c_int, C.c_int, ip]
    L.shim_interface_map.restype = C.c_longlong
    L.shim_interface_map.argtypes = [C.c_void_p, ip]
    L.shim_pages_to_dense.argtypes = [ip, C.c_longlong, ip, C.POINTER(C.c_uint32), C.POINTER(C.c_float),
                                      C.POINTER(C.c_uint32), C.POINTER(C.c_float), cp, C.c_int]
    L.shim_dense_to_pages.argtypes = [ip, C.c_longlong, ip, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.shim_setup_digest.restype = C.c_ulonglong
    L.shim_setup_digest.argtypes = [C.c_void_p]
    L.shim_factor_components.restype = C.c_double
    L.shim_factor_components.argtypes = [C.c_int, C.c_int]
    L.shim_factor_check.restype = C.c_double
    L.shim_factor_check.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.shim_plan_check.restype = C.c_double
    L.shim_plan_check.argtypes = [C.c_void_p, C.c_int, C.c_int, ip]
    L.shim_plan_emulate.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    return L
