"""CPU checks of the product's host-side setup (no GPU): the layout, interface
assembly and supernodal Cholesky sources of the CUDA library compiled on their
own into a test shim (tests/host_shim.cpp).

* the interface matrices (Arr, Aii, Air, Prr) equal the oracle's bit for bit;
* the supernodal factorisation solves (A + 1e-5 I) x = b to FP64 accuracy for
  every matrix kind, and its explicit solve blocks [L^-1; -L_RJ L^-1] (what the
  GPU kernels read) give the same solution.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ROOT
from hierarchicaldd_b200 import domains
from oracle_ffi import Oracle

CSRC = os.path.join(ROOT, "hierarchicaldd_b200", "csrc")
BUILD = os.path.join(ROOT, "hierarchicaldd_b200", "_build")
SHIM = os.path.join(BUILD, "libhost_shim.so")


@pytest.fixture(scope="module")
def shim():
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(ROOT, "tests", "host_shim.cpp")] + [
        os.path.join(CSRC, f) for f in ("host_setup.cpp", "host_interface.cpp", "host_cholesky.cpp")]
    if not os.path.exists(SHIM) or any(os.path.getmtime(f) > os.path.getmtime(SHIM) for f in srcs):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
                        "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                        "-o", SHIM] + srcs, check=True)
    L = C.CDLL(SHIM)
    ip = C.POINTER(C.c_int)
    L.shim_build.restype = C.c_void_p
    L.shim_build.argtypes = [ip, ip, C.c_int, C.c_int, C.POINTER(C.c_uint32), C.c_char_p, C.c_int]
    L.shim_free.argtypes = [C.c_void_p]
    L.shim_num_subdomains.argtypes = [C.c_void_p]
    L.shim_matrix_shape.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, ip]
    L.shim_matrix_get.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, ip, ip, C.POINTER(C.c_double)]
    L.shim_factor_check.restype = C.c_double
    L.shim_factor_check.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    return L


def build(L, d, M):
    size = (C.c_int * 3)(*d.size)
    sub = (C.c_int * 3)(*d.sub_size)
    flags = np.ascontiguousarray(d.flags, np.uint32)
    err = C.create_string_buffer(512)
    h = L.shim_build(size, sub, d.meta["vlevels"], M, flags.ctypes.data_as(C.POINTER(C.c_uint32)), err, 512)
    assert h, err.value
    return h


def matrix(L, h, kind, level, sub=0):
    shape = (C.c_int * 3)()
    assert L.shim_matrix_shape(h, kind, level, sub, shape) == 0
    rows, cols, nnz = shape
    ptr = np.zeros(rows + 1, np.int32)
    col = np.zeros(max(nnz, 1), np.int32)
    val = np.zeros(max(nnz, 1), np.float64)
    L.shim_matrix_get(h, kind, level, sub, ptr.ctypes.data_as(C.POINTER(C.c_int)),
                      col.ctypes.data_as(C.POINTER(C.c_int)), val.ctypes.data_as(C.POINTER(C.c_double)))
    return sp.csr_matrix((val[:nnz], col[:nnz], ptr), shape=(rows, cols))


@pytest.mark.parametrize("n,sub,radius", [(32, 8, 6), (32, 16, 5),
                                           # ragged: the last subdomains along y and z (and x) are partial
                                           ((40, 36, 44), 8, 6), ((33, 40, 40), 8, 5), ((48, 40, 56), 16, 7)])
def test_interface_matrices_match_oracle(shim, n, sub, radius):
    d = domains.small(n, sub, radius, seed=4)
    M = d.meta["sigma_levels"]
    h = build(shim, d, M)
    m = d.meta
    o = Oracle(d.size, d.sub_size, d.flags, vlevels=m["vlevels"], nVcycles=1, interior_smoothing=1,
               boundary_smoothing=1, sigma_levels=M, sigma_smoothing=3, sigma_mg=1)
    try:
        for l in range(M):
            kinds = [(0, "Arr", None)] + ([(3, "Prr", None)] if l + 1 < M else [])
            for kind, name, _ in kinds:
                a, b = matrix(shim, h, kind, l), o.matrix(name, l)
                assert a.shape == b.shape and (a != b).nnz == 0, (name, l)
            for sd in range(shim.shim_num_subdomains(h)):
                for kind, name in ((1, "Aii"), (2, "Air")):
                    a, b = matrix(shim, h, kind, l, sd), o.matrix(name, l, sd)
                    assert a.shape == b.shape and (a != b).nnz == 0, (name, l, sd)
    finally:
        shim.shim_free(h)


def test_supernodal_factorisation_solves(shim):
    d = domains.small(32, 8, 6, seed=4)
    M = d.meta["sigma_levels"]
    h = build(shim, d, M)
    try:
        diff = C.c_double()
        for l in range(M):
            res = shim.shim_factor_check(h, 0, l, 0, C.byref(diff))
            assert 0 <= res < 1e-10 and diff.value < 1e-10, ("Arr", l, res, diff.value)
            for sd in range(shim.shim_num_subdomains(h)):
                res = shim.shim_factor_check(h, 1, l, sd, C.byref(diff))
                if res < 0:
                    continue  # no interior DOFs
                assert res < 1e-10 and diff.value < 1e-10, ("Aii", l, sd, res, diff.value)
    finally:
        shim.shim_free(h)


def test_domain_without_active_cells_is_rejected(shim):
    d = domains.small(16, 8, 0, seed=1)
    d.flags[:] = 0
    size = (C.c_int * 3)(*d.size)
    sub = (C.c_int * 3)(*d.sub_size)
    flags = np.ascontiguousarray(d.flags, np.uint32)
    err = C.create_string_buffer(512)
    h = shim.shim_build(size, sub, 3, 2, flags.ctypes.data_as(C.POINTER(C.c_uint32)), err, 512)
    assert not h and b"no Active cells" in err.value


def test_single_subdomain_has_no_level0_interface(shim):
    """A domain inside one subdomain: no level-0 interface DOFs (the solver then
    runs the subdomain V-cycles alone), same as the oracle."""
    d = domains.small(16, 16, 3, seed=1)
    h = build(shim, d, 2)
    try:
        assert shim.shim_num_subdomains(h) == 1
        assert matrix(shim, h, 0, 0).shape == (0, 0)
    finally:
        shim.shim_free(h)
    o = Oracle(d.size, d.sub_size, d.flags, vlevels=3, nVcycles=1, interior_smoothing=3, boundary_smoothing=3,
               sigma_levels=2, sigma_smoothing=3, sigma_mg=1)
    assert o.num_interface(0) == 0
