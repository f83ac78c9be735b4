"""CPU checks of two-level DD (the reference's -multilevel yes,
demos/Domain_Decomposition_CPU_Only_Two_Levels), no GPU:

* the product stacks all first-level subdomains' second-level interface
  systems (first-level planes made Dirichlet, boxes of sub/2) into one
  block-diagonal system; its blocks equal the oracle's per-subdomain systems
  (SPGrid_Subdomain_Splitter.h:168-193 of that demo) bit for bit at every
  level (Arr, Prr, every box's Aii and Air), and nothing couples two blocks;
* the oracle's two-level PCG converges in FP32 and FP64 and its
  preconditioner is linear.
"""
import ctypes as C

import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from oracle_ffi import Oracle
from shim_ffi import load_shim
from test_cpu_host import matrix


@pytest.fixture(scope="module")
def shim():
    return load_shim()


def _second_level(L, d, M):
    size = (C.c_int * 3)(*d.size)
    sub = (C.c_int * 3)(*d.sub_size)
    flags = np.ascontiguousarray(d.flags, np.uint32)
    err = C.create_string_buffer(512)
    h = L.shim_build_second_level(size, sub, M, flags.ctypes.data_as(C.POINTER(C.c_uint32)), err, 512)
    assert h, err.value
    return h


def _map(L, h):
    n = L.shim_interface_map(h, None)
    out = np.zeros((n, 3), np.int32)
    L.shim_interface_map(h, out.ctypes.data_as(C.POINTER(C.c_int)))
    return out


@pytest.mark.parametrize("n,sub,radius", [(32, 16, 6), ((40, 36, 44), 16, 6), (48, 16, 9)])
def test_second_level_system_is_the_per_subdomain_blocks(shim, n, sub, radius):
    import oracle_ffi
    OL = oracle_ffi.lib()
    d = domains.small(n, sub, radius, seed=7)
    M = 2
    h = _second_level(shim, d, M)
    o = Oracle(d.size, d.sub_size, d.flags, vlevels=3, nVcycles=1, interior_smoothing=1, boundary_smoothing=1,
               sigma_levels=M, sigma_smoothing=3, sigma_mg=1, multilevel=True)
    try:
        nsys = len(o.second_level_sizes())
        assert nsys > 1
        # The product's level-0 interface cells are the systems' cells, stacked.
        assert np.array_equal(_map(shim, h), np.concatenate([o.second_level_map(i) for i in range(nsys)]))
        off = [0] * M          # DOF offset of system i per level
        box = 0                # first box of sub/2 of system i
        for i in range(nsys):
            n_i = [OL.hddo_sl_num_interface(o.h, i, l) for l in range(M)]
            for l in range(M):
                r = slice(off[l], off[l] + n_i[l])
                assert (matrix(shim, h, 0, l)[r, r] != o.second_level_matrix(i, "Arr", l)).nnz == 0, (i, l)
                if l + 1 < M:
                    c = slice(off[l + 1], off[l + 1] + n_i[l + 1])
                    assert (matrix(shim, h, 3, l)[r, c] != o.second_level_matrix(i, "Prr", l)).nnz == 0, (i, l)
                for b in range(OL.hddo_sl_num_subdomains(o.h, i)):
                    assert (matrix(shim, h, 1, l, box + b) != o.second_level_matrix(i, "Aii", l, b)).nnz == 0
                    air = matrix(shim, h, 2, l, box + b)
                    assert air.nnz == air[:, r].nnz
                    assert (air[:, r] != o.second_level_matrix(i, "Air", l, b)).nnz == 0, (i, l, b)
            for l in range(M):
                off[l] += n_i[l]
            box += OL.hddo_sl_num_subdomains(o.h, i)
        for l in range(M):
            assert shim.shim_num_interface(h, l) == off[l]
            # nothing couples two subdomains: the blocks hold every Arr entry
            a = matrix(shim, h, 0, l)
            assert a.nnz == sum(o.second_level_matrix(i, "Arr", l).nnz for i in range(nsys))
        assert shim.shim_num_subdomains(h) == box
    finally:
        shim.shim_free(h)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_two_level_oracle_converges(dtype):
    d = domains.small(32, 16, 6, seed=3)
    m = dict(d.meta, sigma_levels=2)
    o = Oracle(d.size, d.sub_size, d.flags, dtype=dtype, multilevel=True, **m)
    x, it, info = o.solve(d.rhs, tol=1e-6, relative=True, max_it=100)
    assert it < 30
    assert info["true_res_inf"] <= 3e-6 * info["b_inf"]
    z = o.apply_preconditioner(d.rhs)
    assert np.array_equal(o.apply_preconditioner(2 * d.rhs), 2 * z)
    assert np.abs(z).max() > 0
