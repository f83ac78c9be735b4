"""The oracle pinned to the reference's own code: the reference's CPU V-cycle,
V-cycle topology, Flaging, Domain_Divider, CG Laplacian (SPGrid_Laplace),
interface gather (Laplace_ri), the interface hierarchy's adaptive strides
(STRIDE_GENERATOR) and the two-level demo's subdomain couplings
(Laplace_ri_Subdomain, Laplace_ir_Subdomain, oracle/_ref/libref_two_level.so) (CPU/SPGrid_Library/SPGrid_V_Cycle_Helper.h,
SPGrid_V_Cycle_Topology.h, SPGrid_Flag_Helper.h, CPU/SPGrid_Domain_Decomposition_Solver/
SPGrid_Domain_Divider_Helper.h), compiled from the reference tree by
oracle/Makefile.ref into oracle/_ref/libref_vcycle.so (driver: oracle/ref_vcycle.cpp),
give bit for bit the oracle's flags at every V-cycle level and its V-cycle
result, on sphere domains, a ragged grid and the reference generator's own
Neumann-bubble domain (whose coarse levels depend on the order in which the
reference visits the fine cells).  The GPU path is bit-exact against the
oracle on the same operations (tests/test_gpu_parity.py, test_gpu_bubble.py).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from hierarchicaldd_b200 import domains
from hierarchicaldd_b200.domains import ACTIVE, INTERFACE
from oracle_ffi import Oracle

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_vcycle.so")
REF2_SO = os.path.join(ROOT, "oracle", "_ref", "libref_two_level.so")


@pytest.fixture(scope="module")
def ref():
    tree = os.environ.get("HDD_REFERENCE_ROOT")
    if tree and os.path.isdir(tree):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-f", "Makefile.ref", "REF=" + tree],
                       check=True)
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/libref_vcycle.so not built (needs the reference tree, HDD_REFERENCE_ROOT)")
    L = C.CDLL(REF_SO)
    ip, up, fp = C.POINTER(C.c_int), C.POINTER(C.c_uint32), C.POINTER(C.c_float)
    L.refv_vcycle.argtypes = [ip, ip, up, C.c_int, C.c_int, C.c_int, fp, fp, up, fp]
    L.refv_laplace.argtypes = [ip, ip, up, fp, fp, fp, fp]
    L.refv_adaptive_stride.argtypes = [ip, ip, ip]
    return L


def ref_laplace(L, d, sub, u, b):
    lu = np.zeros(d.size, np.float32)
    ri = np.zeros(d.size, np.float32)
    f = np.ascontiguousarray(d.flags, np.uint32)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    L.refv_laplace((C.c_int * 3)(*d.size), (C.c_int * 3)(*sub), f.ctypes.data_as(C.POINTER(C.c_uint32)), fp(u),
                   fp(b), fp(lu), fp(ri))
    return lu, ri


def ref_vcycle(L, d, sub, levels, interior, boundary, u, b):
    sizes, n = [], list(d.size)
    for _ in range(levels):
        sizes.append(tuple(n))
        n = [x // 2 + 1 for x in n]
    lf = np.zeros(sum(int(np.prod(s)) for s in sizes), np.uint32)
    out = np.zeros(d.size, np.float32)
    f = np.ascontiguousarray(d.flags, np.uint32)
    L.refv_vcycle((C.c_int * 3)(*d.size), (C.c_int * 3)(*sub), f.ctypes.data_as(C.POINTER(C.c_uint32)), levels,
                  interior, boundary, u.ctypes.data_as(C.POINTER(C.c_float)), b.ctypes.data_as(C.POINTER(C.c_float)),
                  lf.ctypes.data_as(C.POINTER(C.c_uint32)), out.ctypes.data_as(C.POINTER(C.c_float)))
    levels_out, o = [], 0
    for s in sizes:
        c = int(np.prod(s))
        levels_out.append(lf[o:o + c].reshape(s))
        o += c
    return levels_out, out


CASES = [("sphere 32^3, sub 8", lambda: domains.small(32, 8, 6, seed=1), (8,) * 3, 3, 3),
         ("sphere 48^3, sub 16", lambda: domains.small(48, 16, 8, seed=7), (16,) * 3, 3, 1),
         ("ragged 40x36x44, sub 8", lambda: domains.small((40, 36, 44), 8, 6, seed=4), (8,) * 3, 3, 3),
         ("generator bubble 35^3, sub 8", lambda: domains.reference_generator((35, 35, 35), (4, 16, 16)), (8,) * 3,
          3, 3),
         ("generator bubble 65^3, sub 16", lambda: domains.reference_generator((65, 65, 65), (8, 32, 32)),
          (16,) * 3, 3, 1)]


@pytest.mark.parametrize("name,make,sub,levels,interior", CASES, ids=[c[0] for c in CASES])
def test_reference_vcycle_equals_oracle(ref, name, make, sub, levels, interior):
    d = make()
    o = Oracle(d.size, sub, d.flags, vlevels=levels, nVcycles=1, interior_smoothing=interior, boundary_smoothing=3,
               sigma_levels=2, sigma_smoothing=3, sigma_mg=1)
    f0 = o.level_flags(0)
    rng = np.random.default_rng(3)
    u = rng.standard_normal(d.size).astype(np.float32)
    u[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
    b = rng.standard_normal(d.size).astype(np.float32)
    b[(f0 & ACTIVE) == 0] = 0
    lf, ur = ref_vcycle(ref, d, sub, levels, interior, 3, u, b)
    for l in range(levels):
        assert np.array_equal(lf[l], o.level_flags(l)), (name, l)
    uo, _ = o.vcycle(u, np.zeros_like(u), b)
    assert np.array_equal(ur.view(np.uint32), uo.view(np.uint32)), (name, float(np.max(np.abs(ur - uo))))


@pytest.mark.parametrize("name,make,sub,levels,interior", CASES, ids=[c[0] for c in CASES])
def test_reference_laplacian_and_interface_gather_equal_oracle(ref, name, make, sub, levels, interior):
    """CG_SYSTEM::Multiply's SPGrid_Laplace and Apply_Preconditioner's Laplace_ri."""
    d = make()
    o = Oracle(d.size, sub, d.flags, vlevels=levels, nVcycles=1, interior_smoothing=interior, boundary_smoothing=3,
               sigma_levels=2, sigma_smoothing=3, sigma_mg=1)
    f0 = o.level_flags(0)
    rng = np.random.default_rng(8)
    u = rng.standard_normal(d.size).astype(np.float32)
    u[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
    b = rng.standard_normal(d.size).astype(np.float32)
    lu_ref, ri_ref = ref_laplace(ref, d, sub, u, b)
    assert np.array_equal(o.multiply(u).view(np.uint32), lu_ref.view(np.uint32)), name
    assert np.array_equal(o.laplace_ri(u, b).view(np.uint32), ri_ref.view(np.uint32)), name


@pytest.mark.parametrize("n,sub,radius,kind", [(32, 16, 6, "sphere"), ((40, 36, 44), 16, 6, "sphere"),
                                               (64, 16, 0, "bubble")])
def test_reference_two_level_couplings_equal_oracle(ref, n, sub, radius, kind):
    """The two-level demo's Laplace_ri_Subdomain and Laplace_ir_Subdomain
    (TWO/SPGrid_Library/SPGrid_Laplace_Legacy.h:120-178, 232-290)."""
    if not os.path.exists(REF2_SO):
        pytest.skip("oracle/_ref/libref_two_level.so not built")
    L = C.CDLL(REF2_SO)
    d = (domains.small(n, sub, radius, seed=2) if kind == "sphere"
         else domains.reference_generator((n + 1,) * 3, (8, n // 2, n // 2)))
    s3 = (sub,) * 3
    o = Oracle(d.size, s3, d.flags, vlevels=3, nVcycles=1, interior_smoothing=1, boundary_smoothing=3,
               sigma_levels=2, sigma_smoothing=3, sigma_mg=1, multilevel=True)
    rng = np.random.default_rng(9)
    f0 = o.level_flags(0)
    u = rng.standard_normal(d.size).astype(np.float32)
    u[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
    b = rng.standard_normal(d.size).astype(np.float32)
    ri = np.zeros(d.size, np.float32)
    ir = np.zeros(d.size, np.float32)
    f = np.ascontiguousarray(d.flags, np.uint32)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    L.reft_subdomain_couplings((C.c_int * 3)(*d.size), (C.c_int * 3)(*s3), f.ctypes.data_as(C.POINTER(C.c_uint32)),
                               fp(u), fp(b), fp(ri), fp(ir))
    assert np.array_equal(o.laplace_subdomain("ri", u, b).view(np.uint32), ri.view(np.uint32))
    assert np.array_equal(o.laplace_subdomain("ir", u, np.zeros_like(u)).view(np.uint32), ir.view(np.uint32))


def test_reference_adaptive_stride_equals_oracle(ref):
    """STRIDE_GENERATOR<3>::Generate_Adaptive_Stride (CPU/Interface_Solver/STRIDE_GENERATOR.h:23-54),
    the graded node spacing of the interface hierarchy, against the oracle's restatement for every
    box extent 2..129 and two box origins.  (Extent 1 writes one entry past the array in both.)"""
    from oracle_ffi import lib as oracle_lib
    O = oracle_lib()
    O.hddo_adaptive_stride.restype = C.c_int
    ip = C.POINTER(C.c_int)
    for n in range(2, 130):
        for lo in [(0, 0, 0), (8, 16, 24)]:
            lo3 = (C.c_int * 3)(*lo)
            hi3 = (C.c_int * 3)(*(x + n for x in lo))
            q_o = np.zeros(3 * (n + 1), np.int32)
            q_r = np.zeros_like(q_o)
            filled = (C.c_int * 3)()
            lv_o = O.hddo_adaptive_stride(lo3, hi3, q_o.ctypes.data_as(ip), filled)
            lv_r = ref.refv_adaptive_stride(lo3, hi3, q_r.ctypes.data_as(ip))
            assert list(filled) == [n + 1] * 3, (n, list(filled))
            assert lv_o == lv_r, (n, lo, lv_o, lv_r)
            assert np.array_equal(q_o, q_r), (n, lo)
