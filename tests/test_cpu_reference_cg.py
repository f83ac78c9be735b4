"""The oracle's PCG loop pinned to the reference's own: PhysBAM's
CONJUGATE_GRADIENT<float>::Solve (PB/Public_Library/PhysBAM_Tools/Krylov_Solvers/
CONJUGATE_GRADIENT.cpp:22-67, the loop the demo's CONJUGATE_GRADIENT_DUMPING runs with
visualisation added, CPU/SPGrid_Domain_Decomposition_Solver/CONJUGATE_GRADIENT_DUMPING.cpp:146-205)
with KRYLOV_SYSTEM_BASE::Precondition and the demo's CG_VECTOR, compiled from the
reference tree by oracle/Makefile.ref into oracle/_ref/libref_cg.so (driver:
oracle/ref_cg.cpp).  The driver's operator is the reference's SPGrid_Laplace; its
preconditioner is the oracle's own (the reference's needs MKL PARDISO), handed over as a
function pointer, so what is compared is the recurrence: the stopping rule, the
rho / beta / alpha sequence, the projections, the FP32 vector updates and the FP64
inner products.  Iteration counts, the convergence norm at every iteration and the
solutions equal the oracle's hddo_solve bit for bit;
the GPU path's iteration parity with the oracle is tested in tests/test_gpu_parity.py
and test_gpu_c2_parity.py.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from hierarchicaldd_b200 import domains
from hierarchicaldd_b200.domains import ACTIVE, INTERFACE
from oracle_ffi import Oracle, lib as oracle_lib

REF_CG_SO = os.path.join(ROOT, "oracle", "_ref", "libref_cg.so")


@pytest.fixture(scope="module")
def refcg():
    tree = os.environ.get("HDD_REFERENCE_ROOT")
    if tree and os.path.isdir(tree):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-f", "Makefile.ref", "REF=" + tree],
                       check=True)
    if not os.path.exists(REF_CG_SO):
        pytest.skip("oracle/_ref/libref_cg.so not built (needs the reference tree, HDD_REFERENCE_ROOT)")
    L = C.CDLL(REF_CG_SO)
    L.refcg_solve.restype = C.c_int
    L.refcg_solve.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_uint32), C.POINTER(C.c_float),
                              C.POINTER(C.c_float), C.c_float, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                              C.POINTER(C.c_double), C.c_int]
    return L


def ref_solve(L, o, flags0, b, tol, max_it):
    """PhysBAM's CG over flags0 with the oracle o's preconditioner:
    (x, iterations or -1, convergence-norm history)."""
    size = flags0.shape
    f = np.ascontiguousarray(flags0, np.uint32)
    b = np.ascontiguousarray(b, np.float32)
    x = np.zeros(size, np.float32)
    hist = np.zeros(max_it + 1, np.float64)
    pre = C.cast(oracle_lib().hddo_apply_preconditioner, C.c_void_p)
    it = L.refcg_solve((C.c_int * 3)(*size), f.ctypes.data_as(C.POINTER(C.c_uint32)),
                       b.ctypes.data_as(C.POINTER(C.c_float)), x.ctypes.data_as(C.POINTER(C.c_float)),
                       float(tol), 0, max_it, pre, C.c_void_p(o.h), hist.ctypes.data_as(C.POINTER(C.c_double)),
                       max_it + 1)
    return x, it, hist


CASES = [("sphere 32^3, sub 8", lambda: domains.small(32, 8, 6, seed=1), 8, False),
         ("ragged 40x36x44, sub 8", lambda: domains.small((40, 36, 44), 8, 6, seed=4), 8, False),
         ("sphere 48^3, sub 16", lambda: domains.small(48, 16, 8, seed=7), 16, False),
         ("generator bubble 35^3, sub 8", lambda: domains.reference_generator((35, 35, 35), (4, 16, 16)), 8, False),
         ("two-level sphere 32^3, sub 16", lambda: domains.small(32, 16, 6, seed=2), 16, True)]


def test_reference_cg_equals_oracle_pcg_on_the_64cube_workload(refcg):
    """The 64^3 sub-16 workload at its own settings and right-hand side (a unit
    point source), relative stop at 1e-6 expressed as PhysBAM's absolute one."""
    d = domains.config1()
    m = d.meta
    o = Oracle(d.size, d.sub_size, d.flags, vlevels=m["vlevels"], nVcycles=m["nVcycles"],
               interior_smoothing=m["interior_smoothing"], boundary_smoothing=m["boundary_smoothing"],
               sigma_levels=m["sigma_levels"], sigma_smoothing=m["sigma_smoothing"], sigma_mg=m["sigma_mg"])
    f0 = o.level_flags(0)
    b = np.where((f0 & (ACTIVE | INTERFACE)) != 0, d.rhs, 0).astype(np.float32)
    tol = float(np.float32(1e-6 * float(np.abs(b).max())))
    x_o, it_o, info = o.solve(b, tol=tol, relative=False, max_it=200)
    x_r, it_r, hist_r = ref_solve(refcg, o, f0, b, tol, 200)
    assert it_r == it_o and 0 < it_o < 200, (it_r, it_o)
    assert np.array_equal(hist_r[:it_r + 1], info["history"][:it_o + 1])
    assert np.array_equal(x_r.view(np.uint32), x_o.view(np.uint32))


@pytest.mark.parametrize("name,make,sub,multilevel", CASES, ids=[c[0] for c in CASES])
def test_reference_cg_equals_oracle_pcg(refcg, name, make, sub, multilevel):
    d = make()
    o = Oracle(d.size, (sub,) * 3, d.flags, vlevels=3, nVcycles=1, interior_smoothing=1, boundary_smoothing=3,
               sigma_levels=2, sigma_smoothing=3, sigma_mg=1, multilevel=multilevel)
    f0 = o.level_flags(0)
    rng = np.random.default_rng(3)
    b = np.where((f0 & (ACTIVE | INTERFACE)) != 0, rng.uniform(-1, 1, d.size), 0).astype(np.float32)
    # The demo's stop test is absolute (Solve(..., 1e-5, 0, 5000)).
    tol = 1e-5
    max_it = 200
    x_o, it_o, info = o.solve(b, tol=tol, relative=False, max_it=max_it)
    x_r, it_r, hist_r = ref_solve(refcg, o, f0, b, tol, max_it)
    assert it_r == it_o, (name, it_r, it_o)
    assert it_o < max_it, name
    # Bit for bit: the convergence norm at every iteration and the solution.
    assert np.array_equal(hist_r[:it_r + 1], info["history"][:it_o + 1]), name
    assert np.array_equal(x_r.view(np.uint32), x_o.view(np.uint32)), name
