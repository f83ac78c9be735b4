"""The supernodal solve kernels (the GPU stand-in for the reference's PARDISO
phase-33 solves in SIGMA_SMOOTHER::Smooth) against the host reference of the
same plan (tests/host_shim.cpp; PlanHost::emulate in sn_plan.cpp): the same
FP32 blocks Fw = [L_JJ^{-1}; -L_RJ L_JJ^{-1}], FP64 accumulation, FP64
vectors between fronts.  The two differ only in the order of FP64 sums, so
after the final rounding to FP32 they agree to within a float ulp or two; the
tolerance is 4e-7 of the solution's max-norm.  The host reference itself is
checked against the FP64 factorisation on the CPU
(test_cpu_host.py::test_solve_plan_walk_matches_the_factorisation).
"""
import ctypes as C

import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from shim_ffi import load_shim

pytestmark = pytest.mark.gpu

RTOL = 4e-7


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


@pytest.mark.parametrize("n,sub,radius,levels", [(32, 8, 6, 2), (64, 16, 12, 3), ((40, 36, 44), 8, 6, 2),
                                                 (96, 32, 20, 3)])
def test_gpu_plan_solves_match_the_host_reference(n, sub, radius, levels):
    from hierarchicaldd_b200 import _lib
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    d = domains.small(n, sub, radius, seed=4)
    m = dict(d.meta)
    shim = load_shim()
    size = (C.c_int * 3)(*d.size)
    sb = (C.c_int * 3)(*d.sub_size)
    flags = np.ascontiguousarray(d.flags, np.uint32)
    err = C.create_string_buffer(512)
    h = shim.shim_build(size, sb, m["vlevels"], levels, flags.ctypes.data_as(C.POINTER(C.c_uint32)), err, 512)
    assert h, err.value
    s = SPGrid_Domain_Decomposition_Solver()
    lib = _lib.load()
    rng = np.random.default_rng(5)
    try:
        s.Set_Domain(d.flags, d.rhs)
        s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, levels, m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"])
        checked = 0
        for level in range(levels):
            for kind in (0, 1):
                nn = C.c_int()
                assert lib.hdd_interface_solve(s.h, kind, level, None, None, C.byref(nn)) == 0
                if nn.value == 0:
                    continue
                b = rng.uniform(-1, 1, nn.value).astype(np.float32)
                x = np.zeros(nn.value, np.float32)
                st = lib.hdd_interface_solve(s.h, kind, level, _fp(b), _fp(x), C.byref(nn))
                if st == 5 and level == levels - 1:
                    continue  # coarsest level solved as a whole: no separate plans
                assert st == 0, lib.hdd_last_error(s.h)
                xe = np.zeros(nn.value, np.float32)
                assert shim.shim_plan_emulate(h, kind, level, _fp(b), _fp(xe)) == 0
                diff = float(np.max(np.abs(x.astype(np.float64) - xe)))
                assert diff <= RTOL * float(np.max(np.abs(xe))), (level, kind, diff)
                checked += 1
        assert checked >= 2 * (levels - 1)
    finally:
        s.close()
        shim.shim_free(h)


@pytest.mark.parametrize("n,sub,radius,levels", [(64, 16, 12, 3), (96, 32, 20, 3)])
def test_batched_plan_solves_equal_single_solves(n, sub, radius, levels):
    # 2 and 4 right-hand sides in one launch pair: every solution bit for bit
    # the solve of its right-hand side alone.
    from hierarchicaldd_b200 import _lib
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    d = domains.small(n, sub, radius, seed=6)
    m = dict(d.meta)
    s = SPGrid_Domain_Decomposition_Solver()
    lib = _lib.load()
    rng = np.random.default_rng(7)
    try:
        s.Set_Domain(d.flags, d.rhs)
        s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, levels, m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"])
        checked = 0
        for level in range(levels):
            for kind in (0, 1):
                nn = C.c_int()
                assert lib.hdd_interface_solve(s.h, kind, level, None, None, C.byref(nn)) == 0
                if nn.value == 0:
                    continue
                bs = rng.uniform(-1, 1, (4, nn.value)).astype(np.float32)
                singles = []
                for k in range(4):
                    x = np.zeros(nn.value, np.float32)
                    st = lib.hdd_interface_solve(s.h, kind, level, _fp(bs[k]), _fp(x), C.byref(nn))
                    singles.append((st, x))
                if singles[0][0] == 5:
                    continue  # coarsest level solved as a whole
                assert all(st == 0 for st, _ in singles)
                for nrhs in (1, 2, 4):
                    xb = np.zeros((nrhs, nn.value), np.float32)
                    bb = np.ascontiguousarray(bs[:nrhs])
                    st = lib.hdd_interface_solve_batch(s.h, kind, level, nrhs, _fp(bb), _fp(xb), C.byref(nn))
                    assert st == 0, (level, kind, nrhs, st)
                    for k in range(nrhs):
                        assert np.array_equal(xb[k], singles[k][1]), (level, kind, nrhs, k)
                checked += 1
        assert checked >= 2
    finally:
        s.close()
