"""The velocity -> divergence right-hand side on the GPU (the reference
Test_Bench's "velocity" mode on a uniform grid, hdd_velocity_divergence_dense
and hdd_set_domain_velocity_dense), against the oracle:

* the converted flags and the right-hand side bit for bit (the float rounding
  of each double step is the reference's), on random face velocities, random
  fluid flags (Interior, Ghost, Dirichlet, Active and face-valid bits set at
  random) and a ragged grid;
* a solve of a sphere domain given as fluid flags and face velocities: PCG
  iterations within +-1 of the oracle's on the oracle's converted domain.
"""
import ctypes as C

import numpy as np
import pytest

from hierarchicaldd_b200 import _lib, domains
from oracle_ffi import Oracle, velocity_divergence
from velocity_cases import face_velocities, fluid_flags

pytestmark = pytest.mark.gpu


def _solver(size):
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    lib = _lib.load()
    o = _lib.hdd_options()
    lib.hdd_options_default(C.byref(o))
    for a in range(3):
        o.size[a] = size[a]
        o.sub_size[a] = 8
    h = C.c_void_p()
    assert lib.hdd_create(C.byref(o), C.byref(h)) == 0
    return lib, h


@pytest.mark.parametrize("shape,dx", [((33, 33, 33), 1.0 / 32), ((29, 37, 41), 0.3)])
def test_divergence_matches_oracle(shape, dx):
    rng = np.random.default_rng(5)
    ff = rng.integers(0, 0x80, shape, dtype=np.uint32)  # every combination of the low bits
    u, v, w = face_velocities(shape, 9)
    lib, h = _solver(shape)
    try:
        flags = np.zeros(shape, np.uint32)
        rhs = np.zeros(shape, np.float32)
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        up = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
        assert lib.hdd_velocity_divergence_dense(h, up(ff), fp(u), fp(v), fp(w), dx, up(flags), fp(rhs)) == 0
        fo, ro = velocity_divergence(ff, u, v, w, dx)
        assert np.array_equal(flags, fo)
        assert np.array_equal(rhs.view(np.uint32), ro.view(np.uint32))
        assert lib.hdd_velocity_divergence_dense(h, up(ff), fp(u), fp(v), fp(w), -1.0, up(flags), fp(rhs)) == 1
    finally:
        lib.hdd_destroy(h)


def test_solve_from_velocity():
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    d = domains.small(32, 8, 6, seed=2)
    ff = fluid_flags(d.flags)
    u, v, w = face_velocities(d.size, 3)
    dx = 1.0 / 32
    flags, rhs = velocity_divergence(ff, u, v, w, dx)
    m = d.meta
    s = SPGrid_Domain_Decomposition_Solver()
    try:
        s.Set_Domain_Velocity(ff, u, v, w, dx)
        s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"])
        res = s.Solve()
        o = Oracle(d.size, d.sub_size, flags, vlevels=m["vlevels"], nVcycles=m["nVcycles"],
                   interior_smoothing=m["interior_smoothing"], boundary_smoothing=m["boundary_smoothing"],
                   sigma_levels=m["sigma_levels"], sigma_smoothing=m["sigma_smoothing"], sigma_mg=m["sigma_mg"])
        xo, it_o, _ = o.solve(rhs, tol=1e-6)
        assert res["converged"] == 1
        assert abs(res["iterations"] - it_o) <= 1, (res["iterations"], it_o)
        x = s.Solution()
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-5
    finally:
        s.close()
