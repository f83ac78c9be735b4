"""The reference generator's own domain (a Neumann bubble: exterior cells
face-adjacent to Active ones, Create_3D_Domain/main.cpp:100-149) on the GPU.

Its exterior region couples neighbouring subdomain boxes at the coarse
V-cycle levels, so the solver runs the whole-grid V-cycle there
(kernels_vcycle_global.cu), as the reference's CPU V-cycle does:

* the V-cycle bit for bit against the oracle's;
* the preconditioner within 1e-4 relative max-norm (the sigma solves' FP32
  rounding), PCG iterations within +-1 of the oracle's, the true residual and
  the solution within 1e-5 relative L2 of the oracle's;
* the same under two-level DD.
"""
import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from hierarchicaldd_b200.domains import ACTIVE, INTERFACE
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu

META = dict(vlevels=3, nVcycles=1, interior_smoothing=3, boundary_smoothing=3, sigma_levels=2, sigma_smoothing=3,
            sigma_mg=1)


def make(d, sub, multilevel=False):
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    m = META
    s = SPGrid_Domain_Decomposition_Solver()
    s.Set_Domain(d.flags, d.rhs)
    s.Initialize_Preconditioner(m["vlevels"], d.size, (sub,) * 3, m["sigma_levels"], m["nVcycles"],
                                m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"], m["sigma_mg"],
                                multilevel=multilevel)
    o = Oracle(d.size, (sub,) * 3, d.flags, multilevel=multilevel, **m)
    return s, o


def rel_inf(a, b):
    return float(np.max(np.abs(a.astype(np.float64) - b)) / max(np.max(np.abs(b)), 1e-30))


@pytest.mark.parametrize("size,sub,delta,multilevel", [((35, 35, 35), 8, (4, 16, 16), False),
                                                      ((65, 65, 65), 16, (8, 32, 32), False),
                                                      ((65, 65, 65), 16, (8, 32, 32), True)])
def test_bubble_domain(size, sub, delta, multilevel):
    d = domains.reference_generator(size, delta)
    assert np.any(d.flags == 0) and d.n_active > 0
    s, o = make(d, sub, multilevel)
    try:
        f0 = o.level_flags(0)
        rng = np.random.default_rng(21)
        u = rng.standard_normal(d.size).astype(np.float32)
        u[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
        b = rng.standard_normal(d.size).astype(np.float32)
        b[(f0 & ACTIVE) == 0] = 0
        ug = s.V_Cycle(u, b, 1)
        uo, _ = o.vcycle(u, np.zeros_like(u), b)
        assert np.array_equal(ug, uo), np.max(np.abs(ug - uo))
        r = rng.standard_normal(d.size).astype(np.float32)
        r[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
        assert rel_inf(s.Apply_Preconditioner(r), o.apply_preconditioner(r)) < 1e-4
        res = s.Solve()
        xo, it_o, info = o.solve(d.rhs, tol=1e-6)
        assert res["converged"] == 1
        assert abs(res["iterations"] - it_o) <= 1, (res["iterations"], it_o)
        assert res["true_residual_inf"] <= max(2e-6, 2 * info["true_res_inf"] / info["b_inf"])
        x = s.Solution()
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-5
    finally:
        s.close()
