"""Edge cases of the CUDA path (through the C ABI) against the CPU oracle.

* ragged domains: (size - 1) not a multiple of the subdomain size on some axes,
  so the last subdomains and tiles are partial (Domain_Divider's
  ceil((size - 1) / sub) subdomains per axis, SPGrid_Domain_Divider_Helper.h:31-35);
* a domain inside one subdomain: no interface, so the preconditioner is the two
  subdomain V-cycle passes alone;
* a zero right-hand side: converged before the first iteration with x = 0
  (CONJUGATE_GRADIENT.cpp:40-42 tests the residual before iterating);
* a domain without Active cells: rejected with HDD_ERR_INVALID_ARGUMENT.
"""
import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from hierarchicaldd_b200.domains import ACTIVE, INTERFACE
from test_gpu_parity import PRECOND_RTOL, make_pair, rel_inf

pytestmark = pytest.mark.gpu


def random_fields(d, o, seed):
    rng = np.random.default_rng(seed)
    f0 = o.level_flags(0)
    u = rng.standard_normal(d.size).astype(np.float32)
    u[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
    b = rng.standard_normal(d.size).astype(np.float32)
    b[(f0 & ACTIVE) == 0] = 0
    return u, b


@pytest.mark.parametrize("cells,sub,radius", [((40, 36, 44), 8, 6), ((33, 40, 40), 8, 5), ((48, 40, 56), 16, 7)])
def test_ragged_domain(cells, sub, radius):
    d = domains.small(cells, sub, radius, seed=11)
    s, o = make_pair(d)
    try:
        u, b = random_fields(d, o, 12)
        x = np.where((o.level_flags(0) & (ACTIVE | INTERFACE)) != 0, u, 0).astype(np.float32)
        assert np.array_equal(s.Multiply(x), o.multiply(x))
        ug = s.V_Cycle(u, b, 1)
        uo, _ = o.vcycle(u, np.zeros_like(u), b)
        assert np.array_equal(ug, uo), np.max(np.abs(ug - uo))
        r = b.copy()
        assert rel_inf(s.Apply_Preconditioner(r), o.apply_preconditioner(r)) < PRECOND_RTOL
        res = s.Solve()
        xg = s.Solution()
    finally:
        s.close()
    xo, it_o, _ = o.solve(d.rhs, tol=1e-6)
    assert res["converged"] == 1 and abs(res["iterations"] - it_o) <= 1, (res["iterations"], it_o)
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) < 1e-5


def test_single_subdomain_without_interface():
    d = domains.small(16, 16, 3, seed=1)
    s, o = make_pair(d)
    try:
        assert s.Interface_Size(0) == 0 and o.num_interface(0) == 0
        _, r = random_fields(d, o, 13)
        assert rel_inf(s.Apply_Preconditioner(r), o.apply_preconditioner(r)) < PRECOND_RTOL
        res = s.Solve()
        xg = s.Solution()
    finally:
        s.close()
    xo, it_o, _ = o.solve(d.rhs, tol=1e-6)
    assert res["converged"] == 1 and abs(res["iterations"] - it_o) <= 1, (res["iterations"], it_o)
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) < 1e-5


def test_zero_rhs_converges_immediately():
    d = domains.small(32, 8, 6, seed=1)
    s, _ = make_pair(d)
    try:
        s.Set_RHS(np.zeros(d.size, np.float32))
        res = s.Solve()
        assert res["converged"] == 1 and res["iterations"] == 0
        assert not np.any(s.Solution())
    finally:
        s.close()


def test_domain_without_active_cells_is_rejected():
    from hierarchicaldd_b200._lib import HddError
    d = domains.small(16, 8, 0, seed=1)
    d.flags[:] = 0
    d.rhs[:] = 0
    with pytest.raises(HddError) as e:
        s, _ = make_pair(d)
        s.close()
    assert e.value.status == 1 and "no Active cells" in str(e.value)
