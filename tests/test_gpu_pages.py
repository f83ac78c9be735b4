"""SPGrid page input on the GPU path (hdd_set_domain_pages, hdd_set_rhs_pages,
hdd_get_solution_pages: the reference's Convert / Copy from an SPGrid
allocator): the same domain given as 4x8x8 pages, in any order, solves to the
same PCG iterations and the same solution, bit for bit, as the dense input."""
import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver

pytestmark = pytest.mark.gpu


def init(s, d):
    m = d.meta
    s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                m["sigma_mg"])


def test_pages_solve_like_the_dense_input():
    d = domains.small((40, 36, 44), 8, 6, seed=7)
    origin, fp, rp = domains.to_pages(d.flags, d.rhs)
    order = np.random.default_rng(1).permutation(len(origin))
    origin, fp, rp = origin[order], fp[order], rp[order]
    rhs2 = np.where((d.flags & domains.ACTIVE) != 0,
                    np.random.default_rng(2).uniform(-1, 1, d.size), 0).astype(np.float32)
    _, _, r2p = domains.to_pages(d.flags, rhs2)
    r2p = r2p[order]
    a = SPGrid_Domain_Decomposition_Solver()
    b = SPGrid_Domain_Decomposition_Solver()
    try:
        a.Set_Domain(d.flags, d.rhs)
        init(a, d)
        b.Set_Domain_Pages(origin, fp, rp)
        init(b, d)
        ra, rb = a.Solve(), b.Solve()
        xa = a.Solution()
        assert ra["iterations"] == rb["iterations"]
        assert np.array_equal(xa, b.Solution())
        _, _, xa_pages = domains.to_pages(d.flags, xa)
        assert np.array_equal(b.Solution_Pages(origin), xa_pages[order])
        a.Set_RHS(rhs2)
        b.Set_RHS_Pages(origin, r2p)
        ra, rb = a.Solve(), b.Solve()
        assert ra["iterations"] == rb["iterations"]
        assert np.array_equal(a.Solution(), b.Solution())
    finally:
        a.close()
        b.close()
