"""Interface dump and reload on the GPU path: the reference's -iomode output /
input (SPGrid_Domain_Decomposition_Solver.h:121-161 of the CPU demo).

* a solver set up from the dump another solver wrote holds the same interface
  matrices and gives the same PCG iterations and the same solution, bit for bit;
* a dump that does not fit the domain is refused with HDD_ERR_INVALID_ARGUMENT,
  a missing one with HDD_ERR_IO.
"""
import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from hierarchicaldd_b200._lib import HddError
from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver

pytestmark = pytest.mark.gpu


def setup(d, **kw):
    m = d.meta
    s = SPGrid_Domain_Decomposition_Solver()
    s.Set_Domain(d.flags, d.rhs)
    try:
        s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"], **kw)
    except Exception:
        s.close()
        raise
    return s


def matrices(s, M, nsub):
    out = {}
    for l in range(M):
        out[("Arr", l, 0)] = s.Interface_Matrix("Arr", l)
        if l + 1 < M:
            out[("Prr", l, 0)] = s.Interface_Matrix("Prr", l)
        for sd in range(nsub):
            out[("Aii", l, sd)] = s.Interface_Matrix("Aii", l, sd)
            out[("Air", l, sd)] = s.Interface_Matrix("Air", l, sd)
    return out


def test_reload_gives_the_same_solve(tmp_path):
    d = domains.small(32, 8, 6, seed=5)
    M, nsub = d.meta["sigma_levels"], 4 ** 3
    a = setup(d, iomode="output", dump_directory=str(tmp_path))
    try:
        ra, xa = a.Solve(), a.Solution()
        ma, mapa = matrices(a, M, nsub), a.Interface_Map()
    finally:
        a.close()
    assert (tmp_path / "levels").exists() and (tmp_path / "Arr_0").exists()
    b = setup(d, iomode="input", dump_directory=str(tmp_path))
    try:
        rb, xb = b.Solve(), b.Solution()
        mb, mapb = matrices(b, M, nsub), b.Interface_Map()
    finally:
        b.close()
    assert np.array_equal(mapa, mapb)
    for k, A in ma.items():
        B = mb[k]
        assert A.shape == B.shape and (A != B).nnz == 0, k
    assert ra["converged"] == 1 and ra["iterations"] == rb["iterations"]
    assert np.array_equal(xa, xb)


def test_reload_refuses_a_dump_that_does_not_fit(tmp_path):
    d = domains.small(32, 8, 6, seed=5)
    setup(d, iomode="output", dump_directory=str(tmp_path)).close()
    # 8 subdomains of 16^3 instead of the dump's 64 of 8^3.
    with pytest.raises(HddError) as e:
        setup(domains.small(32, 16, 5, seed=5), iomode="input", dump_directory=str(tmp_path)).close()
    assert e.value.status == 1 and "subdomains" in str(e.value)
    with pytest.raises(HddError) as e:
        setup(d, iomode="input", dump_directory=str(tmp_path / "missing")).close()
    assert e.value.status == 9
