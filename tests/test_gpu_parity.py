"""Parity of the CUDA path (through the C ABI) against the CPU oracle.

* Laplacian, V-cycle and interface gathers follow the reference's float
  operation order exactly, so they are compared bit for bit.
* The interface matrices are assembled in the same order as the oracle and
  compared bit for bit.
* Sparse Cholesky solves differ from the oracle's FP64 solves by float
  rounding, so the sigma V-cycle and the full preconditioner are compared with
  a relative max-norm tolerance of 1e-4 (FP32 rounding through ~200 dependent
  triangular solves), and PCG by iteration count (+-1) and residual.
"""
import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from hierarchicaldd_b200.domains import ACTIVE, INTERFACE
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu

PRECOND_RTOL = 1e-4


def make_pair(d, **over):
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    m = dict(d.meta)
    m.update(over)
    s = SPGrid_Domain_Decomposition_Solver()
    s.Set_Domain(d.flags, d.rhs)
    s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                m["sigma_mg"])
    o = Oracle(d.size, d.sub_size, d.flags, vlevels=m["vlevels"], nVcycles=m["nVcycles"],
               interior_smoothing=m["interior_smoothing"], boundary_smoothing=m["boundary_smoothing"],
               sigma_levels=m["sigma_levels"], sigma_smoothing=m["sigma_smoothing"], sigma_mg=m["sigma_mg"])
    return s, o


@pytest.fixture(scope="module")
def small_pair():
    d = domains.small(32, 8, 6, seed=1)
    s, o = make_pair(d)
    yield d, s, o
    s.close()


def rel_inf(a, b):
    return float(np.max(np.abs(a.astype(np.float64) - b)) / max(np.max(np.abs(b)), 1e-30))


def test_multiply_bitexact(small_pair):
    d, s, o = small_pair
    rng = np.random.default_rng(3)
    x = rng.standard_normal(d.size).astype(np.float32)
    x[(d.flags & ACTIVE) == 0] = 0  # Dirichlet/exterior carry zero
    o_flags = o.level_flags(0)
    x[(o_flags & (ACTIVE | INTERFACE)) == 0] = 0
    y = s.Multiply(x)
    yo = o.multiply(x)
    assert np.array_equal(y, yo)


@pytest.mark.parametrize("n,sub", [((40, 36, 44), 8), (48, 16), ((50, 40, 33), 16), (64, 32), ((70, 64, 40), 32)])
def test_multiply_bitexact_sub_sizes(n, sub):
    # The marching-plane Laplacian at every supported tile edge, on ragged
    # grids (partial last tiles, absent neighbour tiles); unmasked values in
    # Dirichlet and exterior cells must not leak into the result.
    d = domains.small(n, sub, 6 if sub < 32 else 10, seed=2)
    s, o = make_pair(d)
    try:
        rng = np.random.default_rng(5)
        x = rng.standard_normal(d.size).astype(np.float32)
        f0 = o.level_flags(0)
        x[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
        assert np.array_equal(s.Multiply(x), o.multiply(x))
    finally:
        s.close()


def test_vcycle_bitexact(small_pair):
    d, s, o = small_pair
    rng = np.random.default_rng(4)
    f0 = o.level_flags(0)
    u = rng.standard_normal(d.size).astype(np.float32)
    u[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
    b = rng.standard_normal(d.size).astype(np.float32)
    b[(f0 & ACTIVE) == 0] = 0
    for nv in (1, 2):
        ug = s.V_Cycle(u, b, nv)
        uo, r = u.copy(), np.zeros_like(u)
        for _ in range(nv):
            uo, r = o.vcycle(uo, r, b)
        assert np.array_equal(ug, uo), f"nv={nv}: max diff {np.max(np.abs(ug - uo))}"


def test_interface_matrices_bitexact(small_pair):
    d, s, o = small_pair
    M = d.meta["sigma_levels"]
    assert np.array_equal(s.Interface_Map(), o.interface_map())
    for l in range(M):
        a, b = s.Interface_Matrix("Arr", l), o.matrix("Arr", l)
        assert a.shape == b.shape and (a != b).nnz == 0
        if l + 1 < M:
            a, b = s.Interface_Matrix("Prr", l), o.matrix("Prr", l)
            assert a.shape == b.shape and (a != b).nnz == 0
        for sd in range(o.num_subdomains):
            for kind in ("Aii", "Air"):
                a, b = s.Interface_Matrix(kind, l, sd), o.matrix(kind, l, sd)
                assert a.shape == b.shape and (a != b).nnz == 0, (kind, l, sd)


def test_sigma_vcycle(small_pair):
    d, s, o = small_pair
    rng = np.random.default_rng(5)
    b0 = rng.standard_normal(o.num_interface(0)).astype(np.float32)
    ug = s.Sigma_V_Cycle(b0)
    uo = o.sigma_vcycle(b0)
    assert rel_inf(ug, uo) < PRECOND_RTOL


def test_apply_preconditioner(small_pair):
    d, s, o = small_pair
    rng = np.random.default_rng(6)
    f0 = o.level_flags(0)
    r = rng.standard_normal(d.size).astype(np.float32)
    r[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
    zg = s.Apply_Preconditioner(r)
    zo = o.apply_preconditioner(r)
    assert rel_inf(zg, zo) < PRECOND_RTOL


def test_pcg_small_matches_oracle(small_pair):
    d, s, o = small_pair
    res = s.Solve()
    xo, it_o, info = o.solve(d.rhs, tol=1e-6)
    assert res["converged"] == 1
    assert abs(res["iterations"] - it_o) <= 1
    assert res["true_residual_inf"] <= 2e-6
    x = s.Solution()
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-5


def test_pcg_config1_against_fp64_oracle():
    """Config 1 (64^3, 64 subdomains): iteration parity with the FP32 oracle at
    1e-6, solution error no worse than the oracle's own at that tolerance, and
    1e-5 relative L2 against the FP64 discrete solution once the residual is
    driven to 1e-7 in mixed precision."""
    d = domains.config1()
    s, o = make_pair(d)
    res = s.Solve()
    x = s.Solution()
    xo, it_o, _ = o.solve(d.rhs, tol=1e-6)
    assert res["converged"] == 1
    assert abs(res["iterations"] - it_o) <= 1, (res["iterations"], it_o)
    assert res["true_residual_inf"] <= 2e-6
    o64 = Oracle(d.size, d.sub_size, d.flags, vlevels=3, nVcycles=1, interior_smoothing=3,
                 boundary_smoothing=3, sigma_levels=3, sigma_smoothing=3, sigma_mg=1, dtype=np.float64)
    x64, _, _ = o64.solve(d.rhs, tol=1e-12, max_it=200)
    nrm = np.linalg.norm(x64)
    err = np.linalg.norm(x.astype(np.float64) - x64) / nrm
    err_o = np.linalg.norm(xo.astype(np.float64) - x64) / nrm
    assert err <= 2.0 * err_o + 1e-6, (err, err_o)
    m = d.meta
    s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                m["sigma_mg"], tol=1e-7, precision_mode=1, true_residual_every=10)
    res7 = s.Solve()
    x7 = s.Solution()
    s.close()
    err7 = np.linalg.norm(x7.astype(np.float64) - x64) / nrm
    assert res7["converged"] == 1
    assert err7 <= 1e-5, err7


@pytest.mark.parametrize("cluster", ["1", "2"])
def test_vcycle_sub16_cluster_variants_bitexact(cluster, monkeypatch):
    """The 16^3 V-cycle runs either in one CTA or split over a 2-CTA cluster."""
    monkeypatch.setenv("HDD_VCYCLE_CLUSTER", cluster)
    d = domains.small(48, 16, 8, seed=7)
    s, o = make_pair(d)
    rng = np.random.default_rng(8)
    f0 = o.level_flags(0)
    u = rng.standard_normal(d.size).astype(np.float32)
    u[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
    b = rng.standard_normal(d.size).astype(np.float32)
    b[(f0 & ACTIVE) == 0] = 0
    ug = s.V_Cycle(u, b, 1)
    s.close()
    uo, _ = o.vcycle(u, np.zeros_like(u), b)
    assert np.array_equal(ug, uo), np.max(np.abs(ug - uo))


def test_sub32_cluster_vcycle_and_pcg():
    """32^3 subdomains use the 4-CTA cluster kernel: bit-exact V-cycle, PCG parity."""
    d = domains.small(64, 32, 10, seed=9)
    d.meta.update(vlevels=4, interior_smoothing=4, boundary_smoothing=4, sigma_levels=4)
    s, o = make_pair(d)
    rng = np.random.default_rng(10)
    f0 = o.level_flags(0)
    u = rng.standard_normal(d.size).astype(np.float32)
    u[(f0 & (ACTIVE | INTERFACE)) == 0] = 0
    b = rng.standard_normal(d.size).astype(np.float32)
    b[(f0 & ACTIVE) == 0] = 0
    for nv in (1, 2):
        ug = s.V_Cycle(u, b, nv)
        uo, r = u.copy(), np.zeros_like(u)
        for _ in range(nv):
            uo, r = o.vcycle(uo, r, b)
        assert np.array_equal(ug, uo), (nv, np.max(np.abs(ug - uo)))
    res = s.Solve()
    x = s.Solution()
    s.close()
    xo, it_o, _ = o.solve(d.rhs, tol=1e-6)
    assert res["converged"] == 1 and abs(res["iterations"] - it_o) <= 1, (res["iterations"], it_o)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-5


def test_sigma_literal_bottom_smoothing(capfd, monkeypatch):
    """A coarsest sigma level whose smoother contracts slowly (rho ~0.96 here):
    the 200 bottom smoothing steps have not converged to the Schur solve, so the
    GPU runs them literally, as the reference does; it must match the oracle."""
    monkeypatch.setenv("HDD_VERBOSE", "1")
    d = domains.profile_case()
    s, o = make_pair(d, sigma_levels=2)
    try:
        err = capfd.readouterr().err
        assert "200 literal smoothing steps" in err, err[-2000:]
        rng = np.random.default_rng(7)
        b0 = rng.standard_normal(o.num_interface(0)).astype(np.float32)
        assert rel_inf(s.Sigma_V_Cycle(b0), o.sigma_vcycle(b0)) < PRECOND_RTOL
    finally:
        s.close()


def test_spgrid_directory_load_matches_dense(tmp_path):
    """hdd_load_spgrid_dir reads the reference's on-disk format (padded size,
    page offsets, per-block flags/data arrays) to the same domain as the dense
    input: identical PCG iterations and solution."""
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    from spgrid_format import write_spgrid_dir
    d = domains.small(32, 8, 6, seed=1)
    write_spgrid_dir(str(tmp_path), d.flags, d.rhs)
    m = d.meta
    args = (m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"], m["interior_smoothing"],
            m["boundary_smoothing"], m["sigma_smoothing"], m["sigma_mg"])
    a = SPGrid_Domain_Decomposition_Solver()
    a.Read_SPGrid(str(tmp_path))
    a.Initialize_Preconditioner(*args)
    ra, xa = a.Solve(), a.Solution()
    a.close()
    b = SPGrid_Domain_Decomposition_Solver()
    b.Set_Domain(d.flags, d.rhs)
    b.Initialize_Preconditioner(*args)
    rb, xb = b.Solve(), b.Solution()
    b.close()
    assert ra["iterations"] == rb["iterations"]
    assert np.array_equal(xa, xb)
