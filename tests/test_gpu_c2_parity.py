"""Parity at the 256^3 workload (257^3 flags, Dirichlet sphere r=48, delta plus
noise, 32^3 subdomains, vlevels 4, smoothing 4/4, sigma_levels 4) against the
oracle's full solves stored in tests/golden/c2_oracle.npz (made by
tests/golden/make_c2_fixture.py):

* PCG iteration count within +-1 of the FP32 oracle's (the reference's
  precision) at 1e-6 relative max-norm residual;
* the max|r| history agrees with the oracle's to 1 % over the first 15
  iterations (after that the max-norm of an FP32 residual near 1e-5 moves with
  rounding in both);
* true relative residual of the returned x <= 1e-6;
* the solution within 1e-5 relative L2 of the FP64 oracle's discrete solution
  (compared on every 4th cell along each axis, 65^3 cells).  A residual of
  1e-6 bounds the error only through the condition number: at that tolerance
  the error is about 3e-4 here, for the oracle's solve as for the GPU's.  The
  bound is met by the precision form (FP64 iterate, FP32 preconditioner)
  solved to 1e-8, which is what this test runs for it.
"""
import os

import numpy as np
import pytest

from conftest import ROOT
from hierarchicaldd_b200 import domains

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(ROOT, "tests", "golden", "c2_oracle.npz")


def _solve(tol, precision_mode, max_iters=5000):
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    d = domains.config2()
    m = d.meta
    s = SPGrid_Domain_Decomposition_Solver()
    try:
        s.Set_Domain(d.flags, d.rhs)
        s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"], tol=tol, precision_mode=precision_mode, max_iters=max_iters)
        r = s.Solve()
        return r, s.Residual_History(), s.Solution_F64()
    finally:
        s.close()


@pytest.fixture(scope="module")
def c2_solve():
    return _solve(1e-6, 0)


def rel_l2_to_oracle(x):
    z = np.load(FIXTURE)
    st = int(z["stride"])
    xs = x[::st, ::st, ::st].astype(np.float64)
    ref = z["x64_sub"].astype(np.float64)
    return float(np.linalg.norm(xs - ref) / np.linalg.norm(ref))


def test_c2_iterations_within_one_of_the_oracle(c2_solve):
    r, hist, _ = c2_solve
    z = np.load(FIXTURE)
    assert abs(r["iterations"] - int(z["iterations_fp32"])) <= 1, (r["iterations"], int(z["iterations_fp32"]))
    h_o = z["history_fp32"]
    n = 15
    rel = np.abs(hist[:n] - h_o[:n]) / h_o[:n]
    assert np.all(rel <= 1e-2), rel


def test_c2_true_residual_and_solution_error(c2_solve):
    r, _, x = c2_solve
    assert r["true_residual_inf"] <= 1e-6, r["true_residual_inf"]
    # Stated, not bounded here: the error a 1e-6 residual leaves (about 3e-4).
    assert rel_l2_to_oracle(x) <= 1e-3


def test_c2_precision_form_reaches_the_fp64_oracle_solution():
    r, _, x = _solve(1e-8, 1, max_iters=200)
    assert r["converged"] == 1 and r["true_residual_inf"] <= 1e-8, r
    err = rel_l2_to_oracle(x)
    assert err <= 1e-5, err
