"""Parity on the sparse sphere-union workload (the 1024^3-cell box with 64
spheres, about a tenth of it inside them, exterior cells unallocated) at 1/8
scale: config5(8), a 128^3-cell box with the same seeds and shape, given to
the GPU as SPGrid pages (hdd_set_domain_pages: only pages holding a cell of the
union, as an SPGrid allocator holds them).

* Reference precision: PCG iterations within +-1 of the FP32 oracle's at 1e-6
  relative residual (max|r| of the recursively updated residual), true
  residual within twice the oracle's (FP32 iterates floor near 1e-6 here).
* The workload's precision form (FP32 preconditioner, FP64 iterate) solved to
  1e-8: within 1e-5 relative L2 of the FP64 oracle's discrete solution.
"""
import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu


def _oracle(d, dtype):
    m = d.meta
    return Oracle(d.size, d.sub_size, d.flags, vlevels=m["vlevels"], nVcycles=m["nVcycles"],
                  interior_smoothing=m["interior_smoothing"], boundary_smoothing=m["boundary_smoothing"],
                  sigma_levels=m["sigma_levels"], sigma_smoothing=m["sigma_smoothing"], sigma_mg=m["sigma_mg"],
                  dtype=dtype)


def _gpu(d, tol, precision_mode):
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    m = d.meta
    origin, fp, rp = domains.to_pages(d.flags, d.rhs)  # only pages holding a cell of the union
    box_pages = int(np.prod([-(-n // b) for n, b in zip(d.size, (4, 8, 8))]))
    s = SPGrid_Domain_Decomposition_Solver()
    try:
        s.Set_Domain_Pages(origin, fp, rp)
        s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"], tol=tol, precision_mode=precision_mode, max_iters=500)
        r = s.Solve()
        return r, s.Solution_F64(), len(origin), box_pages
    finally:
        s.close()


@pytest.fixture(scope="module")
def c5_small():
    return domains.config5(8)


def test_c5_eighth_scale_iterations_match_the_oracle(c5_small):
    d = c5_small
    r, _, held, total = _gpu(d, 1e-6, 0)
    assert held < total  # the page list leaves the empty part of the box out
    _, it, info = _oracle(d, np.float32).solve(d.rhs, tol=1e-6)
    assert abs(r["iterations"] - it) <= 1, (r["iterations"], it)
    # An FP32 iterate's true residual sits near 1e-6 here (the oracle's own is
    # about 1.4e-6): bounded by twice the oracle's.
    o_true = info["true_res_inf"] / info["b_inf"]
    assert r["true_residual_inf"] <= max(1e-6, 2 * o_true), (r, o_true)


def test_c5_eighth_scale_precision_form_reaches_the_fp64_solution(c5_small):
    d = c5_small
    r, x, _, _ = _gpu(d, 1e-8, 1)
    assert r["converged"] == 1 and r["true_residual_inf"] <= 1e-8, r
    x64, _, info = _oracle(d, np.float64).solve(d.rhs, tol=1e-11, max_it=500)
    err = float(np.linalg.norm(x - x64) / np.linalg.norm(x64))
    assert err <= 1e-5, err
