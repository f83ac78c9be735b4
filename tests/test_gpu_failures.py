"""Failure reporting on the GPU path without a GPU fault: a NaN in the
right-hand side ends PCG with HDD_ERR_BREAKDOWN (the non-finite scalar is seen
on the host after the iteration; every kernel has a fixed trip count, so none
waits on the bad value), and the same handle then solves a finite right-hand
side as if nothing had happened."""
import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from hierarchicaldd_b200._lib import HddError
from hierarchicaldd_b200.domains import ACTIVE
from test_gpu_parity import make_pair

pytestmark = pytest.mark.gpu


def test_nan_rhs_reports_breakdown_and_the_handle_recovers():
    d = domains.small(32, 8, 6, seed=9)
    s, o = make_pair(d)
    try:
        r_ok = s.Solve()
        x_ok = s.Solution()
        bad = d.rhs.copy()
        act = np.argwhere((d.flags & ACTIVE) != 0)
        bad[tuple(act[len(act) // 2])] = np.nan
        s.Set_RHS(bad)
        with pytest.raises(HddError) as e:
            s.Solve(allow_not_converged=True)
        assert e.value.status == 7, e.value   # HDD_ERR_BREAKDOWN
        s.Set_RHS(d.rhs)
        r = s.Solve()
        assert r["converged"] == 1 and r["iterations"] == r_ok["iterations"]
        assert np.array_equal(s.Solution(), x_ok)
    finally:
        s.close()


def test_bounded_wait_runs_out_reports_timeout_and_the_handle_recovers():
    """A dependency made unsatisfiable (one parent front waits for a task more
    than its child runs) with a short poll limit: the wait gives up, raises the
    error word, later waits return at once, PCG stops after that iteration with
    HDD_ERR_TIMEOUT well within the wait's bound, and once the dependency is
    restored the same handle solves to the same bits as before.  Nothing faults
    or hangs: the wait is a bounded poll loop that returns a status."""
    import time
    from hierarchicaldd_b200 import _lib
    d = domains.small(32, 8, 6, seed=9)
    s, o = make_pair(d)
    lib = _lib.load()
    try:
        r_ok = s.Solve()
        x_ok = s.Solution()
        assert lib.hdd_set_wait_limit(s.h, 1000) == 0
        assert lib.hdd_test_stall_dependency(s.h, 1) == 0
        t0 = time.perf_counter()
        with pytest.raises(HddError) as e:
            s.Solve(allow_not_converged=True)
        dt = time.perf_counter() - t0
        assert e.value.status == 8, e.value   # HDD_ERR_TIMEOUT
        assert dt < 10.0, dt
        assert len(s.Residual_History()) <= 2   # stopped after the first iteration
        assert lib.hdd_test_stall_dependency(s.h, 0) == 0
        assert lib.hdd_set_wait_limit(s.h, 1 << 22) == 0
        r = s.Solve()
        assert r["converged"] == 1 and r["iterations"] == r_ok["iterations"]
        assert np.array_equal(s.Solution(), x_ok)
    finally:
        s.close()
