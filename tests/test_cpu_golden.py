"""The oracle against its committed golden fixtures (tests/golden, made by
tests/golden/make_golden.py).  The reference ships no golden vectors for this
path and cannot be built here, so these fixtures anchor the oracle itself:
the generator, the level-0 topology, the Laplacian and the V-cycle bit for bit,
the level-0 interface matrix exactly, and the PCG iteration count and residual
history of a full solve."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402


@pytest.mark.parametrize("name", sorted(make_golden.CASES))
def test_oracle_reproduces_golden(name):
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    now = make_golden.compute(name)
    for key in ("flags", "rhs", "level0_flags", "x", "b", "laplacian", "vcycle", "arr_ptr", "arr_col",
                "arr_val"):
        assert np.array_equal(now[key], g[key]), key
    assert int(now["iterations"]) == int(g["iterations"])
    np.testing.assert_allclose(now["history"], g["history"], rtol=1e-4)
