"""The velocity -> divergence right-hand side (the reference Test_Bench's
"velocity" mode on a uniform grid) in the oracle, without a GPU: a known answer
and the flag conversion."""
import numpy as np

from hierarchicaldd_b200 import domains
from hierarchicaldd_b200.domains import ACTIVE, DIRICHLET
from oracle_ffi import velocity_divergence
from velocity_cases import F_ACTIVE, F_DIRICHLET, INTERIOR, fluid_flags


def test_linear_velocity_has_constant_divergence():
    """u on the -x face of cell i is i (v = w = 0), dx = 0.5: scale =
    (1/dx)^3 * (-dx^2) = -2, so every interior cell gets -2 * (u(i+1) - u(i)) = -2
    exactly, and the Dirichlet and exterior cells 0."""
    d = domains.small(8, 8, 0, seed=1)
    ff = fluid_flags(d.flags)
    i = np.arange(d.size[0], dtype=np.float32)[:, None, None]
    u = np.broadcast_to(i, d.size).astype(np.float32)
    z = np.zeros(d.size, np.float32)
    flags, rhs = velocity_divergence(ff, u, z, z, 0.5)
    interior = (ff & INTERIOR) != 0
    assert np.all(rhs[interior] == -2.0)
    assert np.all(rhs[~interior] == 0.0)
    assert np.array_equal(flags == ACTIVE, (ff & F_ACTIVE) != 0)
    assert np.array_equal(flags == DIRICHLET, (ff & F_DIRICHLET) != 0)
    assert np.all((flags == 0) == ((ff & (F_ACTIVE | F_DIRICHLET)) == 0))
