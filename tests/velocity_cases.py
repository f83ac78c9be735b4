"""Fluid-simulation inputs for the velocity -> divergence tests: SPGrid_Fluids
cell flags (FLUIDS_SIMULATION_FLAGS.h:13-25) built from a solver domain, and
face velocities."""
import numpy as np

from hierarchicaldd_b200.domains import ACTIVE, DIRICHLET

INTERIOR, F_DIRICHLET, GHOST, F_ACTIVE = 0x1, 0x2, 0x4, 0x8
X_VALID, Y_VALID, Z_VALID = 0x10, 0x20, 0x40


def fluid_flags(flags):
    """Active solver cells -> Interior|Active fluid cells, Dirichlet ->
    Dirichlet; a cell's -x/-y/-z face is valid when the cell or its minus
    neighbour is Interior (the face belongs to an interior cell)."""
    interior = (flags & ACTIVE) != 0
    ff = np.zeros(flags.shape, np.uint32)
    ff[interior] |= INTERIOR | F_ACTIVE
    ff[(flags & DIRICHLET) != 0] |= F_DIRICHLET
    for a, bit in enumerate((X_VALID, Y_VALID, Z_VALID)):
        minus = np.zeros_like(interior)
        sl_dst = [slice(None)] * 3
        sl_src = [slice(None)] * 3
        sl_dst[a] = slice(1, None)
        sl_src[a] = slice(0, -1)
        minus[tuple(sl_dst)] = interior[tuple(sl_src)]
        ff[interior | minus] |= bit
    return ff


def face_velocities(shape, seed):
    rng = np.random.Generator(np.random.Philox(seed))
    return [rng.uniform(-1, 1, shape).astype(np.float32) for _ in range(3)]
