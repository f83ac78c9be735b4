"""CPU checks of the oracle (no GPU).

The reference ships no golden vectors or known-answer tests for this path, so
the oracle is pinned on its own:

* known answers on analytic fields: A applied to the constant field counts
  each cell's Dirichlet faces (the Laplacian of the reference sums
  (c - n) over flagged faces, and Dirichlet neighbours carry 0);
* the preconditioner is symmetric, <y, P x> = <x, P y>, as CG requires
  (PB/Public_Library/PhysBAM_Tools/Krylov_Solvers/KRYLOV_SYSTEM_BASE.cpp:81-85);
* FP32 and FP64 builds of the oracle take the same PCG iteration count (+-1);
* a tight FP64 solve reaches a tiny true residual (the operator and PCG agree).
"""
import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from hierarchicaldd_b200.domains import ACTIVE, DIRICHLET, FACE_MX, INTERFACE
from oracle_ffi import Oracle


def make_oracle(d, dtype):
    m = d.meta
    return Oracle(d.size, d.sub_size, d.flags, vlevels=m["vlevels"], nVcycles=m["nVcycles"],
                  interior_smoothing=m["interior_smoothing"], boundary_smoothing=m["boundary_smoothing"],
                  sigma_levels=m["sigma_levels"], sigma_smoothing=m["sigma_smoothing"], sigma_mg=m["sigma_mg"],
                  dtype=dtype)


@pytest.fixture(scope="module")
def dom():
    return domains.small(16, 8, 3, seed=1)


@pytest.fixture(scope="module", params=[np.float64, np.float32], ids=["f64", "f32"])
def oracle(request, dom):
    return make_oracle(dom, request.param)


def dirichlet_face_count(flags):
    """Per cell, the number of flagged faces whose neighbour is Dirichlet."""
    n = flags.shape
    out = np.zeros(n, np.float64)
    pad = np.zeros(tuple(s + 2 for s in n), np.uint32)
    pad[1:-1, 1:-1, 1:-1] = flags
    offs = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    for f, (dx, dy, dz) in enumerate(offs):
        nb = pad[1 + dx:1 + dx + n[0], 1 + dy:1 + dy + n[1], 1 + dz:1 + dz + n[2]]
        has_face = (flags & (FACE_MX << f)) != 0
        out += (has_face & ((nb & DIRICHLET) != 0)).astype(np.float64)
    return out


def test_laplacian_of_constant_counts_dirichlet_faces(oracle):
    f0 = oracle.level_flags(0)
    solve = (f0 & (ACTIVE | INTERFACE)) != 0
    ones = np.zeros(oracle.size, oracle.dtype)
    ones[solve] = 1
    y = oracle.multiply(ones)
    expect = np.where(solve, dirichlet_face_count(f0), 0.0)
    assert np.array_equal(y.astype(np.float64), expect)
    # Interior cells away from Dirichlet give exactly 0; some cells see Dirichlet faces.
    assert np.count_nonzero(expect) > 0 and np.count_nonzero(solve & (expect == 0)) > 0


def test_divider_marks_interface_planes(dom, oracle):
    f0 = oracle.level_flags(0)
    sub = dom.sub_size[0]
    i, j, k = np.ogrid[0:dom.size[0], 0:dom.size[1], 0:dom.size[2]]
    on_plane = (i % sub == 0) | (j % sub == 0) | (k % sub == 0)
    was_active = (dom.flags & ACTIVE) != 0
    assert np.array_equal((f0 & INTERFACE) != 0, was_active & on_plane)
    assert np.array_equal((f0 & ACTIVE) != 0, was_active & ~on_plane)


def test_preconditioner_symmetric(dom):
    o = make_oracle(dom, np.float64)
    f0 = o.level_flags(0)
    mask = (f0 & (ACTIVE | INTERFACE)) != 0
    rng = np.random.default_rng(0)
    x, y = rng.standard_normal(dom.size), rng.standard_normal(dom.size)
    x[~mask] = 0
    y[~mask] = 0
    a = float(np.sum(y * o.apply_preconditioner(x)))
    b = float(np.sum(x * o.apply_preconditioner(y)))
    assert abs(a - b) <= 1e-6 * max(abs(a), abs(b))


def test_fp32_fp64_iteration_counts_agree(dom):
    its = {}
    for dt in (np.float32, np.float64):
        o = make_oracle(dom, dt)
        _, it, info = o.solve(dom.rhs.astype(dt), tol=1e-6)
        assert info["true_res_inf"] <= 2e-6 * info["b_inf"] + 1e-30
        its[dt] = it
    assert abs(its[np.float32] - its[np.float64]) <= 1


def test_tight_fp64_solve_has_tiny_true_residual(dom):
    o = make_oracle(dom, np.float64)
    x, it, info = o.solve(dom.rhs.astype(np.float64), tol=1e-12)
    assert info["true_res_inf"] <= 1e-11 * info["b_inf"]
    # A x reproduces b on the solve cells.
    f0 = o.level_flags(0)
    mask = (f0 & (ACTIVE | INTERFACE)) != 0
    ax = o.multiply(x)
    assert np.max(np.abs(ax[mask] - dom.rhs[mask])) <= 1e-10
