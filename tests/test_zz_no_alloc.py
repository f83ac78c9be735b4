"""The allocation-free entry point hdd_multiply_dot_dense_device_noalloc.

It exists for callers that cannot allocate device memory at the moment they
apply the operator (their own allocator owns the GPU's memory, or the loop
cannot stall on an allocation), so it keeps its per-tile partial sums in a
fixed device array instead of allocating.  Here it is called twice in a row
through the C ABI on device arrays and checked against hdd_multiply_dense:
y bit for bit (same kernel arithmetic), the dot against an FP64 sum of the
FP32 products with a relative tolerance of 1e-12 (only the summation order
differs).  The second call checks that the shared scratch carries nothing
over from the first.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from hierarchicaldd_b200 import domains
from hierarchicaldd_b200.domains import ACTIVE

pytestmark = pytest.mark.gpu

DOT_RTOL = 1e-12


def test_noalloc_multiply_dot_matches_multiply_dense():
    import torch
    from hierarchicaldd_b200 import _lib
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver

    d = domains.small(32, 8, 6, seed=1)
    m = d.meta
    s = SPGrid_Domain_Decomposition_Solver()
    try:
        s.Set_Domain(d.flags, d.rhs)
        s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"])
        lib = _lib.load()
        dev = torch.device("cuda:0")
        stream = torch.cuda.current_stream(dev)
        rng = np.random.default_rng(11)
        for call in range(2):
            x = rng.standard_normal(d.size).astype(np.float32)
            x[(d.flags & ACTIVE) == 0] = 0
            y_ref = s.Multiply(x)

            xd = torch.from_numpy(x).to(dev)
            yd = torch.zeros(d.size, dtype=torch.float32, device=dev)
            dotd = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
            st = lib.hdd_multiply_dot_dense_device_noalloc(
                s.h, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), C.c_void_p(dotd.data_ptr()),
                C.c_void_p(stream.cuda_stream))
            assert st == _lib.HDD_OK, lib.hdd_last_error(s.h)
            torch.cuda.synchronize(dev)
            y = yd.cpu().numpy()
            dot = float(dotd.cpu().item())

            assert np.array_equal(y, y_ref), f"call {call}: max diff {np.max(np.abs(y - y_ref))}"
            # FP32 products summed in FP64, as the kernel does.
            dot_ref = float(np.sum((x * y_ref).astype(np.float64)))
            assert abs(dot - dot_ref) <= DOT_RTOL * max(abs(dot_ref), 1e-30), (call, dot, dot_ref)
    finally:
        s.close()


def test_noalloc_on_a_ragged_domain_reads_and_leaves_cells_like_the_tiled_path():
    """A grid whose sizes (41 x 37 x 45 cells) are not multiples of the 8^3
    subdomains, x random everywhere (Dirichlet and exterior cells included), y
    prefilled with a sentinel: inside the stored tiles y equals
    hdd_multiply_dense bit for bit (Dirichlet and inactive neighbour values are
    read the same way), cells outside them keep the sentinel, and the caller's
    current device is unchanged."""
    import torch
    from hierarchicaldd_b200 import _lib
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver

    d = domains.small((40, 36, 44), 8, 6, seed=4)
    m = d.meta
    S = d.sub_size[0]
    s = SPGrid_Domain_Decomposition_Solver()
    try:
        s.Set_Domain(d.flags, d.rhs)
        s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"])
        lib = _lib.load()
        dev = torch.device("cuda:0")
        stream = torch.cuda.current_stream(dev)
        # Stored tiles: those holding an Active (after the divider: Active or Interface) cell.
        act = (d.flags & ACTIVE) != 0
        nt = [(n + S - 1) // S for n in d.size]
        pad = np.zeros([t * S for t in nt], bool)
        pad[:d.size[0], :d.size[1], :d.size[2]] = act
        tiles = pad.reshape(nt[0], S, nt[1], S, nt[2], S).any(axis=(1, 3, 5))
        inside = np.repeat(np.repeat(np.repeat(tiles, S, 0), S, 1), S, 2)[:d.size[0], :d.size[1], :d.size[2]]
        assert inside.any() and not inside.all()
        rng = np.random.default_rng(12)
        sentinel = np.float32(12345.0)
        for call in range(2):
            x = rng.standard_normal(d.size).astype(np.float32)
            y_ref = s.Multiply(x)
            xd = torch.from_numpy(x).to(dev)
            yd = torch.full(d.size, float(sentinel), dtype=torch.float32, device=dev)
            dotd = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
            before = torch.cuda.current_device()
            st = lib.hdd_multiply_dot_dense_device_noalloc(
                s.h, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), C.c_void_p(dotd.data_ptr()),
                C.c_void_p(stream.cuda_stream))
            assert st == _lib.HDD_OK, lib.hdd_last_error(s.h)
            assert torch.cuda.current_device() == before
            torch.cuda.synchronize(dev)
            y = yd.cpu().numpy()
            assert np.array_equal(y[inside], y_ref[inside]), call
            assert np.all(y[~inside] == sentinel), call
            dot_ref = float(np.sum((x[inside] * y_ref[inside]).astype(np.float64)))
            dot = float(dotd.cpu().item())
            assert abs(dot - dot_ref) <= DOT_RTOL * max(abs(dot_ref), 1e-30), (call, dot, dot_ref)
    finally:
        s.close()
