"""The SPGrid format and the reference's domain generator, pinned to the one
artifact the reference ships: the 2D directory written by Create_2D_Domain
(demos/SPGrid_Create_Simple_Domain/Create_2D_Domain/output, 256 x 256 cells).

* the dimension-general address masks reproduce the 3D constants;
* the restated generator (domains.reference_generator) gives, cell for cell,
  the flags and right-hand side that directory decodes to: compared through
  the digests in tests/golden/spgrid2d_fixture.json (made by
  tests/golden/make_spgrid2d_golden.py), and against the directory itself
  where the reference tree is present;
* the generator's Neumann bubble in 3D: the oracle solves it; the product's
  host setup takes it with the whole-grid V-cycle (its subdomain boxes couple
  at coarse levels) and assembles the oracle's interface matrices bit for bit.
"""
import ctypes as C
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT
from hierarchicaldd_b200 import domains
from oracle_ffi import Oracle
from spgrid_format import XM, YM, ZM, axis_masks, read_spgrid_dir_any

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "spgrid2d_fixture.json")))
# The reference checkout, when one is at hand (HDD_REFERENCE_ROOT); the digests
# above were made from it by tests/golden/make_spgrid2d_golden.py.
REFERENCE_DIR = (os.path.join(os.environ["HDD_REFERENCE_ROOT"], GOLDEN["source"])
                 if os.environ.get("HDD_REFERENCE_ROOT") else None)


def digest(a, dt):
    return hashlib.sha256(np.ascontiguousarray(a, dt).tobytes()).hexdigest()


def test_axis_masks_restate_the_3d_constants():
    masks, block = axis_masks(3)
    assert masks == [XM, YM, ZM] and block == (4, 8, 8)
    masks2, block2 = axis_masks(2)
    assert block2 == (16, 16) and masks2[0] & masks2[1] == 0
    assert (masks2[0] | masks2[1]) & 0xFFF == 0x3FC


def test_generator_matches_the_reference_2d_output():
    d = domains.reference_generator(GOLDEN["size"], GOLDEN["delta"])
    assert digest(d.flags, "<u4") == GOLDEN["flags_sha256"]
    assert digest(d.rhs, "<f4") == GOLDEN["data_sha256"]
    cells = GOLDEN["cells"]
    assert int(np.sum((d.flags & domains.ACTIVE) != 0)) == cells["active"]
    assert int(np.sum((d.flags & domains.DIRICHLET) != 0)) == cells["dirichlet"]


@pytest.mark.skipif(not REFERENCE_DIR or not os.path.isdir(REFERENCE_DIR),
                    reason="reference tree not given (HDD_REFERENCE_ROOT)")
def test_reference_2d_directory_decodes_to_the_generator():
    size, flags, data, blocks = read_spgrid_dir_any(REFERENCE_DIR)
    assert list(size) == GOLDEN["size"] and blocks == GOLDEN["blocks"]
    d = domains.reference_generator(size, GOLDEN["delta"])
    assert np.array_equal(flags, d.flags)
    assert np.array_equal(data, d.rhs)


def test_neumann_bubble_3d_oracle_solves_product_accepts():
    """The generator's Neumann bubble couples subdomain boxes at coarse V-cycle
    levels: the oracle solves it, and the product's layout takes it with the
    whole-grid V-cycle and assembles the same interface matrices bit for bit."""
    from test_cpu_host import matrix, shim as shim_fixture
    d = domains.reference_generator((35, 35, 35), (4, 16, 16))
    assert np.any(d.flags == 0) and d.n_active > 0
    o = Oracle(d.size, (8, 8, 8), d.flags, vlevels=3, nVcycles=1, interior_smoothing=3, boundary_smoothing=3,
               sigma_levels=2, sigma_smoothing=3, sigma_mg=1)
    _, it, info = o.solve(d.rhs, tol=1e-6)
    assert 0 < it < 50 and info["true_res_inf"] < 1e-5
    lib = shim_fixture.__wrapped__()
    size = (C.c_int * 3)(*d.size)
    sub = (C.c_int * 3)(8, 8, 8)
    flags = np.ascontiguousarray(d.flags, np.uint32)
    err = C.create_string_buffer(512)
    h = lib.shim_build(size, sub, 3, 2, flags.ctypes.data_as(C.POINTER(C.c_uint32)), err, 512)
    assert h, err.value
    try:
        assert lib.shim_global_vcycle(h) == 1
        # A Dirichlet-sphere domain keeps the per-box V-cycle.
        ds = domains.small(32, 8, 6, seed=1)
        fs = np.ascontiguousarray(ds.flags, np.uint32)
        hs = lib.shim_build((C.c_int * 3)(*ds.size), sub, 3, 2, fs.ctypes.data_as(C.POINTER(C.c_uint32)), err, 512)
        assert hs, err.value
        assert lib.shim_global_vcycle(hs) == 0
        lib.shim_free(hs)
        for l in range(2):
            a, b = matrix(lib, h, 0, l), o.matrix("Arr", l)
            assert a.shape == b.shape and (a != b).nnz == 0, l
            for sd in range(lib.shim_num_subdomains(h)):
                for kind, name in ((1, "Aii"), (2, "Air")):
                    a, b = matrix(lib, h, kind, l, sd), o.matrix(name, l, sd)
                    assert a.shape == b.shape and (a != b).nnz == 0, (name, l, sd)
    finally:
        lib.shim_free(h)
