"""CPU checks of the CUDA library and the host-side Python mirror (no GPU).

* libhdd_b200.so loads and exports every function that include/hdd.h
  declares, and the ctypes table covers exactly those;
* option defaults equal the reference Test_Bench defaults
  (demos/Domain_Decomposition_CPU_Only/Test_Bench_3D/main.cpp:236-251);
* without a GPU, creating a solver fails loudly with HDD_ERR_CUDA: there is no
  CPU fallback;
* the synthetic domain generator follows its rules (Dirichlet outer layer and
  spheres, orphan Dirichlet cells dropped, face bits on Active cells), and so
  does the sparse sphere-union generator.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available
from hierarchicaldd_b200 import _lib, domains
from hierarchicaldd_b200.domains import ACTIVE, DIRICHLET, FACE_ALL, FACE_MX


def header_functions():
    text = open(os.path.join(ROOT, "include", "hdd.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(hdd_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_header_symbol(hdd_lib):
    names = header_functions()
    assert len(names) >= 20
    for n in sorted(names):
        assert hasattr(hdd_lib, n), n
    assert names == set(_lib.SIGNATURES), names.symmetric_difference(set(_lib.SIGNATURES))


def test_options_default_match_test_bench(hdd_lib):
    o = _lib.hdd_options()
    hdd_lib.hdd_options_default(C.byref(o))
    assert o.vlevels == 3 and o.nVcycles == 1 and o.interior_smoothing == 1 and o.boundary_smoothing == 3
    assert o.sigma_levels == 3 and o.sigma_smoothing == 3 and o.sigma_mg == 1
    assert o.max_iters == 5000 and o.relative_tol == 1 and abs(o.tol - 1e-6) < 1e-18
    assert o.multilevel == 0  # -multilevel no


@pytest.mark.parametrize("multilevel,sub,status", [(2, 64, 1), (1, 15, 1), (1, 24, 5), (1, 128, 5)])
def test_two_level_options_are_checked_before_any_gpu_call(hdd_lib, multilevel, sub, status):
    """multilevel must be 0 or 1; two-level DD needs an even sub_size whose half
    is a V-cycle box size (8, 16, 32): refused before the device is touched."""
    o = _lib.hdd_options()
    hdd_lib.hdd_options_default(C.byref(o))
    o.multilevel = multilevel
    for a in range(3):
        o.sub_size[a] = sub
    h = C.c_void_p()
    assert hdd_lib.hdd_create(C.byref(o), C.byref(h)) == status and not h.value


def test_status_strings(hdd_lib):
    for code, name in _lib.STATUS_NAMES.items():
        s = hdd_lib.hdd_status_string(code)
        assert s and isinstance(s, bytes)


def test_server_options_default(hdd_lib):
    o = _lib.hdd_server_options()
    hdd_lib.hdd_server_options_default(C.byref(o))
    assert o.slots == 4 and o.hbm_budget_bytes == 0 and o.device == 0 and o.setup_threads == 0
    h = C.c_void_p()
    o.slots = 0
    assert hdd_lib.hdd_server_create(C.byref(o), C.byref(h)) == 1 and not h.value


@pytest.mark.skipif(gpu_available(), reason="checks the GPU-less failure path")
def test_server_create_fails_loudly_without_gpu(hdd_lib):
    o = _lib.hdd_server_options()
    hdd_lib.hdd_server_options_default(C.byref(o))
    h = C.c_void_p()
    assert hdd_lib.hdd_server_create(C.byref(o), C.byref(h)) == 2 and not h.value


@pytest.mark.skipif(gpu_available(), reason="checks the GPU-less failure path")
def test_create_fails_loudly_without_gpu(hdd_lib):
    o = _lib.hdd_options()
    hdd_lib.hdd_options_default(C.byref(o))
    h = C.c_void_p()
    st = hdd_lib.hdd_create(C.byref(o), C.byref(h))
    assert st == 2, _lib.STATUS_NAMES.get(st, st)  # HDD_ERR_CUDA
    assert not h.value


def test_generator_rules():
    d = domains.small(24, 8, 5, seed=3)
    f = d.flags
    n = d.size
    # Outer layer is never Active.
    for a in range(3):
        for side in (0, n[a] - 1):
            sl = [slice(None)] * 3
            sl[a] = side
            assert not np.any(f[tuple(sl)] & ACTIVE)
    # Sphere cells are not Active; cells outside sphere and outer layer are Active.
    i, j, k = np.ogrid[0:n[0], 0:n[1], 0:n[2]]
    c = 12
    inside = (i - c) ** 2 + (j - c) ** 2 + (k - c) ** 2 <= 25
    outer = (i == 0) | (i == n[0] - 1) | (j == 0) | (j == n[1] - 1) | (k == 0) | (k == n[2] - 1)
    assert np.array_equal((f & ACTIVE) != 0, ~(inside | outer))
    # Every Dirichlet cell has an Active face neighbour (orphans were dropped).
    act = np.pad((f & ACTIVE) != 0, 1)
    nb_active = np.zeros(n, bool)
    for a in range(3):
        for s in (-1, 1):
            nb_active |= np.roll(act, s, axis=a)[1:-1, 1:-1, 1:-1]
    dir_mask = (f & DIRICHLET) != 0
    assert np.all(nb_active[dir_mask])
    # Face bits only on Active cells; every Active cell has all 6 faces here
    # (neighbours are Active or Dirichlet).
    assert not np.any(f[(f & ACTIVE) == 0] & FACE_ALL)
    assert np.all((f[(f & ACTIVE) != 0] & FACE_ALL) == FACE_ALL)
    # The right-hand side lives on Active cells only.
    assert not np.any(d.rhs[(f & ACTIVE) == 0])


def test_config_shapes():
    d1 = domains.config1()
    assert d1.size == (65, 65, 65) and d1.sub_size == (16, 16, 16)
    assert d1.rhs[16, 16, 16] == 1.0 and np.count_nonzero(d1.rhs) == 1
    assert not (d1.flags[32, 32, 32] & ACTIVE) and (d1.flags[32, 32, 32 + 13] & ACTIVE)
    assert FACE_MX == 0x100000


def test_sparse_sphere_union_rules():
    """The sparse workload's generator (at 1/8 scale): Active cells are the union
    cells whose six neighbours are all in the union, the union's edge is
    Dirichlet, the rest exterior; so no exterior cell touches an Active cell (the
    subdomain V-cycles need that), about a tenth of the box is Active, and the
    right-hand side has zero mean on the Active cells."""
    d = domains.config5(8)
    f = d.flags
    act = (f & ACTIVE) != 0
    dirichlet = (f & DIRICHLET) != 0
    ext = f == 0
    assert not np.any(act & dirichlet)
    pad = np.pad(ext, 1, constant_values=True)
    n0, n1, n2 = f.shape
    for a, b, c in [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]:
        assert not np.any(act & pad[1 + a:1 + a + n0, 1 + b:1 + b + n1, 1 + c:1 + c + n2])
    assert 0.05 < act.mean() < 0.15
    assert np.all(d.rhs[~act] == 0) and abs(float(d.rhs[act].astype(np.float64).mean())) < 1e-6
    assert d.sub_size == (32, 32, 32) and d.meta["sigma_levels"] == 4 and d.meta["vlevels"] == 5


def test_header_is_plain_c():
    """include/hdd.h is a C ABI: it compiles as C99 (for C, cgo or other FFI
    callers) as well as C++."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    hdr = os.path.join(ROOT, "include", "hdd.h")
    p = subprocess.run([gcc, "-fsyntax-only", "-x", "c", "-std=c99", "-Wall", "-Wextra", "-Werror", hdr],
                       capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
