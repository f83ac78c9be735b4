"""CPU checks of the product's host-side setup (no GPU): the layout, interface
assembly and supernodal Cholesky sources of the CUDA library compiled on their
own into a test shim (tests/host_shim.cpp).

* the interface matrices (Arr, Aii, Air, Prr) equal the oracle's bit for bit;
* the interface dump (the reference's -iomode output layout) reads back
  unchanged, follows the reference's file layout, reads hand-written Matrix
  Market files, and is checked against the domain on reload;
* the host setup gives the same bits with 1, 3 and 8 threads;
* SPGrid pages (hdd_set_domain_pages) scatter to and gather from the dense grid
  as the page layout says, and bad page lists are refused;
* the supernodal factorisation solves (A + 1e-5 I) x = b to FP64 accuracy for
  every matrix kind, and its explicit solve blocks [L^-1; -L_RJ L^-1] (what the
  GPU kernels read) give the same solution.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ROOT
from hierarchicaldd_b200 import domains
from oracle_ffi import Oracle
from shim_ffi import BUILD, SHIM, load_shim  # noqa: F401

@pytest.fixture(scope="module")
def shim():
    return load_shim()


def build(L, d, M):
    size = (C.c_int * 3)(*d.size)
    sub = (C.c_int * 3)(*d.sub_size)
    flags = np.ascontiguousarray(d.flags, np.uint32)
    err = C.create_string_buffer(512)
    h = L.shim_build(size, sub, d.meta["vlevels"], M, flags.ctypes.data_as(C.POINTER(C.c_uint32)), err, 512)
    assert h, err.value
    return h


def matrix(L, h, kind, level, sub=0):
    shape = (C.c_int * 3)()
    assert L.shim_matrix_shape(h, kind, level, sub, shape) == 0
    rows, cols, nnz = shape
    ptr = np.zeros(rows + 1, np.int32)
    col = np.zeros(max(nnz, 1), np.int32)
    val = np.zeros(max(nnz, 1), np.float64)
    L.shim_matrix_get(h, kind, level, sub, ptr.ctypes.data_as(C.POINTER(C.c_int)),
                      col.ctypes.data_as(C.POINTER(C.c_int)), val.ctypes.data_as(C.POINTER(C.c_double)))
    return sp.csr_matrix((val[:nnz], col[:nnz], ptr), shape=(rows, cols))


@pytest.mark.parametrize("n,sub,radius", [(32, 8, 6), (32, 16, 5),
                                           # ragged: the last subdomains along y and z (and x) are partial
                                           ((40, 36, 44), 8, 6), ((33, 40, 40), 8, 5), ((48, 40, 56), 16, 7)])
def test_interface_matrices_match_oracle(shim, n, sub, radius):
    d = domains.small(n, sub, radius, seed=4)
    M = d.meta["sigma_levels"]
    h = build(shim, d, M)
    m = d.meta
    o = Oracle(d.size, d.sub_size, d.flags, vlevels=m["vlevels"], nVcycles=1, interior_smoothing=1,
               boundary_smoothing=1, sigma_levels=M, sigma_smoothing=3, sigma_mg=1)
    try:
        for l in range(M):
            kinds = [(0, "Arr", None)] + ([(3, "Prr", None)] if l + 1 < M else [])
            for kind, name, _ in kinds:
                a, b = matrix(shim, h, kind, l), o.matrix(name, l)
                assert a.shape == b.shape and (a != b).nnz == 0, (name, l)
            for sd in range(shim.shim_num_subdomains(h)):
                for kind, name in ((1, "Aii"), (2, "Air")):
                    a, b = matrix(shim, h, kind, l, sd), o.matrix(name, l, sd)
                    assert a.shape == b.shape and (a != b).nnz == 0, (name, l, sd)
    finally:
        shim.shim_free(h)


def test_supernodal_factorisation_solves(shim):
    d = domains.small(32, 8, 6, seed=4)
    M = d.meta["sigma_levels"]
    h = build(shim, d, M)
    try:
        diff = C.c_double()
        for l in range(M):
            res = shim.shim_factor_check(h, 0, l, 0, C.byref(diff))
            assert 0 <= res < 1e-10 and diff.value < 1e-10, ("Arr", l, res, diff.value)
            for sd in range(shim.shim_num_subdomains(h)):
                res = shim.shim_factor_check(h, 1, l, sd, C.byref(diff))
                if res < 0:
                    continue  # no interior DOFs
                assert res < 1e-10 and diff.value < 1e-10, ("Aii", l, sd, res, diff.value)
    finally:
        shim.shim_free(h)


@pytest.mark.parametrize("n,sub,radius", [(32, 8, 6), (64, 16, 12), ((40, 36, 44), 8, 6)])
def test_solve_plan_walk_matches_the_factorisation(shim, n, sub, radius):
    """The device solve plans' FP32 blocks Fw = [L_JJ^{-1}; -L_RJ L_JJ^{-1}],
    solved on the host front by front with the kernels' arithmetic (FP64
    accumulation, FP64 vectors between fronts), solve (A + 1e-5 I) x = b like
    the FP64 factorisation itself, up to the FP32 rounding of the stored
    coefficients and of x."""
    d = domains.small(n, sub, radius, seed=4)
    M = d.meta["sigma_levels"]
    h = build(shim, d, M)
    try:
        nn = C.c_int()
        for l in range(M):
            for kind in (0, 1):
                err = shim.shim_plan_check(h, kind, l, C.byref(nn))
                assert 0 <= err < 2e-6, (kind, l, nn.value, err)
    finally:
        shim.shim_free(h)


@pytest.mark.parametrize("ncomp,csize", [(300000, 3), (2000, 40), (37, 33)])
def test_factorisation_of_many_disconnected_pieces(shim, ncomp, csize):
    """The interface system of a sparse domain falls apart into many pieces; the
    ordering visits them in one pass (300000 pieces once overflowed the stack
    by recursing once per piece)."""
    assert 0 <= shim.shim_factor_components(ncomp, csize) < 1e-12


def test_domain_without_active_cells_is_rejected(shim):
    d = domains.small(16, 8, 0, seed=1)
    d.flags[:] = 0
    size = (C.c_int * 3)(*d.size)
    sub = (C.c_int * 3)(*d.sub_size)
    flags = np.ascontiguousarray(d.flags, np.uint32)
    err = C.create_string_buffer(512)
    h = shim.shim_build(size, sub, 3, 2, flags.ctypes.data_as(C.POINTER(C.c_uint32)), err, 512)
    assert not h and b"no Active cells" in err.value


def test_single_subdomain_has_no_level0_interface(shim):
    """A domain inside one subdomain: no level-0 interface DOFs (the solver then
    runs the subdomain V-cycles alone), same as the oracle."""
    d = domains.small(16, 16, 3, seed=1)
    h = build(shim, d, 2)
    try:
        assert shim.shim_num_subdomains(h) == 1
        assert matrix(shim, h, 0, 0).shape == (0, 0)
    finally:
        shim.shim_free(h)
    o = Oracle(d.size, d.sub_size, d.flags, vlevels=3, nVcycles=1, interior_smoothing=3, boundary_smoothing=3,
               sigma_levels=2, sigma_smoothing=3, sigma_mg=1)
    assert o.num_interface(0) == 0


# ---- interface dump / reload (the reference's -iomode output / input) ---------------------


def raw_matrix(L, h, kind, level, sub=0):
    shape = (C.c_int * 3)()
    if L.shim_matrix_shape(h, kind, level, sub, shape) != 0:
        return None
    rows, cols, nnz = shape
    ptr = np.zeros(rows + 1, np.int32)
    col = np.zeros(max(nnz, 1), np.int32)
    val = np.zeros(max(nnz, 1), np.float64)
    L.shim_matrix_get(h, kind, level, sub, ptr.ctypes.data_as(C.POINTER(C.c_int)),
                      col.ctypes.data_as(C.POINTER(C.c_int)), val.ctypes.data_as(C.POINTER(C.c_double)))
    return rows, cols, ptr, col[:nnz], val[:nnz]


def points(L, h, level, sub):
    n = L.shim_positions(h, level, sub, None)
    out = np.zeros((max(n, 0), 3), np.int32)
    if n > 0:
        L.shim_positions(h, level, sub, out.ctypes.data_as(C.POINTER(C.c_int)))
    return out


def imap(L, h):
    n = L.shim_interface_map(h, None)
    out = np.zeros((n, 3), np.int32)
    if n:
        L.shim_interface_map(h, out.ctypes.data_as(C.POINTER(C.c_int)))
    return out


def read_dump(L, path):
    err = C.create_string_buffer(512)
    h = L.shim_read_interface(str(path).encode(), err, 512)
    return h, err.value.decode()


def test_interface_dump_reads_back_unchanged(shim, tmp_path):
    d = domains.small((40, 36, 44), 8, 6, seed=4)
    M = d.meta["sigma_levels"]
    h = build(shim, d, M)
    err = C.create_string_buffer(512)
    try:
        assert shim.shim_write_interface(h, str(tmp_path).encode(), err, 512) == 0, err.value
        h2, msg = read_dump(shim, tmp_path)
        assert h2, msg
        try:
            nsub = shim.shim_num_subdomains(h)
            assert shim.shim_num_subdomains(h2) == nsub
            for l in range(M):
                mats = [(0, 0)] + ([(3, 0)] if l + 1 < M else []) + [(k, s) for s in range(nsub) for k in (1, 2)]
                for kind, sub in mats:
                    a, b = raw_matrix(shim, h, kind, l, sub), raw_matrix(shim, h2, kind, l, sub)
                    assert a[:2] == b[:2], (kind, l, sub)
                    for x, y in zip(a[2:], b[2:]):
                        assert np.array_equal(x, y), (kind, l, sub)
                assert np.array_equal(points(shim, h, l, -1), points(shim, h2, l, -1))
                for s in range(nsub):
                    assert np.array_equal(points(shim, h, l, s), points(shim, h2, l, s))
            assert np.array_equal(imap(shim, h), imap(shim, h2))
            assert shim.shim_check_interface(h, h2, M, err, 512) == 0, err.value
        finally:
            shim.shim_free(h2)
    finally:
        shim.shim_free(h)


def _market(path):
    lines = open(path).read().splitlines()
    rows, cols, nnz = (int(v) for v in lines[1].split())
    ent = np.array([ln.split() for ln in lines[2:]], dtype=object).reshape(-1, 3)
    return lines[0], (rows, cols, nnz), ent[:, 0].astype(int), ent[:, 1].astype(int), ent[:, 2].astype(np.float32)


def test_interface_dump_follows_the_reference_layout(shim, tmp_path):
    """levels / number_of_subdomains (int32), Matrix Market Aii/Arr in column-major
    and Air/Prr in row-major entry order with 1-based indices, interface_map as a
    uint64 count and int32 triples (INTERFACE_SOLVER_DATA.h:177-212,
    INTERFACE_MATRIX_GENERATOR.h:66-72)."""
    d = domains.small(32, 8, 6, seed=4)
    M = d.meta["sigma_levels"]
    h = build(shim, d, M)
    err = C.create_string_buffer(512)
    try:
        assert shim.shim_write_interface(h, str(tmp_path).encode(), err, 512) == 0, err.value
        nsub = shim.shim_num_subdomains(h)
        assert np.fromfile(tmp_path / "levels", np.int32).tolist() == [M]
        assert np.fromfile(tmp_path / "number_of_subdomains", np.int32).tolist() == [nsub]
        for name, kind, sub, col_major in (("Arr_0", 0, 0, True), ("Aii_0_3", 1, 3, True),
                                           ("Air_0_3", 2, 3, False), ("Prr_0", 3, 0, False)):
            head, shape, r, c, v = _market(tmp_path / name)
            assert head == "%%MatrixMarket matrix coordinate real general"
            ref = matrix(shim, h, kind, 0, sub).tocoo()
            assert shape == (ref.shape[0], ref.shape[1], ref.nnz) and len(r) == ref.nnz
            assert r.min() >= 1 and c.min() >= 1
            outer = c if col_major else r
            assert np.all(np.diff(outer) >= 0), name
            got = sp.csr_matrix((v.astype(np.float64), (r - 1, c - 1)), shape=ref.shape)
            assert (got != ref.tocsr()).nnz == 0, name
        raw = (tmp_path / "interface_map").read_bytes()
        n = int(np.frombuffer(raw[:8], np.uint64)[0])
        assert len(raw) == 8 + 12 * n
        assert np.array_equal(np.frombuffer(raw[8:], np.int32).reshape(n, 3), imap(shim, h))
    finally:
        shim.shim_free(h)


def test_reload_reads_hand_written_market_files(shim, tmp_path):
    """A one-subdomain dump written by hand the way Eigen's saveMarket writes it:
    comment lines, a symmetric header storing one triangle, duplicate entries
    summed."""
    np.array([1], np.int32).tofile(tmp_path / "levels")
    np.array([1], np.int32).tofile(tmp_path / "number_of_subdomains")
    (tmp_path / "Arr_0").write_text("%%MatrixMarket matrix coordinate real symmetric\n% interface\n2 2 3\n"
                                    "1 1 2.0\n2 1 -5.00000000e-01\n2 2 3.0\n")
    (tmp_path / "Aii_0_0").write_text("%%MatrixMarket matrix coordinate real general\n1 1 2\n1 1 1.5\n1 1 0.25\n")
    (tmp_path / "Air_0_0").write_text("%%MatrixMarket matrix coordinate real general\n1 2 1\n1 2 -0.125\n")
    with open(tmp_path / "interface_map", "wb") as f:
        np.array([2], np.uint64).tofile(f)
        np.array([[0, 0, 4], [0, 0, 8]], np.int32).tofile(f)
    h, msg = read_dump(shim, tmp_path)
    assert h, msg
    try:
        assert np.array_equal(matrix(shim, h, 0, 0).toarray(), [[2.0, -0.5], [-0.5, 3.0]])
        assert np.array_equal(matrix(shim, h, 1, 0, 0).toarray(), [[1.75]])
        assert np.array_equal(matrix(shim, h, 2, 0, 0).toarray(), [[0.0, -0.125]])
        assert imap(shim, h).tolist() == [[0, 0, 4], [0, 0, 8]]
        # No positions file: the level-0 interface positions are the interface cells.
        assert points(shim, h, 0, -1).tolist() == [[0, 0, 4], [0, 0, 8]]
    finally:
        shim.shim_free(h)


def test_reload_errors(shim, tmp_path):
    d = domains.small(32, 8, 6, seed=4)
    M = d.meta["sigma_levels"]
    h = build(shim, d, M)
    err = C.create_string_buffer(512)
    try:
        h0, msg = read_dump(shim, tmp_path / "missing")
        assert not h0 and "cannot open" in msg
        assert shim.shim_write_interface(h, str(tmp_path).encode(), err, 512) == 0, err.value
        h2, msg = read_dump(shim, tmp_path)
        assert h2, msg
        try:
            # A dump of another sigma hierarchy depth, or of another domain, is refused.
            assert shim.shim_check_interface(h, h2, M + 1, err, 512) == 1 and b"levels" in err.value
            other = build(shim, domains.small(32, 16, 5, seed=4), M)
            try:
                assert shim.shim_check_interface(other, h2, M, err, 512) == 1 and b"subdomains" in err.value
            finally:
                shim.shim_free(other)
        finally:
            shim.shim_free(h2)
        (tmp_path / "Arr_0").write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n")
        h3, msg = read_dump(shim, tmp_path)
        assert not h3 and "fewer entries" in msg
    finally:
        shim.shim_free(h)


# ---- SPGrid pages (hdd_set_domain_pages / hdd_get_solution_pages) ------------------------


def _u32(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _f32(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i32(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def test_pages_scatter_and_gather(shim):
    d = domains.small((37, 30, 21), 8, 5, seed=2)   # ragged: the last pages reach past the grid
    origin, fp, rp = domains.to_pages(d.flags, d.rhs)
    rng = np.random.default_rng(0)
    order = rng.permutation(len(origin))          # pages in any order
    origin, fp, rp = (np.ascontiguousarray(a[order]) for a in (origin, fp, rp))
    # A page wholly outside the grid is skipped.
    origin = np.vstack([origin, [[40, 0, 0]]]).astype(np.int32)
    fp = np.vstack([fp, np.full((1, 256), 0x10000, np.uint32)])
    rp = np.vstack([rp, np.ones((1, 256), np.float32)])
    size = (C.c_int * 3)(*d.size)
    df = np.zeros(d.size, np.uint32)
    dr = np.zeros(d.size, np.float32)
    err = C.create_string_buffer(256)
    assert shim.shim_pages_to_dense(size, len(origin), _i32(origin), _u32(fp), _f32(rp), _u32(df), _f32(dr),
                                    err, 256) == 0, err.value
    assert np.array_equal(df, d.flags) and np.array_equal(dr, d.rhs)
    # Gather: cell (x, y, z) of page p at (x*8 + y)*8 + z; 0 outside the grid.
    back = np.full((len(origin), 256), np.nan, np.float32)
    assert shim.shim_dense_to_pages(size, len(origin), _i32(origin), _f32(dr), _f32(back)) == 0
    for p in (0, len(origin) // 2, len(origin) - 1):
        for x, y, z in ((0, 0, 0), (3, 7, 7), (1, 5, 2)):
            i, j, k = origin[p] + (x, y, z)
            want = dr[i, j, k] if i < d.size[0] and j < d.size[1] and k < d.size[2] else 0.0
            assert back[p, (x * 8 + y) * 8 + z] == want


@pytest.mark.parametrize("origin,msg", [([[4, 8, 8], [4, 8, 8]], b"twice"), ([[2, 0, 0]], b"multiple"),
                                        ([[0, -8, 0]], b"negative")])
def test_bad_page_lists_are_refused(shim, origin, msg):
    origin = np.array(origin, np.int32)
    size = (C.c_int * 3)(17, 17, 17)
    v = np.zeros((len(origin), 256), np.uint32)
    f = np.zeros((len(origin), 256), np.float32)
    df = np.zeros((17, 17, 17), np.uint32)
    dr = np.zeros((17, 17, 17), np.float32)
    err = C.create_string_buffer(256)
    assert shim.shim_pages_to_dense(size, len(origin), _i32(origin), _u32(v), _f32(f), _u32(df), _f32(dr),
                                    err, 256) == 1
    assert msg in err.value




def test_setup_bits_do_not_depend_on_thread_count(shim):
    """Interface assembly, orderings, factorisations and solve blocks are split
    over OpenMP threads; every value is computed in the same order whatever the
    thread count, so the digest of all of them is the same for 1, 3 and 8
    threads (each run in its own process, where OMP_NUM_THREADS takes effect)."""
    import subprocess
    import sys
    code = (
        "import ctypes as C, sys, numpy as np\n"
        f"sys.path.insert(0, {os.path.join(ROOT)!r})\n"
        "from hierarchicaldd_b200 import domains\n"
        f"L = C.CDLL({SHIM!r})\n"
        "ip = C.POINTER(C.c_int)\n"
        "L.shim_build.restype = C.c_void_p\n"
        "L.shim_build.argtypes = [ip, ip, C.c_int, C.c_int, C.POINTER(C.c_uint32), C.c_char_p, C.c_int]\n"
        "L.shim_setup_digest.restype = C.c_ulonglong\n"
        "L.shim_setup_digest.argtypes = [C.c_void_p]\n"
        "d = domains.small(96, 16, 20, seed=6)\n"
        "f = np.ascontiguousarray(d.flags, np.uint32)\n"
        "err = C.create_string_buffer(256)\n"
        "h = L.shim_build((C.c_int * 3)(*d.size), (C.c_int * 3)(*d.sub_size), 3, 2,"
        " f.ctypes.data_as(C.POINTER(C.c_uint32)), err, 256)\n"
        "assert h, err.value\n"
        "print(L.shim_setup_digest(h))\n")
    digests = set()
    for threads in ("1", "3", "8"):
        env = dict(os.environ, OMP_NUM_THREADS=threads)
        p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
        assert p.returncode == 0, p.stderr
        digests.add(p.stdout.strip())
    assert len(digests) == 1, digests


@pytest.mark.parametrize("sub", [4, 64])
def test_unsupported_sub_sizes_are_refused_before_setup(shim, sub):
    """The resident V-cycle handles 8^3, 16^3 and 32^3 subdomains; 4 and the
    reference Test_Bench default 64 are refused by the layout, before any
    interface assembly or factorisation."""
    d = domains.small(64, 16, 12, seed=4)
    size = (C.c_int * 3)(*d.size)
    sb = (C.c_int * 3)(sub, sub, sub)
    flags = np.ascontiguousarray(d.flags, np.uint32)
    err = C.create_string_buffer(512)
    h = shim.shim_build(size, sb, 2, 2, flags.ctypes.data_as(C.POINTER(C.c_uint32)), err, 512)
    assert not h
    assert b"sub_size must be 8, 16 or 32" in err.value, err.value
