"""The sparse sphere-union workload built as SPGrid pages (config5_pages, which
never holds dense flag or right-hand-side arrays of the box) equals the pages
of the dense build (config5, then to_pages) bit for bit: page list, flags and
right-hand side.  The GPU takes the paged form through hdd_set_domain_pages
(tests/test_gpu_c5_parity.py, test_gpu_pages.py)."""
import numpy as np
import pytest

from hierarchicaldd_b200 import domains


@pytest.mark.parametrize("scale", [8, 4])
def test_paged_sparse_workload_equals_dense_build(scale):
    d = domains.config5(scale)
    p = domains.config5_pages(scale)
    origin, fpages, rpages = domains.to_pages(d.flags, d.rhs)
    assert p.size == d.size and p.sub_size == d.sub_size and p.name == d.name and p.meta == d.meta
    assert np.array_equal(p.origin, origin)
    assert np.array_equal(p.flags, fpages)
    assert np.array_equal(p.rhs.view(np.uint32), rpages.view(np.uint32))
    # Only pages holding a cell of the union are kept.
    box_pages = int(np.prod([-(-n // b) for n, b in zip(d.size, (4, 8, 8))]))
    assert 0 < len(p.origin) < box_pages
    assert np.count_nonzero(p.flags & domains.ACTIVE) == np.count_nonzero(d.flags & domains.ACTIVE)


def test_slab_pages_round_trip():
    rng = np.random.default_rng(1)
    a = (rng.random((13, 21, 17)) < 0.05).astype(np.uint32) * 7
    keep, origin, pages = domains._slab_pages(a, 8, a.shape[1:])
    full = np.zeros((16, 24, 24), np.uint32)
    for (x, y, z), pg in zip(origin, pages):
        full[x - 8:x - 4, y:y + 8, z:z + 8] = pg.reshape(4, 8, 8)
    assert np.array_equal(full[:13, :21, :17], a)
    assert len(keep) == len(origin) == len(pages)


def test_bench_hands_the_sparse_workloads_over_as_pages(monkeypatch):
    import bench
    calls = []

    class FakeSolver:
        def Set_Domain_Pages(self, origin, flags, rhs):
            calls.append(("pages", len(origin)))

        def Set_Domain(self, flags, rhs):
            calls.append(("dense", flags.shape))

    p = domains.config5_pages(8)
    bench.set_domain(FakeSolver(), p)
    d = domains.config5(8)
    bench.set_domain(FakeSolver(), d)
    assert calls == [("pages", len(p.origin)), ("dense", d.size)]
    monkeypatch.setattr(domains, "config5_pages", lambda scale: ("paged", scale))
    assert bench.workload("c5") == ("paged", 1)
    assert bench.workload("c5_half") == ("paged", 2)
