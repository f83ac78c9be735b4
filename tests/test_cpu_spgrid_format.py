"""CPU checks of the SPGrid directory format helper (no GPU): the page offset
masks interleave coordinates as the reference's SPGrid_Mask<4,2,3> does, and a
written directory reads back to the same dense flags and data."""
import numpy as np

from hierarchicaldd_b200 import domains
from spgrid_format import XM, YM, ZM, pdep, pext, read_spgrid_dir, write_spgrid_dir


def test_masks_partition_the_address_bits():
    assert XM & YM == 0 and XM & ZM == 0 and YM & ZM == 0
    # Within a 4 KB page the flags field (4-byte elements) uses bits 2..9:
    # z bits 2-4, y bits 5-7, x bits 8-9.
    assert (XM | YM | ZM) & 0xFFF == 0x3FC
    for x, y, z in [(0, 0, 0), (3, 7, 7), (4, 8, 8), (13, 22, 31), (64, 64, 64)]:
        off = pdep(x, XM) | pdep(y, YM) | pdep(z, ZM)
        assert (pext(off, XM), pext(off, YM), pext(off, ZM)) == (x, y, z)


def test_round_trip(tmp_path):
    d = domains.small(16, 8, 3, seed=2)
    padded = write_spgrid_dir(str(tmp_path), d.flags, d.rhs)
    assert all(p % b == 0 and p >= n for p, b, n in zip(padded, (4, 8, 8), d.size))
    flags, data = read_spgrid_dir(str(tmp_path), d.size)
    assert np.array_equal(flags, d.flags)
    assert np.array_equal(data, d.rhs)
