"""The reference's SPGrid directory format, written and read in Python (test helper).

Restates SPGRID_READ_WRITE::Write_SPGrid / Read_SPGrid
(demos/SPGrid_Create_Simple_Domain/SPGRID_READ_WRITE.h:43-106) for 3D grids:

* `size`: the allocator's padded size, 3 int32 (here: rounded up to whole blocks);
* `block_offset`: int32 block count, then a PhysBAM array (int32 length + one uint64
  offset per block) of the flags array's page offsets;
* `flags` / `data`: per block a PhysBAM array (int32 length 256 + 256 4-byte values).

A block (page) is 4 x 8 x 8 cells of a 16-byte cell struct, the 4-byte fields stored
field after field inside the 4 KB page; the 64-bit offset interleaves the cell
coordinates with the masks below (SPGrid_Mask<4,2,3>, PB/Common_Libraries/SPGrid/Core/
SPGrid_Mask.h:25-31,74-78).
"""
import os
import struct

import numpy as np

XM = 0x9249249249249000 | 0x300
YM = 0x4924924924924000 | 0x0E0
ZM = 0x2492492492492000 | 0x01C
BLOCK = (4, 8, 8)


def pdep(v, mask):
    """Deposit the low bits of v onto the set bits of mask, lowest first."""
    r, m = 0, mask
    while m:
        low = m & -m
        if v & 1:
            r |= low
        v >>= 1
        m &= m - 1
    return r


def pext(v, mask):
    r, bit, m = 0, 1, mask
    while m:
        low = m & -m
        if v & low:
            r |= bit
        bit <<= 1
        m &= m - 1
    return r


def write_spgrid_dir(path, flags, data):
    """Blocks holding any non-zero flag are written, in offset order."""
    os.makedirs(path, exist_ok=True)
    n = flags.shape
    padded = tuple(-(-n[a] // BLOCK[a]) * BLOCK[a] for a in range(3))
    blocks = []
    for bx in range(0, n[0], BLOCK[0]):
        for by in range(0, n[1], BLOCK[1]):
            for bz in range(0, n[2], BLOCK[2]):
                f = flags[bx:bx + 4, by:by + 8, bz:bz + 8]
                if np.any(f):
                    blocks.append((pdep(bx, XM) | pdep(by, YM) | pdep(bz, ZM), bx, by, bz))
    blocks.sort()
    with open(os.path.join(path, "size"), "wb") as fh:
        fh.write(struct.pack("<3i", *padded))
    with open(os.path.join(path, "block_offset"), "wb") as fh:
        fh.write(struct.pack("<ii", len(blocks), len(blocks)))
        fh.write(struct.pack("<%dQ" % len(blocks), *[b[0] for b in blocks]))
    for name, arr, fmt in (("flags", flags, "<256I"), ("data", data, "<256f")):
        with open(os.path.join(path, name), "wb") as fh:
            for _, bx, by, bz in blocks:
                vals = np.zeros(256, arr.dtype)
                for e in range(256):
                    x, y, z = bx + (e >> 6), by + ((e >> 3) & 7), bz + (e & 7)
                    if x < n[0] and y < n[1] and z < n[2]:
                        vals[e] = arr[x, y, z]
                fh.write(struct.pack("<i", 256))
                fh.write(struct.pack(fmt, *vals.tolist()))
    return padded


def read_spgrid_dir(path, size):
    """Dense (flags, data) of the first `size` cells per axis."""
    with open(os.path.join(path, "block_offset"), "rb") as fh:
        count, _ = struct.unpack("<ii", fh.read(8))
        offs = struct.unpack("<%dQ" % count, fh.read(8 * count))
    flags = np.zeros(size, np.uint32)
    data = np.zeros(size, np.float32)
    for name, arr, fmt in (("flags", flags, "<256I"), ("data", data, "<256f")):
        with open(os.path.join(path, name), "rb") as fh:
            for off in offs:
                assert struct.unpack("<i", fh.read(4))[0] == 256
                vals = struct.unpack(fmt, fh.read(1024))
                for e in range(256):
                    lin = off + 4 * e
                    x, y, z = pext(lin, XM), pext(lin, YM), pext(lin, ZM)
                    if x < size[0] and y < size[1] and z < size[2]:
                        arr[x, y, z] = vals[e]
    return flags, data


def axis_masks(dim, log2_struct=4, log2_field=2):
    """Per-axis address masks of SPGrid_Mask<log2_struct, log2_field, dim>
    (PB/Common_Libraries/SPGrid/Core/SPGrid_Mask.h: the 3D masks at :14-31 and
    :56-60, the 2D ones at :308-358), and the block shape.  Inside the 4 KB page
    the element bits sit above the field's byte bits, the last axis lowest; the
    page bits above bit 12 interleave the axes.  The layout has to match the
    reference's for the on-disk format to be read at all."""
    full = (1 << 64) - 1
    block_bits = 12 - log2_struct
    if dim == 3:
        bits = [block_bits // 3, block_bits // 3 + (block_bits % 3 > 1), block_bits // 3 + (block_bits % 3 > 0)]
        sh = 3 - block_bits % 3
        page = [0x4924924924924924, 0x2492492492492492, 0x9249249249249249]
    elif dim == 2:
        bits = [block_bits // 2, block_bits // 2 + (block_bits % 2 > 0)]
        sh = 2 - block_bits % 2
        page = [0xAAAAAAAAAAAAAAAA, 0x5555555555555555]
    else:
        raise ValueError("dim must be 2 or 3")
    masks, shift = [0] * dim, log2_field
    for a in reversed(range(dim)):
        masks[a] = ((page[a] << sh) & full & 0xFFFFFFFFFFFFF000) | (((1 << bits[a]) - 1) << shift)
        shift += bits[a]
    return masks, tuple(1 << b for b in bits)


def read_spgrid_dir_any(path):
    """(size, flags, data, n_blocks) of a 2D or 3D directory; the dimension
    comes from the length of the `size` file; arrays cover the padded size."""
    with open(os.path.join(path, "size"), "rb") as fh:
        raw = fh.read()
    dim = len(raw) // 4
    size = struct.unpack("<%di" % dim, raw)
    masks, block = axis_masks(dim)
    per_block = int(np.prod(block))
    with open(os.path.join(path, "block_offset"), "rb") as fh:
        count, alen = struct.unpack("<ii", fh.read(8))
        assert alen == count
        offs = struct.unpack("<%dQ" % count, fh.read(8 * count))
    flags = np.zeros(size, np.uint32)
    data = np.zeros(size, np.float32)
    elem = np.arange(per_block, dtype=np.uint64) * 4
    for name, arr, dt in (("flags", flags, "<u4"), ("data", data, "<f4")):
        with open(os.path.join(path, name), "rb") as fh:
            buf = fh.read()
        rec = 4 + 4 * per_block
        assert len(buf) == rec * count
        for b, off in enumerate(offs):
            assert struct.unpack_from("<i", buf, b * rec)[0] == per_block
            vals = np.frombuffer(buf, dt, per_block, b * rec + 4)
            idx = tuple(np.array([pext(int(off) + int(e), m) for e in elem]) for m in masks)
            arr[idx] = vals
    return size, flags, data, count
