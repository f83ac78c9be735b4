"""Synthetic Poisson domains for the DD-PCG solver.

The flag rules follow the reference's domain generator
(demos/SPGrid_Create_Simple_Domain/Create_3D_Domain/main.cpp):

* a grid of ``size`` cells per axis, where ``size`` is the cell count plus one
  (the reference's ``-size`` convention), cells indexed ``0 .. size-1``;
* cells on the outer layer (index 0 or size-1) are Dirichlet (main.cpp:118);
* Dirichlet cells without an Active face neighbour become exterior, flag 0
  (main.cpp:126-140);
* Active and Interface cells carry face bits for neighbours that are
  Active|Interface|Dirichlet (main.cpp:299, SPGrid_Flag_Helper.h).

The reference's own generator carves a Neumann (exterior) bubble; the workloads
here place Dirichlet spheres instead, with every seed and shape fixed below.
Random numbers come from numpy's Philox bit generator so that the inputs are the
same on every host.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

ACTIVE = 0x00010000
DIRICHLET = 0x00020000
BOUNDARY = 0x00040000
INTERFACE = 0x00080000
FACE_MX = 0x00100000
FACE_ALL = 0x03F00000


@dataclass
class Domain:
    """One Poisson problem: cell flags and right-hand side on a dense grid."""

    size: tuple          # cells per axis (reference -size, i.e. cell count + 1)
    flags: np.ndarray    # uint32 [size]: Active / Dirichlet / 0, plus face bits
    rhs: np.ndarray      # float32 [size]
    sub_size: tuple = (16, 16, 16)
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n_active(self) -> int:
        return int(np.count_nonzero(self.flags & ACTIVE))


def _neighbour(mask: np.ndarray, axis: int, step: int) -> np.ndarray:
    """mask at cell + step along axis (False outside the grid)."""
    pad = np.pad(mask, 1, constant_values=False)
    sl = [slice(1, 1 + n) for n in mask.shape]
    sl[axis] = slice(1 + step, 1 + step + mask.shape[axis])
    return pad[tuple(sl)]


def face_bits(flags: np.ndarray) -> np.ndarray:
    """OR face bits into Active|Interface cells (SPGrid_Flag_Helper.h:74-106):
    bit FACE_MX << k for the faces -x, +x, -y, +y (, -z, +z) whose neighbour is
    Active, Interface or Dirichlet.  2D or 3D."""
    f = flags.copy()
    nb_ok = (f & (ACTIVE | INTERFACE | DIRICHLET)) != 0
    solve = (f & (ACTIVE | INTERFACE)) != 0
    for k in range(2 * f.ndim):
        f[solve & _neighbour(nb_ok, k // 2, 1 if k % 2 else -1)] |= np.uint32(FACE_MX << k)
    return f


def reference_generator(size, delta) -> Domain:
    """The reference's own test domain (Create_2D_Domain / Create_3D_Domain
    main.cpp, Rasterizer::Consume at :100-149): a box whose outer cell layer is
    Dirichlet and whose centre holds a Neumann bubble, with the right-hand side
    4.0 at ``delta`` (main.cpp:282-287).  2D or 3D.

    The rasterizer's grid is PhysBAM's GRID of size-2 nodes on the unit box,
    so dx = 1/(size-3) and cell c has centre (c - 0.5) dx, in float; cells with
    |centre - 0.5|^2 <= 0.09 are exterior (flag 0).  Dirichlet cells without an
    Active face neighbour are exterior too, and face bits follow Flaging.  The
    reference's shipped 2D output (256 x 256) decodes to exactly this.

    Exterior cells touch Active ones here, which couples subdomain boxes at the
    coarse V-cycle levels: the solver runs its whole-grid V-cycle for them."""
    n = tuple(int(v) for v in size)
    grids = np.ogrid[tuple(slice(0, v) for v in n)]
    d2 = np.float32(0)
    interior = True
    for a, g in enumerate(grids):
        dx = np.float32(1) / np.float32(n[a] - 3)
        x = (g.astype(np.float32) - np.float32(0.5)) * dx - np.float32(0.5)
        d2 = d2 + x * x
        interior = interior & (g >= 1) & (g <= n[a] - 2)
    active = interior & ~(d2 <= np.float32(0.09))
    touches = np.zeros(n, bool)
    for a in range(len(n)):
        touches |= _neighbour(active, a, -1) | _neighbour(active, a, 1)
    flags = np.zeros(n, np.uint32)
    flags[active] = ACTIVE
    flags[~interior & touches] = DIRICHLET
    flags = face_bits(flags)
    rhs = np.zeros(n, np.float32)
    if flags[tuple(delta)] == 0:
        raise ValueError("the delta must sit on a non-exterior cell (main.cpp:286 asserts it)")
    rhs[tuple(delta)] = 4.0
    return Domain(n, flags, rhs, name="reference_bubble_" + "x".join(map(str, n)))


def _finish(active: np.ndarray, dirichlet: np.ndarray) -> np.ndarray:
    """Apply the generator's exterior rule and face bits."""
    flags = np.zeros(active.shape, np.uint32)
    flags[active] = ACTIVE
    flags[dirichlet & ~active] = DIRICHLET
    # Dirichlet cells with no Active face neighbour become exterior (flag 0).
    pad = np.pad(active, 1, constant_values=False)
    n0, n1, n2 = active.shape
    has_active_nb = np.zeros_like(active)
    for a, b, c in [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]:
        has_active_nb |= pad[1 + a:1 + a + n0, 1 + b:1 + b + n1, 1 + c:1 + c + n2]
    flags[(flags == DIRICHLET) & ~has_active_nb] = 0
    return face_bits(flags)


def box_with_spheres(size, spheres) -> np.ndarray:
    """Flags for a box with Dirichlet outer layer and Dirichlet spheres.

    ``spheres`` is a list of ``(centre_xyz, radius)``; a cell (i, j, k) is inside
    when ``|(i, j, k) - centre|^2 <= radius^2``.
    """
    n = tuple(int(s) for s in size)
    i, j, k = np.ogrid[0:n[0], 0:n[1], 0:n[2]]
    outer = (i == 0) | (i == n[0] - 1) | (j == 0) | (j == n[1] - 1) | (k == 0) | (k == n[2] - 1)
    inside = np.zeros(n, bool)
    for (cx, cy, cz), r in spheres:
        inside |= (i - cx) ** 2 + (j - cy) ** 2 + (k - cz) ** 2 <= r * r
    dirichlet = outer | inside
    active = ~dirichlet
    return _finish(active, dirichlet)


def config1() -> Domain:
    """64^3 cells (size 65), Dirichlet sphere c=(32,32,32) r=12, delta 1.0 at (16,16,16)."""
    size = (65, 65, 65)
    flags = box_with_spheres(size, [((32, 32, 32), 12)])
    rhs = np.zeros(size, np.float32)
    rhs[16, 16, 16] = 1.0
    return Domain(size, flags, rhs, (16, 16, 16), "c1_64cube_sub16",
                  dict(vlevels=3, nVcycles=1, interior_smoothing=3, boundary_smoothing=3,
                       sigma_levels=3, sigma_smoothing=3, sigma_mg=1))


def config2() -> Domain:
    """256^3 cells (size 257), sphere c=(128,128,128) r=48, delta at (64,64,64) + U[-1e-3,1e-3]."""
    size = (257, 257, 257)
    flags = box_with_spheres(size, [((128, 128, 128), 48)])
    rng = np.random.Generator(np.random.Philox(2))
    noise = rng.uniform(-1e-3, 1e-3, size).astype(np.float32)
    rhs = np.where((flags & ACTIVE) != 0, noise, np.float32(0)).astype(np.float32)
    rhs[64, 64, 64] += np.float32(1.0)
    return Domain(size, flags, rhs, (32, 32, 32), "c2_256cube_sub32",
                  dict(vlevels=4, nVcycles=1, interior_smoothing=4, boundary_smoothing=4,
                       sigma_levels=4, sigma_smoothing=3, sigma_mg=1))


def config3() -> Domain:
    """384^3 cells (size 385), sphere scaled from config 2 (r=72), 8 Gaussian sources (sigma 6)."""
    size = (385, 385, 385)
    flags = box_with_spheres(size, [((192, 192, 192), 72)])
    rng = np.random.Generator(np.random.Philox(3))
    act = np.argwhere((flags & ACTIVE) != 0)
    centres = act[rng.integers(0, len(act), 8)]
    i, j, k = np.ogrid[0:size[0], 0:size[1], 0:size[2]]
    rhs = np.zeros(size, np.float32)
    for c in centres:
        rhs += np.exp(-((i - c[0]) ** 2 + (j - c[1]) ** 2 + (k - c[2]) ** 2) / (2 * 36.0)).astype(np.float32)
    rhs[(flags & ACTIVE) == 0] = 0
    return Domain(size, flags, rhs, (32, 32, 32), "c3_384cube_sub32",
                  dict(vlevels=4, nVcycles=1, interior_smoothing=4, boundary_smoothing=4,
                       sigma_levels=4, sigma_smoothing=3, sigma_mg=1, true_residual_every=20))


def config5(scale: int = 1) -> Domain:
    """Sparse domain: a 1024^3-cell bounding box (size 1025) holding the union of
    64 spheres, radii U[40, 120] cells, centres uniform in the box (Philox seed
    5), about a tenth of the box.  Union cells with a face neighbour outside the
    union are Dirichlet, the other union cells Active, everything else exterior
    (flag 0), so SPGrid pages away from the spheres hold nothing.  Right-hand
    side U[0, 1] on the Active cells minus its mean there.  Subdomains 32^3,
    vlevels 5, mixed precision.  The workload asks for 5 sigma levels, but a
    32^3 subdomain's adaptive interface hierarchy has 4, and the reference
    refuses more (INTERFACE_MATRIX_GENERATOR.h:143), so sigma_levels is 4.
    ``scale`` = 2, 4, ... divides the box and the radii (same seeds) for
    smaller runs of the same shape."""
    n = 1024 // scale
    size = (n + 1,) * 3
    rng = np.random.Generator(np.random.Philox(5))
    union = np.zeros(size, bool)
    for _ in range(64):
        c = rng.uniform(0, n, 3)
        r = rng.uniform(40, 120) / scale
        lo = np.maximum(np.floor(c - r).astype(int), 0)
        hi = np.minimum(np.ceil(c + r).astype(int) + 1, n + 1)
        i, j, k = np.ogrid[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        union[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] |= (i - c[0]) ** 2 + (j - c[1]) ** 2 + (k - c[2]) ** 2 <= r * r
    interior = union.copy()
    for axis in range(3):
        for step in (-1, 1):
            interior &= _neighbour(union, axis, step)
    flags = _finish(interior, union & ~interior)
    act = (flags & ACTIVE) != 0
    vals = rng.uniform(0, 1, int(act.sum()))
    rhs = np.zeros(size, np.float32)
    rhs[act] = (vals - vals.mean()).astype(np.float32)
    tag = f"c5_{n}box_sparse_sub32" if scale > 1 else "c5_1024box_sparse_sub32"
    return Domain(size, flags, rhs, (32, 32, 32), tag,
                  dict(vlevels=5, nVcycles=1, interior_smoothing=3, boundary_smoothing=3, sigma_levels=4,
                       sigma_smoothing=3, sigma_mg=1, precision_mode=1, true_residual_every=20))


@dataclass
class PagedDomain:
    """A domain held only as SPGrid pages (4 x 8 x 8 cells), as
    hdd_set_domain_pages takes it: origin (n, 3), flags and rhs (n, 256) with
    cell (x, y, z) of a page at (x*8 + y)*8 + z; pages without a non-zero flag
    are absent."""
    size: tuple
    origin: np.ndarray   # int32 (n, 3)
    flags: np.ndarray    # uint32 (n, 256)
    rhs: np.ndarray      # float32 (n, 256)
    sub_size: tuple
    name: str
    meta: dict = field(default_factory=dict)


def _slab_pages(a: np.ndarray, x0: int, yz: tuple, keep=None):
    """The x-slab a (cells x0 .. x0 + a.shape[0], x0 a multiple of 4) as pages:
    (the page indices kept within the slab, their origins, the page arrays),
    in to_pages() order.  keep None keeps the pages with a non-zero cell."""
    px, py, pz = -(-a.shape[0] // 4) * 4, -(-yz[0] // 8) * 8, -(-yz[1] // 8) * 8
    p = np.zeros((px, py, pz), a.dtype)
    p[:a.shape[0], :yz[0], :yz[1]] = a
    nb = (px // 4, py // 8, pz // 8)
    b = p.reshape(nb[0], 4, nb[1], 8, nb[2], 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1, 256)
    if keep is None:
        keep = np.flatnonzero(b.any(axis=1))
    origin = np.stack(np.unravel_index(keep, nb), axis=1) * np.array([4, 8, 8])
    origin[:, 0] += x0
    return keep, origin.astype(np.int32), b[keep]


def config5_pages(scale: int = 1) -> PagedDomain:
    """config5(scale) built as SPGrid pages without dense flag or right-hand
    side arrays of the box: the same spheres, rules and random draws, so its
    pages equal to_pages() of config5(scale) bit for bit.  Only the union
    mask of the box is dense (1 byte a cell, 1.1 GB at full scale); flags are
    made 64-cell x-slab by x-slab (with a 3-cell halo, the reach of the
    interior, exterior and face-bit rules) and kept as pages, and the
    right-hand side is drawn in one piece (8 bytes an Active cell) and spread
    into the pages slab by slab in the box's x-slowest order."""
    n = 1024 // scale
    size = (n + 1,) * 3
    rng = np.random.Generator(np.random.Philox(5))
    union = np.zeros(size, bool)
    for _ in range(64):
        c = rng.uniform(0, n, 3)
        r = rng.uniform(40, 120) / scale
        lo = np.maximum(np.floor(c - r).astype(int), 0)
        hi = np.minimum(np.ceil(c + r).astype(int) + 1, n + 1)
        i, j, k = np.ogrid[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        union[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] |= (i - c[0]) ** 2 + (j - c[1]) ** 2 + (k - c[2]) ** 2 <= r * r
    X, yz = size[0], size[1:]
    slabs = []   # (x0, depth, kept page indices, origins, flag pages, packed Active mask)
    total = 0
    for x0 in range(0, X, 64):
        x1 = min(x0 + 64, X)
        w0, w1 = max(x0 - 3, 0), min(x1 + 3, X)
        u = union[w0:w1]
        interior = u.copy()
        for axis in range(3):
            for step in (-1, 1):
                interior &= _neighbour(u, axis, step)
        fl = _finish(interior, u & ~interior)[x0 - w0:x1 - w0]
        act = (fl & ACTIVE) != 0
        total += int(np.count_nonzero(act))
        keep, origin, fpages = _slab_pages(fl, x0, yz)
        slabs.append((x0, x1 - x0, keep, origin, fpages, np.packbits(act)))
    del union
    vals = rng.uniform(0, 1, total)
    mean = vals.mean()
    rpages, off = [], 0
    for x0, depth, keep, _, _, packed in slabs:
        act = np.unpackbits(packed, count=depth * yz[0] * yz[1]).astype(bool).reshape(depth, *yz)
        cnt = int(np.count_nonzero(act))
        r = np.zeros(act.shape, np.float32)
        r[act] = (vals[off:off + cnt] - mean).astype(np.float32)
        off += cnt
        rpages.append(_slab_pages(r, x0, yz, keep)[2])
    origin = np.concatenate([sl[3] for sl in slabs]).astype(np.int32)
    flags = np.concatenate([sl[4] for sl in slabs]).astype(np.uint32)
    rhs = np.concatenate(rpages).astype(np.float32)
    tag = f"c5_{n}box_sparse_sub32" if scale > 1 else "c5_1024box_sparse_sub32"
    return PagedDomain(size, origin, flags, rhs, (32, 32, 32), tag,
                       dict(vlevels=5, nVcycles=1, interior_smoothing=3, boundary_smoothing=3, sigma_levels=4,
                            sigma_smoothing=3, sigma_mg=1, precision_mode=1, true_residual_every=20))


def profile_case() -> Domain:
    """128^3 cells (size 129), centred Dirichlet sphere r=24, 32^3 subdomains:
    the 256^3 workload's kernels (sub 32, vlevels 4, smoothing 4/4) on an eighth
    of its cells, small enough for multi-pass profiler captures."""
    d = small(128, 32, 24, seed=5)
    d.meta.update(vlevels=4, interior_smoothing=4, boundary_smoothing=4, sigma_levels=3)
    return Domain(d.size, d.flags, d.rhs, d.sub_size, "p128_128cube_sub32", d.meta)


# The two-level demo's Test_Bench defaults
# (demos/Domain_Decomposition_CPU_Only_Two_Levels/Test_Bench_3D/main.cpp:236-251)
# with -multilevel yes: 64^3 subdomains, each solved by a DD of 32^3 boxes.
TWO_LEVEL_DEFAULTS = dict(vlevels=3, nVcycles=1, interior_smoothing=1, boundary_smoothing=3,
                          sigma_levels=3, sigma_smoothing=3, sigma_mg=1, multilevel=True)


def two_level_case() -> Domain:
    """128^3 cells (size 129), centred Dirichlet sphere r=24, U[-1, 1] right-hand
    side (Philox seed 11), 64^3 subdomains, two-level DD at the demo's defaults."""
    d = small(128, 64, 24, seed=11)
    return Domain(d.size, d.flags, d.rhs, d.sub_size, "tl128_128cube_sub64_two_level", dict(TWO_LEVEL_DEFAULTS))


def config2_two_level() -> Domain:
    """The 256^3 workload's domain and right-hand side (config2) solved by
    two-level DD at the demo's defaults: 64^3 subdomains split into 32^3 boxes."""
    d = config2()
    return Domain(d.size, d.flags, d.rhs, (64, 64, 64), "c2_256cube_sub64_two_level", dict(TWO_LEVEL_DEFAULTS))


SERVING_SIDES = (64, 96, 128, 192)


def serving_mix(n_domains=4, seed=4, sides=SERVING_SIDES) -> list:
    """Uneven domains for the serving workload: cube side drawn from ``sides``
    (cycled, so every side appears), 1-4 Dirichlet spheres with radii
    U[0.05, 0.2] * side at uniform-random centres, subdomains 16^3 for sides
    below 128 and 32^3 from 128 up, mixed precision with a true residual every
    20 iterations.  The right-hand side is 1-3 unit deltas at random Active cells
    (``serving_rhs`` draws more)."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for n in range(n_domains):
        side = int(sides[n % len(sides)])
        size = (side + 1,) * 3
        spheres = []
        for _ in range(int(rng.integers(1, 5))):
            c = tuple(int(v) for v in rng.integers(1, side, 3))
            spheres.append((c, float(rng.uniform(0.05, 0.2)) * side))
        flags = box_with_spheres(size, spheres)
        sub = 16 if side < 128 else 32
        meta = (dict(vlevels=3, nVcycles=1, interior_smoothing=3, boundary_smoothing=3, sigma_levels=3,
                     sigma_smoothing=3, sigma_mg=1) if sub == 16 else
                dict(vlevels=4, nVcycles=1, interior_smoothing=4, boundary_smoothing=4, sigma_levels=3,
                     sigma_smoothing=3, sigma_mg=1))
        meta.update(precision_mode=1, true_residual_every=20)
        d = Domain(size, flags, np.zeros(size, np.float32), (sub,) * 3, f"serve{n}_{side}cube_sub{sub}", meta)
        d.rhs = serving_rhs(d, rng)
        out.append(d)
    return out


def serving_rhs(d: Domain, rng) -> np.ndarray:
    """1-3 unit deltas at uniform-random Active cells of ``d``."""
    act = np.flatnonzero((d.flags & ACTIVE) != 0)
    rhs = np.zeros(d.size, np.float32)
    rhs.reshape(-1)[act[rng.integers(0, len(act), int(rng.integers(1, 4)))]] = 1.0
    return rhs


def small(n_cells=32, sub=8, radius=6, seed=0, delta=None) -> Domain:
    """A small test domain: an n_cells^3 box (or n_cells = (nx, ny, nz) for a
    ragged one, whose last subdomains are partial), one centred Dirichlet sphere,
    random RHS."""
    cells = tuple(n_cells) if isinstance(n_cells, (tuple, list)) else (n_cells,) * 3
    size = tuple(n + 1 for n in cells)
    centre = tuple(n // 2 for n in cells)
    flags = box_with_spheres(size, [(centre, radius)] if radius > 0 else [])
    rng = np.random.Generator(np.random.Philox(seed))
    rhs = rng.uniform(-1, 1, size).astype(np.float32)
    rhs[(flags & ACTIVE) == 0] = 0
    if delta is not None:
        rhs[:] = 0
        rhs[delta] = 1.0
    tag = "x".join(str(n) for n in cells) if len(set(cells)) > 1 else str(cells[0])
    return Domain(size, flags, rhs, (sub, sub, sub), f"small{tag}_sub{sub}",
                  dict(vlevels=3, nVcycles=1, interior_smoothing=3, boundary_smoothing=3,
                       sigma_levels=2, sigma_smoothing=3, sigma_mg=1))


def to_pages(flags: np.ndarray, *fields: np.ndarray):
    """SPGrid pages (4 x 8 x 8 cells) of a dense domain, as hdd_set_domain_pages
    takes them: the pages holding a non-zero flag, their origins (n, 3) and each
    array as (n, 256) with cell (x, y, z) of a page at (x*8 + y)*8 + z."""
    dims = (4, 8, 8)
    size = flags.shape
    padded = tuple(-(-n // d) * d for n, d in zip(size, dims))

    def blocks(a):
        p = np.zeros(padded, a.dtype)
        p[:size[0], :size[1], :size[2]] = a
        p = p.reshape(padded[0] // 4, 4, padded[1] // 8, 8, padded[2] // 8, 8)
        return p.transpose(0, 2, 4, 1, 3, 5).reshape(-1, 256)

    fb = blocks(flags)
    keep = np.flatnonzero(fb.any(axis=1))
    nb = (padded[0] // 4, padded[1] // 8, padded[2] // 8)
    origin = (np.stack(np.unravel_index(keep, nb), axis=1) * np.array(dims)).astype(np.int32)
    return (origin, fb[keep]) + tuple(blocks(f)[keep] for f in fields)


CONFIGS = {"c1": config1, "c2": config2, "c3": config3, "p128": profile_case, "c5": config5,
           "c5_half": lambda: config5(2), "c2ml": config2_two_level, "tl128": two_level_case}
