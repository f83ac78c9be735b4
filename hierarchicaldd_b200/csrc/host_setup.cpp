// Host-side domain setup (see host_setup.h).
#include "host_setup.h"

#include <algorithm>
#include <cstring>
#include <string>
#include <unordered_set>

namespace hdd {

static const int kFace[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

static inline size_t at3(const int n[3], int i, int j, int k) { return ((size_t)i * n[1] + j) * n[2] + k; }
static inline bool in3(const int n[3], int i, int j, int k) {
    return i >= 0 && j >= 0 && k >= 0 && i < n[0] && j < n[1] && k < n[2];
}

void number_of_subdomains(const int size[3], const int sub[3], int out[3]) {
    // SPGrid_Domain_Divider_Helper.h:31-35 (origin 0).
    for (int a = 0; a < 3; ++a) out[a] = (size[a] - 1) / sub[a] + (((size[a] - 1) % sub[a]) ? 1 : 0);
}

void divide_domain(const int size[3], const int sub[3], uint32_t* f) {
    // SPGrid_Domain_Divider_Helper.h:49-74: Active cells on planes index % sub == 0
    // become Interface; the others carry the 1-based partition id.
    int ns[3];
    number_of_subdomains(size, sub, ns);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                uint32_t& v = f[at3(size, i, j, k)];
                if (!(v & F_ACTIVE)) continue;
                if (i % sub[0] == 0 || j % sub[1] == 0 || k % sub[2] == 0) v = (v - F_ACTIVE) | F_INTERFACE;
                else v |= (uint32_t)((((i / sub[0]) * ns[1] + (j / sub[1])) * ns[2] + (k / sub[2])) + 1);
            }
}

void downsample_topology(const int fd[3], const uint32_t* fine, const int cd[3], uint32_t* coarse) {
    // The reference visits the fine cells page by page in SPGrid address
    // order, and within a page x-slowest; coarse cell c = (f+1)/2.  While c is
    // unset (no Dirichlet, Active or Interface bit), an Active child sets it
    // Active and a Dirichlet child sets it Dirichlet (an Interface child
    // without the Dirichlet bit leaves it unset); once set, a Dirichlet or
    // Interface child makes it Dirichlet.  So an Interface child seen before
    // the first Active one does not count.
    std::fill(coarse, coarse + (size_t)cd[0] * cd[1] * cd[2], 0u);
    const int np[3] = {(fd[0] + 3) / 4, (fd[1] + 7) / 8, (fd[2] + 7) / 8};
    std::vector<std::pair<uint64_t, int>> pages;
    pages.reserve((size_t)np[0] * np[1] * np[2]);
    for (int a = 0; a < np[0]; ++a)
        for (int b = 0; b < np[1]; ++b)
            for (int c = 0; c < np[2]; ++c)
                pages.push_back({spgrid_address(4 * a, 8 * b, 8 * c), (a * np[1] + b) * np[2] + c});
    std::sort(pages.begin(), pages.end());
    for (const auto& pg : pages) {
        const int a = pg.second / (np[1] * np[2]), b = (pg.second / np[2]) % np[1], c = pg.second % np[2];
        for (int x = 4 * a; x < std::min(4 * a + 4, fd[0]); ++x)
            for (int y = 8 * b; y < std::min(8 * b + 8, fd[1]); ++y)
                for (int z = 8 * c; z < std::min(8 * c + 8, fd[2]); ++z) {
                    const uint32_t v = fine[at3(fd, x, y, z)];
                    if (!v) continue;
                    uint32_t& o = coarse[at3(cd, (x + 1) / 2, (y + 1) / 2, (z + 1) / 2)];
                    if (!(o & (F_DIRICHLET | F_ACTIVE | F_INTERFACE))) {
                        if (v & F_ACTIVE) o |= F_ACTIVE;
                        else if (v & (F_DIRICHLET | F_INTERFACE)) o |= (v & F_DIRICHLET);
                        continue;
                    }
                    if (v & (F_DIRICHLET | F_INTERFACE)) o = F_DIRICHLET;
                }
    }
}

void clear_planes(const int size[3], const int sub[3], uint32_t* f) {
    // Domain_Divider with clear_flag (two-level demo,
    // TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Divider_Helper.h:61-72):
    // Active cells on planes index % sub == 0 become Dirichlet, nothing else.
#pragma omp parallel for schedule(static)
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                uint32_t& v = f[at3(size, i, j, k)];
                if ((v & F_ACTIVE) && (i % sub[0] == 0 || j % sub[1] == 0 || k % sub[2] == 0)) v = F_DIRICHLET;
            }
}

void flag_faces(const int n[3], uint32_t* f) {
    // SPGrid_Flag_Helper.h:74-106.
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
            for (int k = 0; k < n[2]; ++k) {
                uint32_t& v = f[at3(n, i, j, k)];
                if (!(v & (F_ACTIVE | F_INTERFACE))) continue;
                for (int q = 0; q < 6; ++q) {
                    int a = i + kFace[q][0], b = j + kFace[q][1], c = k + kFace[q][2];
                    if (in3(n, a, b, c) && (f[at3(n, a, b, c)] & (F_ACTIVE | F_INTERFACE | F_DIRICHLET)))
                        v |= (F_FACE_MX << q);
                }
            }
}

void flag_boundary(const int n[3], uint32_t* f) {
    // SPGrid_Flag_Boundary_Helper.h:40-109: Active cells within Manhattan
    // distance 3 of an exterior (flag 0, or outside the grid), Interface or
    // Dirichlet cell are Boundary.  Computed as a separable distance transform.
    const size_t N = (size_t)n[0] * n[1] * n[2];
    std::vector<uint8_t> dist(N);
#pragma omp parallel for schedule(static)
    for (long long x = 0; x < (long long)N; ++x) {
        uint32_t v = f[x];
        dist[x] = (v == 0u || (v & (F_INTERFACE | F_DIRICHLET))) ? 0 : 4;
    }
    // Cells outside the grid are sources: seed distances from the grid edges.
    auto relax_axis = [&](int axis) {
        int o1 = (axis == 0) ? 1 : 0, o2 = (axis == 2) ? 1 : 2;
#pragma omp parallel for schedule(static)
        for (int a = 0; a < n[o1]; ++a)
            for (int b = 0; b < n[o2]; ++b) {
                int idx[3];
                auto cell = [&](int t) -> uint8_t& {
                    idx[axis] = t; idx[o1] = a; idx[o2] = b;
                    return dist[at3(n, idx[0], idx[1], idx[2])];
                };
                int d = 1;  // distance to the virtual source just before index 0
                for (int t = 0; t < n[axis]; ++t) {
                    uint8_t& c = cell(t);
                    if (c > d) c = (uint8_t)d;
                    d = std::min<int>(c + 1, 4);
                }
                d = 1;
                for (int t = n[axis] - 1; t >= 0; --t) {
                    uint8_t& c = cell(t);
                    if (c > d) c = (uint8_t)d;
                    d = std::min<int>(c + 1, 4);
                }
            }
    };
    // L1 distance = successive 1D passes (min-plus convolution is separable).
    relax_axis(0);
    relax_axis(1);
    relax_axis(2);
#pragma omp parallel for schedule(static)
    for (long long x = 0; x < (long long)N; ++x)
        if ((f[x] & F_ACTIVE) && dist[x] <= 3) f[x] |= F_BOUNDARY;
}

void build_layout(const Options& opt, const uint32_t* flags, DomainLayout& L) {
    L.opt = opt;
    for (int a = 0; a < 3; ++a) {
        if (opt.size[a] < 3) throw Error(HDD_ERR_INVALID_ARGUMENT, "size must be >= 3 on every axis");
        int s = opt.sub[a];
        // The resident V-cycle keeps a subdomain's levels on chip: one CTA for
        // 8^3 and 16^3 boxes, a 4-CTA cluster for 32^3.  A 64^3 box (the
        // reference Test_Bench default, CPU/Test_Bench_3D/main.cpp:247) needs
        // 64^3 x 8 B of level-0 state, more than a 16-CTA cluster's shared
        // memory, and 4^3 boxes have no coarse level worth a launch; both are
        // refused here, before any setup work.
        if (s != 8 && s != 16 && s != 32)
            throw Error(HDD_ERR_UNSUPPORTED, "sub_size must be 8, 16 or 32 (got " + std::to_string(s) + ")");
        if ((s >> (opt.vlevels - 1)) < 2)
            throw Error(HDD_ERR_INVALID_ARGUMENT, "vlevels too deep for sub_size (needs sub_size >> (vlevels-1) >= 2)");
    }
    if (opt.vlevels < 1) throw Error(HDD_ERR_INVALID_ARGUMENT, "vlevels must be >= 1");
    const size_t N = (size_t)opt.size[0] * opt.size[1] * opt.size[2];
    L.flags_in.assign(flags, flags + N);
    L.flags0 = L.flags_in;
    const int* n = opt.size;
    {
        long long active = 0;
#pragma omp parallel for schedule(static) reduction(+ : active)
        for (long long x = 0; x < (long long)N; ++x) active += (L.flags0[x] & F_ACTIVE) ? 1 : 0;
        if (active == 0) throw Error(HDD_ERR_INVALID_ARGUMENT, "domain has no Active cells");
    }
    {
        long long bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
        for (int i = 0; i < n[0]; ++i)
            for (int j = 0; j < n[1]; ++j)
                for (int k = 0; k < n[2]; ++k) {
                    if (L.flags0[at3(n, i, j, k)] & (F_INTERFACE | F_BOUNDARY)) ++bad;
                }
        if (bad)
            throw Error(HDD_ERR_INVALID_ARGUMENT,
                        "input flags carry Interface or Boundary bits (set by the solver): " + std::to_string(bad) +
                            " cells");
    }
    // Reference order: global Domain_Divider, Flaging, then the topology's
    // Flaging (faces again) and Flaging_Boundary on level 0.
    divide_domain(opt.size, opt.sub, L.flags0.data());
    flag_faces(n, L.flags0.data());
    flag_boundary(n, L.flags0.data());

    number_of_subdomains(opt.size, opt.sub, L.ns);
    for (int a = 0; a < 3; ++a) L.nt[a] = (opt.size[a] + opt.sub[a] - 1) / opt.sub[a];
    L.tile_cells = opt.sub[0] * opt.sub[1] * opt.sub[2];
    const size_t ntiles = (size_t)L.nt[0] * L.nt[1] * L.nt[2];
    std::vector<uint8_t> used(ntiles, 0);
    for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
            for (int k = 0; k < n[2]; ++k)
                if (L.flags0[at3(n, i, j, k)] & (F_ACTIVE | F_INTERFACE))
                    used[((size_t)(i / opt.sub[0]) * L.nt[1] + j / opt.sub[1]) * L.nt[2] + k / opt.sub[2]] = 1;
    L.tile_of.assign(ntiles, -1);
    L.tiles.clear();
    for (int a = 0; a < L.nt[0]; ++a)
        for (int b = 0; b < L.nt[1]; ++b)
            for (int c = 0; c < L.nt[2]; ++c) {
                size_t t = ((size_t)a * L.nt[1] + b) * L.nt[2] + c;
                if (used[t]) {
                    L.tile_of[t] = (int)L.tiles.size();
                    L.tiles.push_back({a, b, c});
                }
            }
    L.tile_flags.assign(L.tiled_count(), 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
            for (int k = 0; k < n[2]; ++k) {
                long long s = L.tile_slot(i, j, k);
                if (s >= 0) L.tile_flags[s] = compact16(L.flags0[at3(n, i, j, k)]);
            }

    // Whole-grid levels (CPU/SPGrid_Library/SPGrid_V_Cycle_Topology.h:35-178):
    // level l+1 has n/2+1 cells per axis, downsampled from level l
    // (downsample_topology), then Flaging and Flaging_Boundary.
    const int V = opt.vlevels;
    L.g_dims.assign(V, {0, 0, 0});
    L.g_flags.assign(V, {});
    {
        std::vector<uint32_t> fine = L.flags0, coarse;
        std::array<int, 3> fd = {n[0], n[1], n[2]};
        for (int l = 0; l < V; ++l) {
            if (l > 0) {
                const std::array<int, 3> cd = {fd[0] / 2 + 1, fd[1] / 2 + 1, fd[2] / 2 + 1};
                coarse.assign((size_t)cd[0] * cd[1] * cd[2], 0u);
                downsample_topology(fd.data(), fine.data(), cd.data(), coarse.data());
                flag_faces(cd.data(), coarse.data());
                flag_boundary(cd.data(), coarse.data());
                fine.swap(coarse);
                fd = cd;
            }
            L.g_dims[l] = fd;
            L.g_flags[l].resize(fine.size());
            for (size_t x = 0; x < fine.size(); ++x) L.g_flags[l][x] = compact8(fine[x]);
        }
    }

    // Per-box V-cycle levels.
    L.level_e.assign(3 * V, 0);
    L.level_off.assign(V + 1, 0);
    for (int l = 0; l < V; ++l) {
        size_t cnt = 1;
        for (int a = 0; a < 3; ++a) {
            L.level_e[3 * l + a] = (opt.sub[a] >> l) + 1;
            cnt *= (size_t)L.level_e[3 * l + a];
        }
        L.level_off[l + 1] = L.level_off[l] + ((cnt + 15) / 16) * 16;
    }
    L.box_stride = L.level_off[V];
    L.boxes.clear();
    for (int a = 0; a < L.ns[0]; ++a)
        for (int b = 0; b < L.ns[1]; ++b)
            for (int c = 0; c < L.ns[2]; ++c) {
                bool work = false;
                for (int i = a * opt.sub[0] + 1; i < (a + 1) * opt.sub[0] && i < n[0] && !work; ++i)
                    for (int j = b * opt.sub[1] + 1; j < (b + 1) * opt.sub[1] && j < n[1] && !work; ++j)
                        for (int k = c * opt.sub[2] + 1; k < (c + 1) * opt.sub[2] && k < n[2]; ++k)
                            if (L.flags0[at3(n, i, j, k)] & F_ACTIVE) { work = true; break; }
                if (!work) continue;
                Box bx;
                bx.k = {a, b, c};
                bx.tile = L.tile_of[((size_t)a * L.nt[1] + b) * L.nt[2] + c];
                if (bx.tile < 0) throw Error(HDD_ERR_INTERNAL, "box without a stored tile");
                int nbk[3][3] = {{a + 1, b, c}, {a, b + 1, c}, {a, b, c + 1}};
                for (int q = 0; q < 3; ++q) {
                    int* t = nbk[q];
                    bx.nb_tile[q] = (t[0] < L.nt[0] && t[1] < L.nt[1] && t[2] < L.nt[2])
                                        ? L.tile_of[((size_t)t[0] * L.nt[1] + t[1]) * L.nt[2] + t[2]]
                                        : -1;
                }
                L.boxes.push_back(bx);
            }
    L.box_flags.assign(L.boxes.size() * L.box_stride, 0);
    // Per-box levels: the whole grid's levels inside each box.  The per-box
    // V-cycle keeps a coarse box's face cells at zero, which is the whole
    // grid's V-cycle unless one of them is Active; then the boxes couple and
    // the whole-grid V-cycle runs (set inside the parallel loop).
    int coupled = 0;
#pragma omp parallel for schedule(dynamic)
    for (long long bi = 0; bi < (long long)L.boxes.size(); ++bi) {
        const Box& bx = L.boxes[bi];
        uint8_t* rec = L.box_flags.data() + bi * L.box_stride;
        for (int l = 0; l < V; ++l) {
            const int ce[3] = {L.level_e[3 * l], L.level_e[3 * l + 1], L.level_e[3 * l + 2]};
            const std::array<int, 3>& gd = L.g_dims[l];
            const std::vector<uint8_t>& gf = L.g_flags[l];
            const int o[3] = {bx.k[0] * (opt.sub[0] >> l), bx.k[1] * (opt.sub[1] >> l), bx.k[2] * (opt.sub[2] >> l)};
            uint8_t* dst = rec + L.level_off[l];
            for (int x = 0; x < ce[0]; ++x)
                for (int y = 0; y < ce[1]; ++y)
                    for (int z = 0; z < ce[2]; ++z) {
                        const int gx = o[0] + x, gy = o[1] + y, gz = o[2] + z;
                        const bool inside = gx < gd[0] && gy < gd[1] && gz < gd[2];
                        const uint8_t g = inside ? gf[at3(gd.data(), gx, gy, gz)] : 0;
                        dst[at3(ce, x, y, z)] = g;
                        const bool halo = x == 0 || y == 0 || z == 0 || x == ce[0] - 1 || y == ce[1] - 1 || z == ce[2] - 1;
                        if (l > 0 && halo && (g & C_ACTIVE)) {
#pragma omp atomic write
                            coupled = 1;
                        }
                    }
        }
    }
    L.global_vcycle = coupled != 0;
    if (!L.global_vcycle) {
        L.g_dims.clear();
        L.g_flags.clear();
    }
}

void dense_to_tiles(const DomainLayout& L, const float* dense, float* tiled) {
    const int* n = L.opt.size;
    std::memset(tiled, 0, L.tiled_count() * sizeof(float));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
            for (int k = 0; k < n[2]; ++k) {
                long long s = L.tile_slot(i, j, k);
                if (s >= 0) tiled[s] = dense[at3(n, i, j, k)];
            }
}

void tiles_to_dense(const DomainLayout& L, const float* tiled, float* dense) {
    const int* n = L.opt.size;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
            for (int k = 0; k < n[2]; ++k) {
                long long s = L.tile_slot(i, j, k);
                dense[at3(n, i, j, k)] = s >= 0 ? tiled[s] : 0.0f;
            }
}

namespace {

void check_pages(long long n, const int32_t* origin) {
    if (n < 0 || (n > 0 && !origin)) throw Error(HDD_ERR_INVALID_ARGUMENT, "bad page count or origin array");
    std::unordered_set<uint64_t> seen;
    seen.reserve((size_t)n);
    for (long long p = 0; p < n; ++p) {
        uint64_t key = 0;
        for (int a = 0; a < 3; ++a) {
            const int32_t o = origin[3 * p + a];
            if (o < 0 || o % kPageDims[a] != 0)
                throw Error(HDD_ERR_INVALID_ARGUMENT, "page origin " + std::to_string(p) +
                                                          " is negative or not a multiple of (4, 8, 8)");
            if (o / kPageDims[a] >= (1 << 21))
                throw Error(HDD_ERR_INVALID_ARGUMENT, "page origin " + std::to_string(p) + " is too large");
            key = (key << 21) | (uint64_t)(o / kPageDims[a]);
        }
        if (!seen.insert(key).second)
            throw Error(HDD_ERR_INVALID_ARGUMENT, "page " + std::to_string(p) + " is listed twice");
    }
}

// Calls fn(page element, dense index) for every cell of the pages inside the grid.
template <class Fn>
void for_page_cells(const int size[3], long long n, const int32_t* origin, Fn fn) {
    for (long long p = 0; p < n; ++p) {
        const int32_t* o = origin + 3 * p;
        for (int x = 0; x < kPageDims[0]; ++x)
            for (int y = 0; y < kPageDims[1]; ++y)
                for (int z = 0; z < kPageDims[2]; ++z) {
                    const long long i = (long long)o[0] + x, j = (long long)o[1] + y, k = (long long)o[2] + z;
                    if (i >= size[0] || j >= size[1] || k >= size[2]) continue;
                    fn((size_t)p * kPageCells + (size_t)((x * 8 + y) * 8 + z),
                       ((size_t)i * size[1] + (size_t)j) * size[2] + (size_t)k);
                }
    }
}

}  // namespace

void pages_to_dense(const int size[3], long long n, const int32_t* origin, const uint32_t* values, uint32_t* dense) {
    check_pages(n, origin);
    for_page_cells(size, n, origin, [&](size_t e, size_t d) { dense[d] = values[e]; });
}

void pages_to_dense(const int size[3], long long n, const int32_t* origin, const float* values, float* dense) {
    check_pages(n, origin);
    for_page_cells(size, n, origin, [&](size_t e, size_t d) { dense[d] = values[e]; });
}

void dense_to_pages(const int size[3], long long n, const int32_t* origin, const float* dense, float* values) {
    check_pages(n, origin);
    std::fill(values, values + (size_t)n * kPageCells, 0.0f);
    for_page_cells(size, n, origin, [&](size_t e, size_t d) { values[e] = dense[d]; });
}

}  // namespace hdd
