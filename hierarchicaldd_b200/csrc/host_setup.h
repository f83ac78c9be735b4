// Host-side domain setup: reference flag pipeline, subdomain tiles in HBM and
// per-subdomain coarse levels for the resident V-cycle kernel.
//
// Layout.  The grid is cut into tiles of sub_size cells per axis; tile t holds
// cells [t*sub, (t+1)*sub) per axis, z fastest inside a tile.  Tile k coincides
// with the reference's subdomain box k ([k*sub, (k+1)*sub], inclusive,
// SPGrid_Domain_Divider_Helper.h:36-40) minus its upper interface planes,
// which are the lower planes of tiles k+1.  Only tiles holding Active or
// Interface cells are stored; absent tiles read as zero.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

#include "hdd_common.h"

namespace hdd {

// SPGrid_Mask<4,2,3> addresses (4 x 8 x 8-cell pages of a 16-byte struct,
// page coordinates bit-interleaved above 4 KB, cell (x, y, z) of a page at
// (x * 8 + y) * 8 + z, SPGrid_Mask.h:25-31): the order in which the
// reference's block iterators walk cells.
inline uint64_t spgrid_spread_bits(uint64_t v, uint64_t mask) {
    uint64_t r = 0;
    for (uint64_t bit = 1; mask; bit <<= 1) {
        const uint64_t low = mask & (~mask + 1);
        if (v & bit) r |= low;
        mask &= mask - 1;
    }
    return r;
}
inline uint64_t spgrid_address(int x, int y, int z) {
    return spgrid_spread_bits((uint64_t)x, 0x9249249249249000ull | 0x300ull) |
           spgrid_spread_bits((uint64_t)y, 0x4924924924924000ull | 0x0e0ull) |
           spgrid_spread_bits((uint64_t)z, 0x2492492492492000ull | 0x01cull);
}

struct Options {
    int size[3];
    int sub[3];
    int vlevels, nvcycles, interior, boundary, sigma_levels, sigma_smoothing, sigma_mg;
};

// One subdomain box with work for the V-cycle.
struct Box {
    std::array<int, 3> k;    // box coordinates (== its tile coordinates)
    int tile;                // stored tile index of the box's own tile
    int nb_tile[3];          // stored tile index of the +x/+y/+z neighbour tiles (-1 if absent)
};

struct DomainLayout {
    Options opt;
    int nt[3] = {0, 0, 0};   // tiles per axis
    int ns[3] = {0, 0, 0};   // reference subdomain count per axis
    int tile_cells = 0;
    std::vector<int> tile_of;                 // nt0*nt1*nt2 -> stored tile or -1
    std::vector<std::array<int, 3>> tiles;    // stored tile coordinates
    std::vector<uint32_t> flags_in;           // caller flags (dense)
    std::vector<uint32_t> flags0;             // level-0 flags after divider/faces/boundary (dense)
    std::vector<uint16_t> tile_flags;         // compact16 per stored tile cell
    std::vector<Box> boxes;
    // Per-box V-cycle flags: level l box has e_l = (sub >> l) + 1 cells per
    // axis (including the two halo planes); all levels of a box are stored
    // back to back, boxes at a fixed stride.
    std::vector<int> level_e;                 // [vlevels][3]
    std::vector<size_t> level_off;            // offset of level l inside a box record
    size_t box_stride = 0;
    std::vector<uint8_t> box_flags;           // boxes.size() * box_stride
    // Whole-grid levels (V_Cycle_Topology on the whole grid): dims and
    // compact8 flags.  global_vcycle is set when a box's levels differ from
    // the whole grid's inside the box, or a box-face cell of a coarse level
    // is Active there: the boxes' V-cycles would then not be the reference's
    // (an exterior region touching Active cells, as the reference
    // generator's Neumann bubble, couples boxes at coarse levels), and the
    // whole-grid V-cycle runs instead.
    bool global_vcycle = false;
    std::vector<std::array<int, 3>> g_dims;
    std::vector<std::vector<uint8_t>> g_flags;

    size_t cell_count() const { return (size_t)opt.size[0] * opt.size[1] * opt.size[2]; }
    size_t dense_index(int i, int j, int k) const {
        return ((size_t)i * opt.size[1] + j) * opt.size[2] + k;
    }
    // Tile slot of a dense cell, or -1 when its tile is not stored.
    long long tile_slot(int i, int j, int k) const {
        int t = tile_of[((size_t)(i / opt.sub[0]) * nt[1] + (j / opt.sub[1])) * nt[2] + (k / opt.sub[2])];
        if (t < 0) return -1;
        int l = ((i % opt.sub[0]) * opt.sub[1] + (j % opt.sub[1])) * opt.sub[2] + (k % opt.sub[2]);
        return (long long)t * tile_cells + l;
    }
    size_t tiled_count() const { return tiles.size() * (size_t)tile_cells; }
};

// Validates options and flags, runs the level-0 flag pipeline and builds the
// tile layout and per-box coarse levels.  Throws hdd::Error.
void build_layout(const Options& opt, const uint32_t* flags, DomainLayout& out);

// Dense <-> tiled copies of a float field.
void dense_to_tiles(const DomainLayout& L, const float* dense, float* tiled);
void tiles_to_dense(const DomainLayout& L, const float* tiled, float* dense);

// SPGrid pages: 4 x 8 x 8 cells, the 4 KB page of a 16-byte cell struct with
// 4-byte channels (SPGrid_Mask<4,2,3>, SPGrid_Mask.h:25-31); cell (x, y, z) of a
// page is element (x * 8 + y) * 8 + z, and a page's origin (its cell (0,0,0))
// is a multiple of (4, 8, 8).
constexpr int kPageDims[3] = {4, 8, 8};
constexpr int kPageCells = 256;

// Scatters n pages (origin[3*p + a], values[256*p + e]) into a dense grid of
// size[0..2] cells, z fastest; cells outside the grid are skipped, other dense
// cells are left as they are.  Throws HDD_ERR_INVALID_ARGUMENT for a negative or
// misaligned origin or a page listed twice.
void pages_to_dense(const int size[3], long long n, const int32_t* origin, const uint32_t* values, uint32_t* dense);
void pages_to_dense(const int size[3], long long n, const int32_t* origin, const float* values, float* dense);
// Gathers the same pages from a dense grid (0 outside the grid).
void dense_to_pages(const int size[3], long long n, const int32_t* origin, const float* dense, float* values);

// V_Cycle_Topology::Topology_Downsample (CPU/SPGrid_Library/SPGrid_V_Cycle_Topology.h:35-67):
// coarse flags of size cd from fine flags of size fd (cells visited in SPGrid
// address order; the result depends on it).
void downsample_topology(const int fd[3], const uint32_t* fine, const int cd[3], uint32_t* coarse);

// Level-0 flag pipeline pieces (same semantics as the reference passes).
void divide_domain(const int size[3], const int sub[3], uint32_t* f);
// Two-level DD: Active cells on the first-level planes (index % sub == 0)
// become Dirichlet, the flags of a first-level subdomain's own DD.
void clear_planes(const int size[3], const int sub[3], uint32_t* f);
void flag_faces(const int n[3], uint32_t* f);
void flag_boundary(const int n[3], uint32_t* f);
void number_of_subdomains(const int size[3], const int sub[3], int out[3]);

}  // namespace hdd
