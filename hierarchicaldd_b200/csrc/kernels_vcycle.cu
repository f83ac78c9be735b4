// Subdomain-resident multigrid V-cycle for sm_100a.
//
// One CTA owns one subdomain box for the whole V-cycle: the level-0 box
// (sub+1)^3 cells including its two halo planes per axis, and every coarse
// level, live in shared memory.  HBM is touched once to load u, b and the
// flags and once to store u, instead of once per smoothing sweep as in the
// reference (CPU/SPGrid_Library/SPGrid_V_Cycle_Helper.h:156-195, GPU
// CUDA_Kernels/SPGrid_V_Cycle_Helper_CUDA.h:272-301).
//
// Arithmetic follows the reference's float operation order with explicit
// round-to-nearest intrinsics, so no multiply-add is contracted:
//   residual   r = b - sum_faces (u_n - u_c)      (SPGrid_Residual_Legacy.h:52-61)
//   correction u += (omega/face_count) * r        (SPGrid_Correction_Legacy.h:47-80)
//   restriction, prolongation weights and order  (SPGrid_Restriction_Legacy.h:47-186,
//                                                 SPGrid_Prolongation_Legacy.h:46-128)
// Smoothing is Jacobi: every residual of a sweep is computed from the old u
// (held in registers) before any update.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <utility>

#include "hdd_common.h"
#include "kernels.h"

namespace hdd {

namespace cg = cooperative_groups;

namespace {

struct LevelSmem {
    float* u;
    float* b;
    float* r;
    uint8_t* f;
    int e;  // cells per axis including halos
};

__device__ __forceinline__ int box_index(int e, int x, int y, int z) { return (x * e + y) * e + z; }

// Residual of one cell (Active), reference face order -x,+x,-y,+y,-z,+z.
__device__ __forceinline__ float cell_residual(const LevelSmem& L, int i, uint32_t fl) {
    const int sx = L.e * L.e, sy = L.e;
    const float c = L.u[i];
    float res = 0.0f;
    float n;
    n = L.u[i - sx]; if (fl & 0x01u) res = __fsub_rn(res, __fsub_rn(n, c));
    n = L.u[i + sx]; if (fl & 0x02u) res = __fsub_rn(res, __fsub_rn(n, c));
    n = L.u[i - sy]; if (fl & 0x04u) res = __fsub_rn(res, __fsub_rn(n, c));
    n = L.u[i + sy]; if (fl & 0x08u) res = __fsub_rn(res, __fsub_rn(n, c));
    n = L.u[i - 1];  if (fl & 0x10u) res = __fsub_rn(res, __fsub_rn(n, c));
    n = L.u[i + 1];  if (fl & 0x20u) res = __fsub_rn(res, __fsub_rn(n, c));
    return __fsub_rn(L.b[i], res);
}

// Value of a tiled level-0 vector at box cell (x, y, z), 0 <= x, y, z < SUB
// (the box's own tile).
template <int SUB>
__device__ __forceinline__ float own_tile_value(const float* v, int tile, int x, int y, int z) {
    return v[(size_t)tile * (SUB * SUB * SUB) + (x * SUB + y) * SUB + z];
}

// Interior cell q (0 .. (e-2)^3-1) -> box index.
__device__ __forceinline__ int interior_cell(int e, int q) {
    const int m = e - 2;
    const int z = q % m, t = q / m;
    const int y = t % m, x = t / m;
    return box_index(e, x + 1, y + 1, z + 1);
}

// Thread groups that run a level: the whole CTA, or one warp for the small
// coarse levels, where a CTA-wide barrier per half-sweep costs far more than
// the few hundred cells it orders.
struct CtaGroup {
    __device__ int rank() const { return threadIdx.x; }
    __device__ int size() const { return blockDim.x; }
    __device__ void sync() const { __syncthreads(); }
};
struct WarpGroup {
    __device__ int rank() const { return threadIdx.x & 31; }
    __device__ int size() const { return 32; }
    __device__ void sync() const { __syncwarp(); }
};

// Coarse levels with at most this many cells per axis (halos included) run
// in one warp: (5-2)^3 = 27 cells, one per lane.
constexpr int kWarpLevelE = 5;
constexpr int kWarpCH = 1;

// mode: 1 = boundary cells, 2 = interior (non-boundary) cells, 3 = all Active.
template <int CH, class G>
__device__ __noinline__ void jacobi_sweep(const G& g, const LevelSmem& L, int mode, const float* inv_diag) {
    const int m = L.e - 2;
    const int ncell = m * m * m;
    float rr[CH];
    int idx[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        const int q = g.rank() + c * g.size();
        idx[c] = -1;
        if (q < ncell) {
            const int i = interior_cell(L.e, q);
            const uint32_t fl = L.f[i];
            const bool active = fl & C_ACTIVE;
            const bool bnd = fl & C_BOUNDARY8;
            const bool take = active && ((mode == 3) || (mode == 1 && bnd) || (mode == 2 && !bnd));
            if (take) {
                idx[c] = i;
                rr[c] = cell_residual(L, i, fl);
            }
        }
    }
    g.sync();
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        if (idx[c] >= 0) {
            const int i = idx[c];
            const float w = inv_diag[__popc((uint32_t)L.f[i] & C_FACES)];
            L.u[i] = __fadd_rn(L.u[i], __fmul_rn(w, rr[c]));
        }
    }
    g.sync();
}

// Jacobi sweep of a whole box level: each of the NX*NX x-lines (NX cells) is
// cut into PARTS contiguous pieces, one per thread of g, so there is no index
// division per cell and a piece's residuals stay in registers.  The per-cell
// arithmetic is cell_residual's, so results equal jacobi_sweep's.
template <int NX, int PARTS, class G>
__device__ __noinline__ void box_line_sweep(const G& g, const LevelSmem& L, int mode, const float* inv_diag) {
    constexpr int e = NX + 2, PS = e * e;
    constexpr int CPT = (NX + PARTS - 1) / PARTS;   // cells per thread
    const int t = g.rank();
    float rr[CPT];
    uint32_t tk = 0;
    int base = 0, k0 = 0;
    if (t < NX * NX * PARTS) {
        const int line = t % (NX * NX), part = t / (NX * NX);
        const int y = line / NX + 1, z = line % NX + 1;
        k0 = part * CPT;
        base = PS + y * e + z;
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            rr[c] = 0.0f;
            const int k = k0 + c;
            if (k >= NX) continue;
            const int i = base + k * PS;
            const uint32_t fl = L.f[i];
            const bool active = fl & C_ACTIVE;
            const bool bnd = fl & C_BOUNDARY8;
            const bool take = active && ((mode == 3) || (mode == 1 && bnd) || (mode == 2 && !bnd));
            if (take) {
                tk |= 1u << c;
                rr[c] = cell_residual(L, i, fl);
            }
        }
    }
    g.sync();
    if (tk) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            if (tk & (1u << c)) {
                const int i = base + (k0 + c) * PS;
                const float w = inv_diag[__popc((uint32_t)L.f[i] & C_FACES)];
                L.u[i] = __fadd_rn(L.u[i], __fmul_rn(w, rr[c]));
            }
        }
    }
    g.sync();
}

// One Jacobi sweep of a box level; levels up to 17^3 cells cut their x-lines
// over as many threads as the group has, larger ones use the chunked sweep.
template <int CH, class G>
__device__ void sweep_box(const G& g, const LevelSmem& L, int mode, const float* inv_diag) {
    const int n = g.size();
    switch (L.e) {
        case 3: box_line_sweep<1, 1>(g, L, mode, inv_diag); return;
        case 5:
            if (n >= 27) box_line_sweep<3, 3>(g, L, mode, inv_diag);
            else if (n >= 9) box_line_sweep<3, 1>(g, L, mode, inv_diag);
            else break;
            return;
        case 9:
            if (n >= 343) box_line_sweep<7, 7>(g, L, mode, inv_diag);
            else if (n >= 98) box_line_sweep<7, 2>(g, L, mode, inv_diag);
            else if (n >= 49) box_line_sweep<7, 1>(g, L, mode, inv_diag);
            else break;
            return;
        case 17:
            if (n >= 450) box_line_sweep<15, 2>(g, L, mode, inv_diag);
            else if (n >= 225) box_line_sweep<15, 1>(g, L, mode, inv_diag);
            else break;
            return;
        default: break;
    }
    jacobi_sweep<CH>(g, L, mode, inv_diag);
}

// r = b - A u at Active cells (other cells of r keep their zero).
template <class G>
__device__ void residual_store(const G& g, const LevelSmem& L) {
    const int m = L.e - 2;
    const int ncell = m * m * m;
    for (int q = g.rank(); q < ncell; q += g.size()) {
        const int i = interior_cell(L.e, q);
        const uint32_t fl = L.f[i];
        if (fl & C_ACTIVE) L.r[i] = cell_residual(L, i, fl);
    }
    g.sync();
}

template <class G>
__device__ void zero_u(const G& g, const LevelSmem& L) {
    const int n = L.e * L.e * L.e;
    for (int i = g.rank(); i < n; i += g.size()) L.u[i] = 0.0f;
    g.sync();
}

template <class G>
__device__ void restrict_level(const G& g, const LevelSmem& F, const LevelSmem& Cc, const float* sc64) {
    const int m = Cc.e - 2;
    const int ncell = m * m * m;
    const int sx = F.e * F.e, sy = F.e;
    for (int q = g.rank(); q < ncell; q += g.size()) {
        const int z = q % m, t = q / m;
        const int y = t % m, x = t / m;
        const int ci = box_index(Cc.e, x + 1, y + 1, z + 1);
        if (!(Cc.f[ci] & C_ACTIVE)) continue;
        // Fine cells 2C-2 .. 2C+1 per axis (box coordinates, C = x+1).
        const int f0 = box_index(F.e, 2 * x, 2 * y, 2 * z);
        float acc = 0.0f;
#pragma unroll
        for (int i2 = 0; i2 < 4; ++i2)
#pragma unroll
            for (int j2 = 0; j2 < 4; ++j2)
#pragma unroll
                for (int k2 = 0; k2 < 4; ++k2)
                    acc = __fadd_rn(acc, __fmul_rn(sc64[(i2 * 4 + j2) * 4 + k2], F.r[f0 + i2 * sx + j2 * sy + k2]));
        Cc.b[ci] = acc;
    }
    g.sync();
}

template <class G>
__device__ void prolongate_level(const G& g, const LevelSmem& F, const LevelSmem& Cc, const float* sc8) {
    const int m = F.e - 2;
    const int ncell = m * m * m;
    const int csx = Cc.e * Cc.e, csy = Cc.e;
    for (int q = g.rank(); q < ncell; q += g.size()) {
        const int z = q % m + 1, t = q / m;
        const int y = t % m + 1, x = t / m + 1;
        const int fi = box_index(F.e, x, y, z);
        if (!(F.f[fi] & C_ACTIVE)) continue;
        // Box origins are even, so box-local parents follow the global rule:
        // c = (f+1)/2, parity p = 1 - (f - (2c-1)).
        const int cx = (x + 1) >> 1, cy = (y + 1) >> 1, cz = (z + 1) >> 1;
        const int px = 1 - (x - (2 * cx - 1)), py = 1 - (y - (2 * cy - 1)), pz = 1 - (z - (2 * cz - 1));
        const int cbase = box_index(Cc.e, cx, cy, cz);
        float acc = F.u[fi];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int bq = 0; bq < 2; ++bq)
#pragma unroll
                for (int cq = 0; cq < 2; ++cq) {
                    const float w = sc8[((a ^ px) * 2 + (bq ^ py)) * 2 + (cq ^ pz)];
                    const float v = Cc.u[cbase + (a - px) * csx + (bq - py) * csy + (cq - pz)];
                    acc = __fadd_rn(acc, __fmul_rn(w, v));
                }
        F.u[fi] = acc;
    }
    g.sync();
}

// Pre/post smoothing of one level: boundary, interior, boundary sweeps.
template <int CH, class G>
__device__ void smooth_level(const G& g, const LevelSmem& L, const VcycleArgs& a, const float* inv_diag) {
    for (int i = 0; i < a.boundary_itr; ++i) sweep_box<CH>(g, L, 1, inv_diag);
    for (int i = 0; i < a.interior_itr; ++i) sweep_box<CH>(g, L, 2, inv_diag);
    for (int i = 0; i < a.boundary_itr; ++i) sweep_box<CH>(g, L, 1, inv_diag);
}

// n all-Active Jacobi sweeps of a 5^3 box (3^3 interior cells) by one warp:
// lane q < 27 holds cell q in a register and takes interior neighbours by
// shuffle; halo neighbours never change during the sweeps (only Active
// interior cells are updated), so they are read once.  Same arithmetic and
// face order as cell_residual, so the result equals n jacobi_sweep calls.
__device__ __noinline__ void bottom_sweeps_3(const LevelSmem& L, int n, const float* inv_diag) {
    const int lane = threadIdx.x & 31;
    const bool own = lane < 27;
    const int q = own ? lane : 0;
    const int x = q / 9 + 1, y = (q / 3) % 3 + 1, z = q % 3 + 1;
    const int i = (x * 5 + y) * 5 + z;
    const uint32_t fl = own ? (uint32_t)L.f[i] : 0u;
    const bool act = own && (fl & C_ACTIVE);
    const float bb = own ? L.b[i] : 0.0f;
    const float w = inv_diag[__popc(fl & C_FACES)];
    float u = own ? L.u[i] : 0.0f;
    // Per face: source lane for an interior neighbour, or the fixed halo value.
    const int d[6] = {-25, 25, -5, 5, -1, 1};
    const int dl[6] = {-9, 9, -3, 3, -1, 1};
    const int cpos[6] = {x, x, y, y, z, z};
    int src[6];
    float halo[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int np = cpos[f] + ((f & 1) ? 1 : -1);
        const bool inside = np >= 1 && np <= 3;
        src[f] = inside ? q + dl[f] : q;
        halo[f] = (!inside && own) ? L.u[i + d[f]] : 0.0f;
        if (inside) halo[f] = 0.0f;
        src[f] = inside ? src[f] : -1;
    }
    for (int it = 0; it < n; ++it) {
        float nb[6];
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            const float v = __shfl_sync(0xffffffffu, u, src[f] < 0 ? q : src[f]);
            nb[f] = src[f] < 0 ? halo[f] : v;
        }
        float res = 0.0f;
#pragma unroll
        for (int f = 0; f < 6; ++f)
            if (fl & (1u << f)) res = __fsub_rn(res, __fsub_rn(nb[f], u));
        const float r = __fsub_rn(bb, res);
        if (act) u = __fadd_rn(u, __fmul_rn(w, r));
    }
    if (own) L.u[i] = u;
    __syncwarp();
}

// Levels T..Lm-1 of one V-cycle with group g: down-leg from T, bottom
// smoothing at Lm-1, up-leg back to T (the caller has restricted into T).
template <int CH, class G>
__device__ void vcycle_tail(const G& g, LevelSmem* lv, int T, int Lm, const VcycleArgs& a, const float* inv_diag,
                            const float* sc64, const float* sc8) {
    for (int l = T; l < Lm - 1; ++l) {
        smooth_level<CH>(g, lv[l], a, inv_diag);
        residual_store(g, lv[l]);
        zero_u(g, lv[l + 1]);
        restrict_level(g, lv[l], lv[l + 1], sc64);
    }
    if (lv[Lm - 1].e == 5 && g.size() == 32) bottom_sweeps_3(lv[Lm - 1], a.bottom_itr, inv_diag);
    else
        for (int i = 0; i < a.bottom_itr; ++i) sweep_box<CH>(g, lv[Lm - 1], 3, inv_diag);
    for (int l = Lm - 2; l >= T; --l) {
        prolongate_level(g, lv[l], lv[l + 1], sc8);
        smooth_level<CH>(g, lv[l], a, inv_diag);
    }
}

// First level (>= 1) small enough for one warp, or Lm when there is none.
__device__ __forceinline__ int first_warp_level(int sub, int Lm) {
    for (int l = 1; l < Lm; ++l)
        if ((sub >> l) + 1 <= kWarpLevelE) return l;
    return Lm;
}

template <int SUB, int NT>
__global__ void __launch_bounds__(NT, 1) vcycle_kernel(VcycleArgs a) {
    constexpr int E0 = SUB + 1;
    constexpr int CH = ((SUB - 1) * (SUB - 1) * (SUB - 1) + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ float s_inv[8];
    __shared__ float s_sc64[64];
    __shared__ float s_sc8[8];

    const int box = blockIdx.x;
    if (box >= a.nbox) return;
    if (a.active && !a.active[blockIdx.y]) return;
    // System blockIdx.y of a batch: its u and b.
    float* const au = a.u + (size_t)blockIdx.y * a.slot_stride;
    const float* const ab = a.b + (size_t)blockIdx.y * a.slot_stride;
    if (threadIdx.x < 8) s_inv[threadIdx.x] = a.inv_diag[threadIdx.x];
    if (threadIdx.x < 64) s_sc64[threadIdx.x] = a.restrict_w[threadIdx.x];
    if (threadIdx.x < 8) s_sc8[threadIdx.x] = a.prolong_w[threadIdx.x];

    // Carve shared memory: per level u, b, r (float) then f (uint8).
    LevelSmem lv[kMaxLevels];
    {
        unsigned char* p = smem;
        for (int l = 0; l < a.levels; ++l) {
            const int e = (SUB >> l) + 1;
            const int n = e * e * e;
            const int n4 = (n + 3) & ~3;
            lv[l].e = e;
            lv[l].u = reinterpret_cast<float*>(p); p += n4 * 4;
            lv[l].b = reinterpret_cast<float*>(p); p += n4 * 4;
            lv[l].r = reinterpret_cast<float*>(p); p += n4 * 4;
            lv[l].f = p; p += n4;
        }
    }
    const uint8_t* rec = a.box_flags + (size_t)box * a.box_stride;
    const int tile = a.box_tile[box];
    const float* gu = au + (size_t)tile * (SUB * SUB * SUB);
    const float* gb = ab + (size_t)tile * (SUB * SUB * SUB);

    // Zero every level (halo cells, r and coarse values start at zero).
    for (int l = 0; l < a.levels; ++l) {
        const int e = lv[l].e, n = e * e * e;
        for (int i = threadIdx.x; i < n; i += NT) {
            lv[l].u[i] = 0.0f; lv[l].b[i] = 0.0f; lv[l].r[i] = 0.0f;
            lv[l].f[i] = rec[a.level_off[l] + i];
        }
    }
    __syncthreads();
    // Level-0 loads from the box's own tile: cells 0..SUB-1 per axis.
    for (int q = threadIdx.x; q < SUB * SUB * SUB; q += NT) {
        const int z = q % SUB, t = q / SUB;
        const int y = t % SUB, x = t / SUB;
        const int i = box_index(E0, x, y, z);
        const bool halo = (x == 0) || (y == 0) || (z == 0);
        if (halo) {
            if (a.halo_from_u) lv[0].u[i] = gu[q];
        } else {
            if (!a.zero_init) lv[0].u[i] = gu[q];
            lv[0].b[i] = gb[q];
        }
    }
    // Upper halo planes from the +x/+y/+z neighbour tiles (their local plane 0).
    if (a.halo_from_u) {
        for (int axis = 0; axis < 3; ++axis) {
            const int nt = a.box_nb[3 * box + axis];
            if (nt < 0) continue;
            const float* gn = au + (size_t)nt * (SUB * SUB * SUB);
            for (int q = threadIdx.x; q < (SUB - 1) * (SUB - 1); q += NT) {
                const int p1 = q % (SUB - 1) + 1, p0 = q / (SUB - 1) + 1;
                int lx, ly, lz, bx, by, bz;
                if (axis == 0) { lx = 0; ly = p0; lz = p1; bx = SUB; by = p0; bz = p1; }
                else if (axis == 1) { lx = p0; ly = 0; lz = p1; bx = p0; by = SUB; bz = p1; }
                else { lx = p0; ly = p1; lz = 0; bx = p0; by = p1; bz = SUB; }
                lv[0].u[box_index(E0, bx, by, bz)] = gn[(lx * SUB + ly) * SUB + lz];
            }
        }
    }
    // Residual at the lower-face cells, when given (else it stays zero).
    if (a.r_halo) {
        const float* rh = a.r_halo + (size_t)blockIdx.y * a.slot_stride;
        for (int q = threadIdx.x; q < SUB * SUB * SUB; q += NT) {
            const int z = q % SUB, t = q / SUB, y = t % SUB, x = t / SUB;
            if (x == 0 || y == 0 || z == 0) lv[0].r[box_index(E0, x, y, z)] = own_tile_value<SUB>(rh, tile, x, y, z);
        }
    }
    __syncthreads();

    const int Lm = a.levels;
    const int T = first_warp_level(SUB, Lm);  // levels T..Lm-1 run in warp 0
    const CtaGroup cta;
    for (int cycle = 0; cycle < a.n_vcycles; ++cycle) {
        const int Tc = T < Lm ? T : Lm - 1;
        for (int l = 0; l < Tc; ++l) {
            smooth_level<CH>(cta, lv[l], a, s_inv);
            residual_store(cta, lv[l]);
            zero_u(cta, lv[l + 1]);
            restrict_level(cta, lv[l], lv[l + 1], s_sc64);
        }
        if (T < Lm) {
            if (threadIdx.x < 32) vcycle_tail<kWarpCH>(WarpGroup(), lv, T, Lm, a, s_inv, s_sc64, s_sc8);
            __syncthreads();
        } else {
            for (int i = 0; i < a.bottom_itr; ++i) sweep_box<CH>(cta, lv[Lm - 1], 3, s_inv);
        }
        for (int l = Tc - 1; l >= 0; --l) {
            prolongate_level(cta, lv[l], lv[l + 1], s_sc8);
            smooth_level<CH>(cta, lv[l], a, s_inv);
        }
    }

    // Store the interior cells (1..SUB-1 per axis) of level 0.
    float* gw = au + (size_t)tile * (SUB * SUB * SUB);
    for (int q = threadIdx.x; q < SUB * SUB * SUB; q += NT) {
        const int z = q % SUB, t = q / SUB;
        const int y = t % SUB, x = t / SUB;
        if (x == 0 || y == 0 || z == 0) continue;
        gw[q] = lv[0].u[box_index(E0, x, y, z)];
    }
}

template <int SUB>
size_t vcycle_smem_bytes(int levels) {
    size_t total = 0;
    for (int l = 0; l < levels; ++l) {
        const int e = (SUB >> l) + 1;
        const size_t n4 = ((size_t)e * e * e + 3) & ~size_t(3);
        total += n4 * 13;
    }
    return total;
}

// ---------------------------------------------------------------------------
// Cluster variant: one subdomain per thread-block cluster of C CTAs.
//
// Level 0 is cut into C slabs along x; CTA `rank` owns interior planes
// x0..x1.  Each thread owns x-lines of the slab and keeps their u in
// registers (shared memory holds a copy for the y/z neighbours of other
// threads).  After every Jacobi update a CTA stores its first/last owned
// planes straight into its neighbours' shared memory (distributed shared
// memory), double-buffered by sweep parity; one cluster barrier per sweep
// orders the exchange and each thread reads its lines' new x-halos into
// registers.  The coarse levels are small and live in rank 0; the
// restriction into rank 0 and the prolongation out of it are spread over all
// ranks through DSMEM.  Every CTA executes the same sequence of cluster
// barriers.
// ---------------------------------------------------------------------------
template <int SUB, int C>
struct SlabGeom {
    static constexpr int E = SUB + 1;
    static constexpr int PS = E * E;
    static constexpr int P = (SUB - 1 + C - 1) / C;
    static constexpr int M2 = (SUB - 1) * (SUB - 1);
};

// The (y, z) x-line that thread t owns as its l-th line of a slab, or false.
// Lines whose cells all lie within the Boundary band (3 cells) of the box's
// y/z faces take boundary-sweep work on every cell; with 2 lines per thread
// each thread gets at most one such line, so boundary sweeps are not paced by
// threads holding two.  Any assignment gives the same results (Jacobi sweeps).
template <int SUB, int NT, int LPT>
__device__ __forceinline__ bool owned_line(int t, int l, int& y, int& z) {
    constexpr int M1 = SUB - 1, D = 3, W = M1 - 2 * D;
    constexpr int H = 2 * D * M1 + W * 2 * D;   // lines inside the band
    constexpr int L = W * W;                    // the others
    if constexpr (LPT == 2 && H <= NT && NT <= H + L && L <= 2 * NT - H) {
        auto band = [](int i) { return i < D ? i + 1 : SUB - 2 * D + i; };  // 1..D, SUB-D..SUB-1
        auto heavy = [&](int h) {
            if (h < 2 * D * M1) { y = band(h / M1); z = h % M1 + 1; }
            else { const int r = h - 2 * D * M1; y = D + 1 + r / (2 * D); z = band(r % (2 * D)); }
        };
        auto light = [&](int k) { y = D + 1 + k / W; z = D + 1 + k % W; };
        if (t < H) {
            if (l == 0) heavy(t);
            else light(t);
            return true;
        }
        const int j = t - H;
        if (l == 0) { light(H + j); return true; }
        if (NT + j < L) { light(NT + j); return true; }
        return false;
    } else {
        const int q = t + l * NT;
        if (q >= M1 * M1) return false;
        y = q / M1 + 1;
        z = q % M1 + 1;
        return true;
    }
}

template <int SUB, int C>
size_t vcycle_cluster_smem_bytes(int levels) {
    using G = SlabGeom<SUB, C>;
    size_t floats = (size_t)(G::P + 2) * G::PS + 2 * (size_t)G::P * G::PS + 4 * (size_t)G::PS;
    size_t total = floats * 4 + (((size_t)G::P * G::PS + 15) & ~size_t(15));
    for (int l = 1; l < levels; ++l) {
        const int e = (SUB >> l) + 1;
        const size_t n4 = ((size_t)e * e * e + 3) & ~size_t(3);
        total += n4 * 13;
    }
    return total;
}

template <int SUB, int C, int NT>
__global__ void __launch_bounds__(NT, 1) vcycle_cluster_kernel(VcycleArgs a) {
    using G = SlabGeom<SUB, C>;
    constexpr int E = G::E, PS = G::PS, P = G::P, M2 = G::M2;
    constexpr int CH = (P * M2 + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ float s_inv[8];
    __shared__ float s_sc64[64];
    __shared__ float s_sc8[8];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int box = blockIdx.x / C;
    if (box >= a.nbox) return;  // uniform across the cluster
    if (a.active && !a.active[blockIdx.y]) return;  // a cluster shares its blockIdx.y
    // System blockIdx.y of a batch: its u and b.
    float* const au = a.u + (size_t)blockIdx.y * a.slot_stride;
    const float* const ab = a.b + (size_t)blockIdx.y * a.slot_stride;
    if (threadIdx.x < 8) s_inv[threadIdx.x] = a.inv_diag[threadIdx.x];
    if (threadIdx.x < 64) s_sc64[threadIdx.x] = a.restrict_w[threadIdx.x];
    if (threadIdx.x < 8) s_sc8[threadIdx.x] = a.prolong_w[threadIdx.x];

    const int x0 = 1 + rank * P;
    const int x1 = min(x0 + P - 1, SUB - 1);
    const int np = x1 - x0 + 1;

    float* u0 = reinterpret_cast<float*>(smem);            // (P+2) planes, plane lx <-> x = x0-1+lx
    float* b0 = u0 + (P + 2) * PS;                          // P planes, plane k <-> x = x0+k
    float* r0 = b0 + P * PS;
    float* nxt = r0 + P * PS;                               // [parity][side][PS], side 0 = low halo
    uint8_t* f0 = reinterpret_cast<uint8_t*>(nxt + 4 * PS);
    LevelSmem lv[kMaxLevels];
    {
        unsigned char* p = reinterpret_cast<unsigned char*>(f0) + (((size_t)P * PS + 15) & ~size_t(15));
        for (int l = 1; l < a.levels; ++l) {
            const int e = (SUB >> l) + 1;
            const int n4 = (e * e * e + 3) & ~3;
            lv[l].e = e;
            lv[l].u = reinterpret_cast<float*>(p); p += n4 * 4;
            lv[l].b = reinterpret_cast<float*>(p); p += n4 * 4;
            lv[l].r = reinterpret_cast<float*>(p); p += n4 * 4;
            lv[l].f = p; p += n4;
        }
    }
    const uint8_t* rec = a.box_flags + (size_t)box * a.box_stride;
    const int tile = a.box_tile[box];
    constexpr int TC = SUB * SUB * SUB;
    const float* gu = au + (size_t)tile * TC;
    const float* gb = ab + (size_t)tile * TC;

    // Load level 0: halo planes / rows from u (interface values) or zero.
    auto load_u = [&](int x, int y, int z) -> float {
        const bool halo = (x == 0) || (y == 0) || (z == 0) || (x == SUB) || (y == SUB) || (z == SUB);
        if (halo && !a.halo_from_u) return 0.0f;
        if (!halo && a.zero_init) return 0.0f;
        const int hi = (x == SUB) + (y == SUB) + (z == SUB);
        if (hi == 0) return gu[(x * SUB + y) * SUB + z];
        if (hi > 1) return 0.0f;  // edge cells are never read by the stencil
        const int axis = (x == SUB) ? 0 : ((y == SUB) ? 1 : 2);
        const int nt = a.box_nb[3 * box + axis];
        if (nt < 0) return 0.0f;
        const int lx = (axis == 0) ? 0 : x, ly = (axis == 1) ? 0 : y, lz = (axis == 2) ? 0 : z;
        return au[(size_t)nt * TC + (lx * SUB + ly) * SUB + lz];
    };
    for (int q = threadIdx.x; q < (np + 2) * PS; q += NT) {
        const int lx = q / PS, rem = q % PS, y = rem / E, z = rem % E;
        u0[q] = load_u(x0 - 1 + lx, y, z);
    }
    for (int q = threadIdx.x; q < P * PS; q += NT) {
        const int k = q / PS, rem = q % PS, y = rem / E, z = rem % E;
        const int x = x0 + k;
        float bv = 0.0f;
        uint8_t fv = 0;
        if (k < np && y >= 1 && y < SUB && z >= 1 && z < SUB) {
            bv = gb[(x * SUB + y) * SUB + z];
            fv = rec[box_index(E, x, y, z)];
        }
        b0[q] = bv;
        // Residual: zero, or the given values at the lower y/z box faces.
        float rv = 0.0f;
        if (a.r_halo && k < np && (y == 0 || z == 0) && y < SUB && z < SUB)
            rv = own_tile_value<SUB>(a.r_halo + (size_t)blockIdx.y * a.slot_stride, tile, x, y, z);
        r0[q] = rv;
        f0[q] = fv;
    }
    if (rank == 0) {
        for (int l = 1; l < a.levels; ++l) {
            const int e = lv[l].e, n = e * e * e;
            for (int i = threadIdx.x; i < n; i += NT) {
                lv[l].u[i] = 0.0f; lv[l].b[i] = 0.0f; lv[l].r[i] = 0.0f;
                lv[l].f[i] = rec[a.level_off[l] + i];
            }
        }
    }
    __syncthreads();
    cluster.sync();  // every CTA's shared memory is initialised before remote access

    float* nb_lo = (rank > 0) ? cluster.map_shared_rank(nxt, rank - 1) : nullptr;   // left neighbour's buffers
    float* nb_hi = (rank < C - 1) ? cluster.map_shared_rank(nxt, rank + 1) : nullptr;
    int par = 0;

    // Each thread owns LPT x-lines (y, z) of the slab, np <= P cells each, and
    // keeps their u, b and flags in registers for the whole V-cycle; shared
    // memory holds u for the y/z neighbours of other threads.
    constexpr int LPT = (M2 + NT - 1) / NT;
    int off[LPT];                 // (y, z) offset within a plane; -1 if no line
    float uu[LPT][P];             // u of the owned cells (shared memory keeps a copy)
    float hlo[LPT], hhi[LPT];     // u at x0-1 and x1+1 of the line
    auto load_lines = [&]() {
#pragma unroll
        for (int l = 0; l < LPT; ++l) {
#pragma unroll
            for (int k = 0; k < P; ++k) uu[l][k] = (off[l] >= 0 && k < np) ? u0[(k + 1) * PS + off[l]] : 0.0f;
        }
    };
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
        off[l] = -1;
        hlo[l] = hhi[l] = 0.0f;
        int y = 0, z = 0;
        if (owned_line<SUB, NT, LPT>(threadIdx.x, l, y, z)) {
            off[l] = y * E + z;
            hlo[l] = u0[off[l]];
            hhi[l] = u0[(np + 1) * PS + off[l]];
        }
    }
    load_lines();
    auto flag = [&](int l, int k) -> uint32_t { return f0[k * PS + off[l]]; };
    // b - A u at owned cell k of line l (reference face order -x,+x,-y,+y,-z,+z).
    auto residual = [&](int l, int k, uint32_t fl) -> float {
        const float cc = uu[l][k];
        float xm = hlo[l], xp = hhi[l];
#pragma unroll
        for (int kk = 0; kk < P; ++kk) {
            if (kk == k - 1) xm = uu[l][kk];
            if (kk == k + 1 && kk < np) xp = uu[l][kk];
        }
        const int i = (k + 1) * PS + off[l];
        float res = 0.0f;
        if (fl & 0x01u) res = __fsub_rn(res, __fsub_rn(xm, cc));
        if (fl & 0x02u) res = __fsub_rn(res, __fsub_rn(xp, cc));
        if (fl & 0x04u) res = __fsub_rn(res, __fsub_rn(u0[i - E], cc));
        if (fl & 0x08u) res = __fsub_rn(res, __fsub_rn(u0[i + E], cc));
        if (fl & 0x10u) res = __fsub_rn(res, __fsub_rn(u0[i - 1], cc));
        if (fl & 0x20u) res = __fsub_rn(res, __fsub_rn(u0[i + 1], cc));
        return __fsub_rn(b0[k * PS + off[l]], res);
    };
    // Send the first/last owned values to the neighbours' halo buffers,
    // barrier, then take this CTA's new halos.
    auto exchange = [&]() {
#pragma unroll
        for (int l = 0; l < LPT; ++l) {
            if (off[l] < 0) continue;
            float last = uu[l][0];
#pragma unroll
            for (int k = 0; k < P; ++k)
                if (k == np - 1) last = uu[l][k];
            // The low neighbour's high halo is this CTA's first plane, and vice versa.
            if (rank > 0) nb_lo[(par * 2 + 1) * PS + off[l]] = uu[l][0];
            if (rank < C - 1) nb_hi[(par * 2 + 0) * PS + off[l]] = last;
        }
        cluster.sync();
#pragma unroll
        for (int l = 0; l < LPT; ++l) {
            if (off[l] < 0) continue;
            if (rank > 0) hlo[l] = nxt[(par * 2 + 0) * PS + off[l]];
            if (rank < C - 1) hhi[l] = nxt[(par * 2 + 1) * PS + off[l]];
        }
        par ^= 1;
    };
    auto slab_sweep = [&](int mode) {
        float rr[LPT][P];
        uint32_t tk[LPT];
#pragma unroll
        for (int l = 0; l < LPT; ++l) {
            tk[l] = 0u;
            if (off[l] < 0) continue;
#pragma unroll
            for (int k = 0; k < P; ++k) {
                rr[l][k] = 0.0f;
                if (k >= np) continue;
                const uint32_t fl = flag(l, k);
                const bool act = fl & C_ACTIVE, bnd = fl & C_BOUNDARY8;
                if (act && ((mode == 3) || (mode == 1 && bnd) || (mode == 2 && !bnd))) {
                    tk[l] |= 1u << k;
                    rr[l][k] = residual(l, k, fl);
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int l = 0; l < LPT; ++l) {
            if (!tk[l]) continue;
#pragma unroll
            for (int k = 0; k < P; ++k) {
                if (tk[l] & (1u << k)) {
                    uu[l][k] = __fadd_rn(uu[l][k], __fmul_rn(s_inv[__popc(flag(l, k) & C_FACES)], rr[l][k]));
                    u0[(k + 1) * PS + off[l]] = uu[l][k];
                }
            }
        }
        exchange();
    };

    const int Lm = a.levels;
    for (int cycle = 0; cycle < a.n_vcycles; ++cycle) {
        if (Lm == 1) {
            for (int i = 0; i < a.bottom_itr; ++i) slab_sweep(3);
            continue;
        }
        for (int i = 0; i < a.boundary_itr; ++i) slab_sweep(1);
        for (int i = 0; i < a.interior_itr; ++i) slab_sweep(2);
        for (int i = 0; i < a.boundary_itr; ++i) slab_sweep(1);
        // r = b - A u on owned Active cells (halos are current after the last exchange).
#pragma unroll
        for (int l = 0; l < LPT; ++l) {
            if (off[l] < 0) continue;
#pragma unroll
            for (int k = 0; k < P; ++k) {
                if (k >= np) continue;
                const uint32_t fl = flag(l, k);
                if (fl & C_ACTIVE) r0[k * PS + off[l]] = residual(l, k, fl);
            }
        }
        __syncthreads();
        cluster.sync();  // r0 of every slab is complete
        // Restriction into rank 0's level-1 b, coarse cells interleaved over ranks.
        {
            constexpr int E1 = SUB / 2 + 1, m1 = SUB / 2 - 1;
            float* b1 = cluster.map_shared_rank(lv[1].b, 0);
            float* r0r[C];
#pragma unroll
            for (int k = 0; k < C; ++k) r0r[k] = cluster.map_shared_rank(r0, k);
            const uint8_t* f1 = rec + a.level_off[1];
            for (int q = threadIdx.x + rank * NT; q < m1 * m1 * m1; q += NT * C) {
                const int cz = q % m1 + 1, t = q / m1, cy = t % m1 + 1, cx = t / m1 + 1;
                const int ci = box_index(E1, cx, cy, cz);
                if (!(f1[ci] & C_ACTIVE)) continue;
                float acc = 0.0f;
#pragma unroll
                for (int i2 = 0; i2 < 4; ++i2) {
                    const int x = 2 * cx - 2 + i2;
                    // x = 0 is no slab's plane; x <= SUB - 1 here (cx <= SUB/2 - 1).
                    const int owner = (x - 1) / P;           // x >= 1 when owner is used
                    const float* rp = (x == 0) ? nullptr : r0r[owner] + (x - 1 - owner * P) * PS;
#pragma unroll
                    for (int j2 = 0; j2 < 4; ++j2)
#pragma unroll
                        for (int k2 = 0; k2 < 4; ++k2) {
                            const int y = 2 * cy - 2 + j2, z = 2 * cz - 2 + k2;
                            float v = 0.0f;
                            if (rp) v = rp[y * E + z];
                            else if (a.r_halo)
                                v = own_tile_value<SUB>(a.r_halo + (size_t)blockIdx.y * a.slot_stride, tile, 0, y, z);
                            acc = __fadd_rn(acc, __fmul_rn(s_sc64[(i2 * 4 + j2) * 4 + k2], v));
                        }
                }
                b1[ci] = acc;
            }
        }
        cluster.sync();  // level-1 b complete in rank 0
        if (rank == 0) {
            const CtaGroup cta;
            zero_u(cta, lv[1]);
            const int T = first_warp_level(SUB, Lm);  // levels T..Lm-1 run in warp 0
            const int Tc = T < Lm ? T : Lm - 1;
            for (int l = 1; l < Tc; ++l) {
                smooth_level<CH>(cta, lv[l], a, s_inv);
                residual_store(cta, lv[l]);
                zero_u(cta, lv[l + 1]);
                restrict_level(cta, lv[l], lv[l + 1], s_sc64);
            }
            if (T < Lm) {
                if (threadIdx.x < 32) vcycle_tail<kWarpCH>(WarpGroup(), lv, T, Lm, a, s_inv, s_sc64, s_sc8);
                __syncthreads();
            } else {
                for (int i = 0; i < a.bottom_itr; ++i) sweep_box<CH>(cta, lv[Lm - 1], 3, s_inv);
            }
            for (int l = Tc - 1; l >= 1; --l) {
                prolongate_level(cta, lv[l], lv[l + 1], s_sc8);
                smooth_level<CH>(cta, lv[l], a, s_inv);
            }
        }
        cluster.sync();  // level-1 u final
        // Prolongation of rank 0's level-1 u into every owned cell.
        {
            constexpr int E1 = SUB / 2 + 1;
            const float* u1 = cluster.map_shared_rank(lv[1].u, 0);
#pragma unroll
            for (int l = 0; l < LPT; ++l) {
                if (off[l] < 0) continue;
                const int y = off[l] / E, z = off[l] % E;
                const int cy = (y + 1) >> 1, cz = (z + 1) >> 1;
                const int py = 1 - (y - (2 * cy - 1)), pz = 1 - (z - (2 * cz - 1));
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    if (k >= np || !(flag(l, k) & C_ACTIVE)) continue;
                    const int x = x0 + k;
                    const int cx = (x + 1) >> 1;
                    const int px = 1 - (x - (2 * cx - 1));
                    const int cbase = box_index(E1, cx, cy, cz);
                    float v = u0[(k + 1) * PS + off[l]];
#pragma unroll
                    for (int aa = 0; aa < 2; ++aa)
#pragma unroll
                        for (int bq = 0; bq < 2; ++bq)
#pragma unroll
                            for (int cq = 0; cq < 2; ++cq) {
                                const float w = s_sc8[((aa ^ px) * 2 + (bq ^ py)) * 2 + (cq ^ pz)];
                                const float cu = u1[cbase + (aa - px) * E1 * E1 + (bq - py) * E1 + (cq - pz)];
                                v = __fadd_rn(v, __fmul_rn(w, cu));
                            }
                    u0[(k + 1) * PS + off[l]] = v;
                }
            }
            load_lines();
            exchange();
        }
        for (int i = 0; i < a.boundary_itr; ++i) slab_sweep(1);
        for (int i = 0; i < a.interior_itr; ++i) slab_sweep(2);
        for (int i = 0; i < a.boundary_itr; ++i) slab_sweep(1);
    }

    float* gw = au + (size_t)tile * TC;
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
        if (off[l] < 0) continue;
        const int y = off[l] / E, z = off[l] % E;
#pragma unroll
        for (int k = 0; k < P; ++k)
            if (k < np) gw[((x0 + k) * SUB + y) * SUB + z] = uu[l][k];
    }
    cluster.sync();  // no CTA leaves while a peer may still address its shared memory
}

// A kernel's dynamic shared-memory limit is process-wide state.  Solvers on
// other host threads launch the same kernels with other level counts, so the
// limit is only ever raised, under a lock: a concurrent launch can never find
// it lowered between its own check and its launch.
std::mutex g_smem_mu;
std::map<std::pair<const void*, int>, size_t> g_smem_limit;

cudaError_t ensure_smem_limit(const void* kern, size_t smem) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_smem_mu);
    size_t& have = g_smem_limit[{kern, dev}];
    if (have >= smem) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) have = smem;
    return e;
}

template <int SUB, int C, int NT>
cudaError_t launch_cluster(const VcycleArgs& a, cudaStream_t stream) {
    const size_t smem = vcycle_cluster_smem_bytes<SUB, C>(a.levels);
    auto kern = vcycle_cluster_kernel<SUB, C, NT>;
    cudaError_t e = ensure_smem_limit((const void*)kern, smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(a.nbox * C), (unsigned)std::max(1, a.nslots), 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, a);
}

}  // namespace

cudaError_t launch_vcycle(const VcycleArgs& a, cudaStream_t stream) {
    if (a.nbox == 0) return cudaSuccess;
    if (a.levels < 1 || a.levels > kMaxLevels) return cudaErrorInvalidValue;
    switch (a.sub) {
        case 8: {
            constexpr int NT = 128;
            const size_t smem = vcycle_smem_bytes<8>(a.levels);
            vcycle_kernel<8, NT><<<dim3(a.nbox, std::max(1, a.nslots)), NT, smem, stream>>>(a);
            return cudaGetLastError();
        }
        case 16: {
            if (a.cluster == 2) return launch_cluster<16, 2, 256>(a, stream);
            constexpr int NT = 512;
            const size_t smem = vcycle_smem_bytes<16>(a.levels);
            cudaError_t e = ensure_smem_limit((const void*)vcycle_kernel<16, NT>, smem);
            if (e != cudaSuccess) return e;
            vcycle_kernel<16, NT><<<dim3(a.nbox, std::max(1, a.nslots)), NT, smem, stream>>>(a);
            return cudaGetLastError();
        }
        case 32:
            return launch_cluster<32, 4, 512>(a, stream);
        default:
            return cudaErrorNotSupported;
    }
}

}  // namespace hdd
