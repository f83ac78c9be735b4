// Whole-grid V-cycle, for domains whose coarse levels couple neighbouring
// subdomain boxes (an exterior region touching Active cells, as the
// reference generator's Neumann bubble: a coarse cell whose children are
// exterior and Active is Active, so it joins the boxes on either side of an
// interface plane).  The reference's CPU V-cycle runs on the whole grid
// (CPU/SPGrid_Library/SPGrid_V_Cycle_Helper.h:70-195), and so does this one:
// one launch per Jacobi half-step (residual, then correction), restriction
// and prolongation per level, on dense x-slowest arrays.  Float operations
// are those of the per-box kernels (and the reference), in the same order, so
// the result is the same bit for bit.
//
//   smoothing   SPGrid_Residual_Legacy.h:40-61, SPGrid_Correction_Legacy.h:35-76
//   restriction SPGrid_Restriction_Legacy.h:47-186 (the fine stencil 2c-2..2c+1)
//   prolongation SPGrid_Prolongation_Legacy.h:48-118 (parents (f+1)/2, 3/4-1/4 weights)
#include <cuda_runtime.h>

#include <algorithm>

#include "hdd_common.h"
#include "kernels.h"

namespace hdd {

namespace {

constexpr int kGT = 256;

__device__ __forceinline__ size_t gidx(const int* n, int i, int j, int k) {
    return ((size_t)i * n[1] + j) * n[2] + k;
}

struct Dims3 {
    int n[3];
};

__device__ __forceinline__ float val_or_zero(const Dims3& d, const float* v, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= d.n[0] || j >= d.n[1] || k >= d.n[2]) return 0.0f;
    return v[gidx(d.n, i, j, k)];
}

// r = b - A u at Active cells (face order -x,+x,-y,+y,-z,+z).
__global__ void __launch_bounds__(kGT) g_residual(Dims3 d, const uint8_t* __restrict__ f, const float* __restrict__ u,
                                                  float* __restrict__ r, const float* __restrict__ b, size_t n) {
    const size_t x = (size_t)blockIdx.x * kGT + threadIdx.x;
    if (x >= n) return;
    const uint32_t fl = f[x];
    if (!(fl & C_ACTIVE)) return;
    const int k = (int)(x % d.n[2]);
    const size_t t = x / d.n[2];
    const int j = (int)(t % d.n[1]), i = (int)(t / d.n[1]);
    const float c = u[x];
    float res = 0.0f;
    if (fl & 0x01u) res = __fsub_rn(res, __fsub_rn(val_or_zero(d, u, i - 1, j, k), c));
    if (fl & 0x02u) res = __fsub_rn(res, __fsub_rn(val_or_zero(d, u, i + 1, j, k), c));
    if (fl & 0x04u) res = __fsub_rn(res, __fsub_rn(val_or_zero(d, u, i, j - 1, k), c));
    if (fl & 0x08u) res = __fsub_rn(res, __fsub_rn(val_or_zero(d, u, i, j + 1, k), c));
    if (fl & 0x10u) res = __fsub_rn(res, __fsub_rn(val_or_zero(d, u, i, j, k - 1), c));
    if (fl & 0x20u) res = __fsub_rn(res, __fsub_rn(val_or_zero(d, u, i, j, k + 1), c));
    r[x] = __fsub_rn(b[x], res);
}

// u += omega/face_count * r on the cells of the sweep: mode 1 Boundary,
// 2 interior (Active, not Boundary), 3 all Active.
__global__ void __launch_bounds__(kGT) g_correct(const uint8_t* __restrict__ f, float* __restrict__ u,
                                                 const float* __restrict__ r, size_t n, int mode, VcycleWeights w) {
    const size_t x = (size_t)blockIdx.x * kGT + threadIdx.x;
    if (x >= n) return;
    const uint32_t fl = f[x];
    if (!(fl & C_ACTIVE)) return;
    const bool bnd = fl & C_BOUNDARY8;
    if (!((mode == 3) || (mode == 1 && bnd) || (mode == 2 && !bnd))) return;
    u[x] = __fadd_rn(u[x], __fmul_rn(w.inv_diag[__popc(fl & C_FACES)], r[x]));
}

// Coarse b at Active coarse cells from the fine residual (every fine cell of
// the stencil, whatever its flag; outside the grid counts zero).
__global__ void __launch_bounds__(kGT) g_restrict(Dims3 cd, const uint8_t* __restrict__ cf, float* __restrict__ cb,
                                                  Dims3 fd, const float* __restrict__ fr, size_t n, VcycleWeights w) {
    const size_t x = (size_t)blockIdx.x * kGT + threadIdx.x;
    if (x >= n) return;
    if (!(cf[x] & C_ACTIVE)) return;
    const int k = (int)(x % cd.n[2]);
    const size_t t = x / cd.n[2];
    const int j = (int)(t % cd.n[1]), i = (int)(t / cd.n[1]);
    float acc = 0.0f;
#pragma unroll
    for (int i2 = 0; i2 < 4; ++i2)
#pragma unroll
        for (int j2 = 0; j2 < 4; ++j2)
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2)
                acc = __fadd_rn(acc, __fmul_rn(w.restrict_w[(i2 * 4 + j2) * 4 + k2],
                                               val_or_zero(fd, fr, 2 * i - 2 + i2, 2 * j - 2 + j2, 2 * k - 2 + k2)));
    cb[x] = acc;
}

// Fine u += prolongated coarse u at Active fine cells.
__global__ void __launch_bounds__(kGT) g_prolong(Dims3 fd, const uint8_t* __restrict__ ff, float* __restrict__ fu,
                                                 Dims3 cd, const float* __restrict__ cu, size_t n, VcycleWeights w) {
    const size_t x = (size_t)blockIdx.x * kGT + threadIdx.x;
    if (x >= n) return;
    if (!(ff[x] & C_ACTIVE)) return;
    const int k = (int)(x % fd.n[2]);
    const size_t t = x / fd.n[2];
    const int j = (int)(t % fd.n[1]), i = (int)(t / fd.n[1]);
    const int ci = (i + 1) >> 1, cj = (j + 1) >> 1, ck = (k + 1) >> 1;
    const int pi = 1 - (i - (2 * ci - 1)), pj = 1 - (j - (2 * cj - 1)), pk = 1 - (k - (2 * ck - 1));
    float acc = fu[x];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int e = 0; e < 2; ++e)
                acc = __fadd_rn(acc, __fmul_rn(w.prolong_w[((a ^ pi) * 2 + (b ^ pj)) * 2 + (e ^ pk)],
                                               val_or_zero(cd, cu, ci + a - pi, cj + b - pj, ck + e - pk)));
    fu[x] = acc;
}

// Level-0 staging between the tiled vectors and the dense arrays.
// to_dense: dense[c] = tiled value (0 outside stored tiles) where keep[c],
// else 0; keep = Active when active_only, else every cell.
__global__ void __launch_bounds__(kGT) g_from_tiles(TileGeom g, const int* __restrict__ txyz, Dims3 d,
                                                    const float* __restrict__ tiled, float* __restrict__ dense,
                                                    const uint8_t* __restrict__ f0, int drop_active,
                                                    int drop_other) {
    const int t = blockIdx.x, S = g.sub, TC = S * S * S;
    const int ox = txyz[3 * t] * S, oy = txyz[3 * t + 1] * S, oz = txyz[3 * t + 2] * S;
    for (int c = threadIdx.x; c < TC; c += kGT) {
        const int z = c % S, tt = c / S, y = tt % S, xx = tt / S;
        const int gx = ox + xx, gy = oy + y, gz = oz + z;
        if (gx >= d.n[0] || gy >= d.n[1] || gz >= d.n[2]) continue;
        const size_t di = gidx(d.n, gx, gy, gz);
        const bool act = f0[di] & C_ACTIVE;
        float v = tiled[(size_t)t * TC + c];
        if ((act && drop_active) || (!act && drop_other)) v = 0.0f;
        dense[di] = v;
    }
}

// tiled[c] = dense at every stored cell that is not Interface (the V-cycle's
// cells; the interface values stay as they are).
__global__ void __launch_bounds__(kGT) g_to_tiles(TileGeom g, const int* __restrict__ txyz, Dims3 d,
                                                  const float* __restrict__ dense, float* __restrict__ tiled) {
    const int t = blockIdx.x, S = g.sub, TC = S * S * S;
    const int ox = txyz[3 * t] * S, oy = txyz[3 * t + 1] * S, oz = txyz[3 * t + 2] * S;
    for (int c = threadIdx.x; c < TC; c += kGT) {
        const int z = c % S, tt = c / S, y = tt % S, xx = tt / S;
        const int gx = ox + xx, gy = oy + y, gz = oz + z;
        if (gx >= d.n[0] || gy >= d.n[1] || gz >= d.n[2]) continue;
        const size_t q = (size_t)t * TC + c;
        if (g.flags[q] & C_INTERFACE) continue;
        tiled[q] = dense[gidx(d.n, gx, gy, gz)];
    }
}

unsigned blocks_for(size_t n) { return (unsigned)((n + kGT - 1) / kGT); }

}  // namespace

long long launch_vcycle_global(const GlobalVcycleArgs& a, const TileGeom& g, const int* tile_xyz, float* u,
                               const float* b, const float* r_halo, cudaStream_t st) {
    long long launches = 0;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess) throw Error(HDD_ERR_CUDA, std::string("whole-grid V-cycle: ") + cudaGetErrorString(e));
    };
    auto dims = [&](int l) {
        Dims3 d;
        for (int q = 0; q < 3; ++q) d.n[q] = a.dims[l][q];
        return d;
    };
    auto count = [&](int l) { return (size_t)a.dims[l][0] * a.dims[l][1] * a.dims[l][2]; };
    const Dims3 d0 = dims(0);
    const size_t n0 = count(0);
    // Level-0 state: b from the tiles; u's interface (halo) values and/or
    // initial interior from the tiles; r zero, or the given face residual.
    ok(cudaMemsetAsync(a.b[0], 0, n0 * sizeof(float), st));
    g_from_tiles<<<g.ntiles, kGT, 0, st>>>(g, tile_xyz, d0, b, a.b[0], a.f[0], 0, 0);
    ok(cudaMemsetAsync(a.u[0], 0, n0 * sizeof(float), st));
    if (a.halo_from_u || !a.zero_init)
        g_from_tiles<<<g.ntiles, kGT, 0, st>>>(g, tile_xyz, d0, u, a.u[0], a.f[0], a.zero_init, !a.halo_from_u);
    ok(cudaMemsetAsync(a.r[0], 0, n0 * sizeof(float), st));
    if (r_halo) g_from_tiles<<<g.ntiles, kGT, 0, st>>>(g, tile_xyz, d0, r_halo, a.r[0], a.f[0], 1, 0);
    launches += 3;
    const int L = a.levels;
    auto smooth = [&](int l, int mode) {
        g_residual<<<blocks_for(count(l)), kGT, 0, st>>>(dims(l), a.f[l], a.u[l], a.r[l], a.b[l], count(l));
        g_correct<<<blocks_for(count(l)), kGT, 0, st>>>(a.f[l], a.u[l], a.r[l], count(l), mode, a.w);
        launches += 2;
    };
    for (int cycle = 0; cycle < a.n_vcycles; ++cycle) {
        for (int l = 0; l + 1 < L; ++l) {
            for (int i = 0; i < a.boundary_itr; ++i) smooth(l, 1);
            for (int i = 0; i < a.interior_itr; ++i) smooth(l, 2);
            for (int i = 0; i < a.boundary_itr; ++i) smooth(l, 1);
            g_residual<<<blocks_for(count(l)), kGT, 0, st>>>(dims(l), a.f[l], a.u[l], a.r[l], a.b[l], count(l));
            ok(cudaMemsetAsync(a.u[l + 1], 0, count(l + 1) * sizeof(float), st));
            g_restrict<<<blocks_for(count(l + 1)), kGT, 0, st>>>(dims(l + 1), a.f[l + 1], a.b[l + 1], dims(l), a.r[l],
                                                                  count(l + 1), a.w);
            launches += 2;
        }
        const int lb = L - 1;
        g_residual<<<blocks_for(count(lb)), kGT, 0, st>>>(dims(lb), a.f[lb], a.u[lb], a.r[lb], a.b[lb], count(lb));
        for (int i = 0; i < a.bottom_itr; ++i) smooth(lb, 3);
        g_residual<<<blocks_for(count(lb)), kGT, 0, st>>>(dims(lb), a.f[lb], a.u[lb], a.r[lb], a.b[lb], count(lb));
        launches += 2;
        for (int l = L - 2; l >= 0; --l) {
            g_prolong<<<blocks_for(count(l)), kGT, 0, st>>>(dims(l), a.f[l], a.u[l], dims(l + 1), a.u[l + 1], count(l),
                                                             a.w);
            ++launches;
            for (int i = 0; i < a.boundary_itr; ++i) smooth(l, 1);
            for (int i = 0; i < a.interior_itr; ++i) smooth(l, 2);
            for (int i = 0; i < a.boundary_itr; ++i) smooth(l, 1);
        }
    }
    g_to_tiles<<<g.ntiles, kGT, 0, st>>>(g, tile_xyz, d0, a.u[0], u);
    ++launches;
    ok(cudaGetLastError());
    return launches;
}

}  // namespace hdd
