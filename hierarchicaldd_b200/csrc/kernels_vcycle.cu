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
//   correction u += (omega/face_count) * r        (SPGrid_Correction_Legacy.h:161-191)
//   restriction, prolongation weights and order  (SPGrid_Restriction_Legacy.h:47-186,
//                                                 SPGrid_Prolongation_Legacy.h:46-128)
// Smoothing is Jacobi: every residual of a sweep is computed from the old u
// (held in registers) before any update.
#include <cuda_runtime.h>

#include <cstdint>

#include "hdd_common.h"
#include "kernels.h"

namespace hdd {

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

// Interior cell q (0 .. (e-2)^3-1) -> box index.
__device__ __forceinline__ int interior_cell(int e, int q) {
    const int m = e - 2;
    const int z = q % m, t = q / m;
    const int y = t % m, x = t / m;
    return box_index(e, x + 1, y + 1, z + 1);
}

// mode: 1 = boundary cells, 2 = interior (non-boundary) cells, 3 = all Active.
template <int CH>
__device__ void jacobi_sweep(const LevelSmem& L, int mode, const float* inv_diag) {
    const int m = L.e - 2;
    const int ncell = m * m * m;
    float rr[CH];
    int idx[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        const int q = threadIdx.x + c * blockDim.x;
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
    __syncthreads();
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        if (idx[c] >= 0) {
            const int i = idx[c];
            const float w = inv_diag[__popc((uint32_t)L.f[i] & C_FACES)];
            L.u[i] = __fadd_rn(L.u[i], __fmul_rn(w, rr[c]));
        }
    }
    __syncthreads();
}

// r = b - A u at Active cells (other cells of r keep their zero).
__device__ void residual_store(const LevelSmem& L) {
    const int m = L.e - 2;
    const int ncell = m * m * m;
    for (int q = threadIdx.x; q < ncell; q += blockDim.x) {
        const int i = interior_cell(L.e, q);
        const uint32_t fl = L.f[i];
        if (fl & C_ACTIVE) L.r[i] = cell_residual(L, i, fl);
    }
    __syncthreads();
}

__device__ void restrict_level(const LevelSmem& F, const LevelSmem& Cc, const float* sc64) {
    const int m = Cc.e - 2;
    const int ncell = m * m * m;
    const int sx = F.e * F.e, sy = F.e;
    for (int q = threadIdx.x; q < ncell; q += blockDim.x) {
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
    __syncthreads();
}

__device__ void prolongate_level(const LevelSmem& F, const LevelSmem& Cc, const float* sc8) {
    const int m = F.e - 2;
    const int ncell = m * m * m;
    const int csx = Cc.e * Cc.e, csy = Cc.e;
    for (int q = threadIdx.x; q < ncell; q += blockDim.x) {
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
    __syncthreads();
}

template <int SUB, int NT>
__global__ void __launch_bounds__(NT) vcycle_kernel(VcycleArgs a) {
    constexpr int E0 = SUB + 1;
    constexpr int CH = ((SUB - 1) * (SUB - 1) * (SUB - 1) + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ float s_inv[8];
    __shared__ float s_sc64[64];
    __shared__ float s_sc8[8];

    const int box = blockIdx.x;
    if (box >= a.nbox) return;
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
    const float* gu = a.u + (size_t)tile * (SUB * SUB * SUB);
    const float* gb = a.b + (size_t)tile * (SUB * SUB * SUB);

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
            const float* gn = a.u + (size_t)nt * (SUB * SUB * SUB);
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
    __syncthreads();

    const int Lm = a.levels;
    for (int cycle = 0; cycle < a.n_vcycles; ++cycle) {
        for (int l = 0; l < Lm - 1; ++l) {
            for (int i = 0; i < a.boundary_itr; ++i) jacobi_sweep<CH>(lv[l], 1, s_inv);
            for (int i = 0; i < a.interior_itr; ++i) jacobi_sweep<CH>(lv[l], 2, s_inv);
            for (int i = 0; i < a.boundary_itr; ++i) jacobi_sweep<CH>(lv[l], 1, s_inv);
            residual_store(lv[l]);
            {
                const int e = lv[l + 1].e, n = e * e * e;
                for (int i = threadIdx.x; i < n; i += NT) lv[l + 1].u[i] = 0.0f;
            }
            __syncthreads();
            restrict_level(lv[l], lv[l + 1], s_sc64);
        }
        for (int i = 0; i < a.bottom_itr; ++i) jacobi_sweep<CH>(lv[Lm - 1], 3, s_inv);
        for (int l = Lm - 2; l >= 0; --l) {
            prolongate_level(lv[l], lv[l + 1], s_sc8);
            for (int i = 0; i < a.boundary_itr; ++i) jacobi_sweep<CH>(lv[l], 1, s_inv);
            for (int i = 0; i < a.interior_itr; ++i) jacobi_sweep<CH>(lv[l], 2, s_inv);
            for (int i = 0; i < a.boundary_itr; ++i) jacobi_sweep<CH>(lv[l], 1, s_inv);
        }
    }

    // Store the interior cells (1..SUB-1 per axis) of level 0.
    float* gw = a.u + (size_t)tile * (SUB * SUB * SUB);
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

}  // namespace

cudaError_t launch_vcycle(const VcycleArgs& a, cudaStream_t stream) {
    if (a.nbox == 0) return cudaSuccess;
    if (a.levels < 1 || a.levels > kMaxLevels) return cudaErrorInvalidValue;
    switch (a.sub) {
        case 8: {
            constexpr int NT = 128;
            const size_t smem = vcycle_smem_bytes<8>(a.levels);
            vcycle_kernel<8, NT><<<a.nbox, NT, smem, stream>>>(a);
            return cudaGetLastError();
        }
        case 16: {
            constexpr int NT = 512;
            const size_t smem = vcycle_smem_bytes<16>(a.levels);
            cudaError_t e = cudaFuncSetAttribute(vcycle_kernel<16, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            vcycle_kernel<16, NT><<<a.nbox, NT, smem, stream>>>(a);
            return cudaGetLastError();
        }
        default:
            return cudaErrorNotSupported;
    }
}

}  // namespace hdd
