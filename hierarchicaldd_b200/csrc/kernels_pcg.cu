// PCG vector kernels over tiled vectors (HBM-streaming), sm_100a.
//
// Semantics follow CG_SYSTEM / CG_VECTOR / CONJUGATE_GRADIENT of the reference
// (CPU/SPGrid_Domain_Decomposition_Solver/CG_SYSTEM.cpp:28-119,
//  CG_VECTOR.cpp:56-74, PB/.../Krylov_Solvers/CONJUGATE_GRADIENT.cpp:30-60):
// the Laplacian accumulates in FP64 and rounds to FP32, dot products sum FP32
// products in FP64, and vector updates are FP32 a*c+b without contraction.
// Per-tile partial sums are reduced in a fixed order, so every sum is
// deterministic for a given layout.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <cstdlib>

#include "hdd_common.h"
#include "kernels.h"

namespace hdd {

namespace {

constexpr int kNT = 256;

// Value of the face neighbour `face` of local cell (x,y,z) of tile t.
template <class V>
__device__ __forceinline__ V nb_value(const TileGeom& g, const V* v, int t, int x, int y, int z, int face) {
    const int S = g.sub;
    int nx = x, ny = y, nz = z, tt = t;
    switch (face) {
        case 0: if (x > 0) nx = x - 1; else { tt = g.nbr[6 * t + 0]; nx = S - 1; } break;
        case 1: if (x < S - 1) nx = x + 1; else { tt = g.nbr[6 * t + 1]; nx = 0; } break;
        case 2: if (y > 0) ny = y - 1; else { tt = g.nbr[6 * t + 2]; ny = S - 1; } break;
        case 3: if (y < S - 1) ny = y + 1; else { tt = g.nbr[6 * t + 3]; ny = 0; } break;
        case 4: if (z > 0) nz = z - 1; else { tt = g.nbr[6 * t + 4]; nz = S - 1; } break;
        default: if (z < S - 1) nz = z + 1; else { tt = g.nbr[6 * t + 5]; nz = 0; } break;
    }
    if (tt < 0) return V(0);
    return v[(size_t)tt * S * S * S + (nx * S + ny) * S + nz];
}

template <class V>
__device__ __forceinline__ double laplace_cell(const TileGeom& g, const V* v, int t, int x, int y, int z,
                                               uint32_t fl, V c) {
    const double cd = (double)c;
    double result = 0.0;
#pragma unroll
    for (int face = 0; face < 6; ++face)
        if (fl & (1u << face)) result -= ((double)nb_value(g, v, t, x, y, z, face) - cd);
    return result;
}

template <class T>
__device__ __forceinline__ T block_sum(T v) {
    __shared__ T red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < (int)(blockDim.x >> 5)) ? red[l] : T(0);
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

__device__ __forceinline__ float block_max(float v) {
    __shared__ float red[32];
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    return v;
}

__global__ void __launch_bounds__(kNT) laplace_dot_kernel(TileGeom g, const float* __restrict__ s,
                                                          float* __restrict__ q, double* partial, size_t vstride,
                                                          int pstride) {
    s += (size_t)blockIdx.y * vstride;
    q += (size_t)blockIdx.y * vstride;
    partial += (size_t)blockIdx.y * pstride;
    const int t = blockIdx.x;
    const int S = g.sub, TC = S * S * S;
    const size_t base = (size_t)t * TC;
    double acc = 0.0;
    for (int c = threadIdx.x; c < TC; c += kNT) {
        const uint32_t fl = g.flags[base + c];
        float out = 0.0f;
        const float sv = s[base + c];
        if (fl & (C_ACTIVE | C_INTERFACE)) {
            const int z = c % S, tmp = c / S, y = tmp % S, x = tmp / S;
            out = (float)laplace_cell(g, s, t, x, y, z, fl, sv);
        }
        q[base + c] = out;
        acc += (double)(sv * out);
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[t] = acc;
}

// q = Project(A s) and per-work-unit partial sums of s*q, marching x-planes.
//
// A group of S*S/4 threads covers one x-plane of a tile, one float4 of four
// z-consecutive cells per thread (thread i: row y = i / (S/4), quad zq =
// i % (S/4)); a CTA of 256 threads holds G = 1024 / (S*S) groups, each
// marching over the planes [x0, x0 + S/SLABS) of its own (tile, slab) unit.
// Every cell value is read from HBM once per launch: the x neighbours stay in
// registers (previous / current / prefetched next plane), the y neighbours
// come from the current plane staged in shared memory (double-buffered, one
// barrier per plane), the z neighbours from the adjacent lanes of the row
// (shuffles); only the tile-face halos are read from the neighbouring tiles.
// The arithmetic per cell is laplace_cell's (FP64 face sums, faces -x,+x,-y,
// +y,-z,+z), so q is bit-identical to it; the dot sums the same FP32 products
// in FP64 in a fixed order per unit.
template <int S, int SLABS>
struct MarchShape {
    static constexpr int P = S / 4;           // quads per row
    static constexpr int GT = S * S / 4;      // threads per group (one plane)
    static constexpr int G = kNT / GT;        // groups per CTA
    static constexpr int NP = S / SLABS;      // planes per unit
};

template <int S, int SLABS>
__global__ void __launch_bounds__(kNT, 4) laplace_dot_march_kernel(TileGeom g, const float* __restrict__ s,
                                                                float* __restrict__ q, double* partial,
                                                                size_t vstride, int pstride) {
    using M = MarchShape<S, SLABS>;
    s += (size_t)blockIdx.y * vstride;
    q += (size_t)blockIdx.y * vstride;
    partial += (size_t)blockIdx.y * pstride;
    constexpr int P = M::P, GT = M::GT, NP = M::NP, S2 = S * S, S3 = S * S * S;
    __shared__ float4 plane[2][kNT];
    __shared__ double red[kNT / 32];
    const int i = threadIdx.x % GT, grp = threadIdx.x / GT;
    const long long unit = (long long)blockIdx.x * M::G + grp;
    const bool valid = unit < (long long)g.ntiles * SLABS;
    const int t = valid ? (int)(unit / SLABS) : 0;
    const int x0 = valid ? (int)(unit % SLABS) * NP : 0;
    const int y = i / P, zq = i % P;
    const size_t tb = (size_t)t * S3;
    const int nb[6] = {g.nbr[6 * t + 0], g.nbr[6 * t + 1], g.nbr[6 * t + 2],
                       g.nbr[6 * t + 3], g.nbr[6 * t + 4], g.nbr[6 * t + 5]};
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    // float4 of this thread's cells in plane xx of tile tt (zero if absent).
    auto load4 = [&](int tt, int xx) -> float4 {
        if (!valid || tt < 0) return zero4;
        return __ldg(reinterpret_cast<const float4*>(s + (size_t)tt * S3 + (size_t)xx * S2) + i);
    };
    auto flags4 = [&](int xx) -> uint2 {
        if (!valid) return make_uint2(0u, 0u);
        return __ldg(reinterpret_cast<const uint2*>(g.flags + tb + (size_t)xx * S2) + i);
    };
    // Plane x (0 <= x < S) of this tile, or the neighbouring tile's face
    // plane for x = -1 and x = S.
    auto plane4 = [&](int xx) -> float4 {
        if (xx < 0) return load4(nb[0], S - 1);
        if (xx >= S) return load4(nb[1], 0);
        return load4(t, xx);
    };
    // Two planes are in flight ahead of the one being computed.
    float4 prev = plane4(x0 - 1);
    float4 cur = plane4(x0);
    float4 nxt = plane4(x0 + 1);
    uint2 fcur = flags4(x0);
    uint2 fnxt = NP > 1 ? flags4(x0 + 1) : make_uint2(0u, 0u);
    double acc = 0.0;
#pragma unroll 1
    for (int k = 0; k < NP; ++k) {
        const int x = x0 + k;
        const float4 nxt2 = k + 2 <= NP ? plane4(x + 2) : zero4;
        const uint2 fnxt2 = k + 2 < NP ? flags4(x + 2) : make_uint2(0u, 0u);
        // Tile-face halos of this plane (y rows and z ends).
        float4 ym = zero4, yp = zero4;
        float zm = 0.f, zp = 0.f;
        if (valid) {
            if (y == 0 && nb[2] >= 0)
                ym = __ldg(reinterpret_cast<const float4*>(s + (size_t)nb[2] * S3 + (size_t)x * S2 + (S - 1) * S) + zq);
            if (y == S - 1 && nb[3] >= 0)
                yp = __ldg(reinterpret_cast<const float4*>(s + (size_t)nb[3] * S3 + (size_t)x * S2) + zq);
            if (zq == 0 && nb[4] >= 0) zm = __ldg(s + (size_t)nb[4] * S3 + (size_t)x * S2 + y * S + (S - 1));
            if (zq == P - 1 && nb[5] >= 0) zp = __ldg(s + (size_t)nb[5] * S3 + (size_t)x * S2 + y * S);
        }
        float4* buf = plane[k & 1];
        buf[threadIdx.x] = cur;
        __syncthreads();
        if (y > 0) ym = buf[threadIdx.x - P];
        if (y < S - 1) yp = buf[threadIdx.x + P];
        const float zl = __shfl_up_sync(0xffffffffu, cur.w, 1);
        const float zr = __shfl_down_sync(0xffffffffu, cur.x, 1);
        if (zq > 0) zm = zl;
        if (zq < P - 1) zp = zr;
        const float cv[4] = {cur.x, cur.y, cur.z, cur.w};
        const float xm[4] = {prev.x, prev.y, prev.z, prev.w};
        const float xp[4] = {nxt.x, nxt.y, nxt.z, nxt.w};
        const float ymv[4] = {ym.x, ym.y, ym.z, ym.w};
        const float ypv[4] = {yp.x, yp.y, yp.z, yp.w};
        const uint32_t fw[4] = {fcur.x & 0xffffu, fcur.x >> 16, fcur.y & 0xffffu, fcur.y >> 16};
        float out[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t fl = fw[e];
            out[e] = 0.0f;
            if (fl & (C_ACTIVE | C_INTERFACE)) {
                const double cd = (double)cv[e];
                const float zmv = e == 0 ? zm : cv[e > 0 ? e - 1 : 0];
                const float zpv = e == 3 ? zp : cv[e < 3 ? e + 1 : 3];
                double r = 0.0;
                if (fl & 1u) r -= ((double)xm[e] - cd);
                if (fl & 2u) r -= ((double)xp[e] - cd);
                if (fl & 4u) r -= ((double)ymv[e] - cd);
                if (fl & 8u) r -= ((double)ypv[e] - cd);
                if (fl & 16u) r -= ((double)zmv - cd);
                if (fl & 32u) r -= ((double)zpv - cd);
                out[e] = (float)r;
            }
            acc += (double)(cv[e] * out[e]);
        }
        if (valid)
            reinterpret_cast<float4*>(q + tb + (size_t)x * S2)[i] = make_float4(out[0], out[1], out[2], out[3]);
        prev = cur;
        cur = nxt;
        nxt = nxt2;
        fcur = fnxt;
        fnxt = fnxt2;
    }
    // Per-unit sums: warps never straddle groups (GT is a multiple of 32 or
    // the group is a half or quarter warp, summed by masked shuffles below).
    if (GT >= 32) {
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) red[w] = acc;
        __syncthreads();
        constexpr int WPG = GT / 32;  // warps per group
        if (threadIdx.x < M::G) {
            const long long u = (long long)blockIdx.x * M::G + threadIdx.x;
            double v = 0.0;
            for (int j = 0; j < WPG; ++j) v += red[threadIdx.x * WPG + j];
            if (u < (long long)g.ntiles * SLABS) partial[u] = v;
        }
    } else {
        for (int o = GT / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, GT);
        if (i == 0 && valid) partial[unit] = acc;
    }
}

// precise = 0: r = b - (float)(A x), the reference's float subtraction;
// precise = 1: r = (float)(b - A x) with A x kept in FP64 (the FP64 true
// residual of the precision form).
__global__ void __launch_bounds__(kNT) residual_kernel(TileGeom g, const float* __restrict__ b,
                                                       const float* __restrict__ x, float* __restrict__ r,
                                                       float* partial_max, int precise) {
    const int t = blockIdx.x;
    const int S = g.sub, TC = S * S * S;
    const size_t base = (size_t)t * TC;
    float m = 0.0f;
    for (int c = threadIdx.x; c < TC; c += kNT) {
        const uint32_t fl = g.flags[base + c];
        float out = 0.0f;
        if (fl & (C_ACTIVE | C_INTERFACE)) {
            const int z = c % S, tmp = c / S, y = tmp % S, xx = tmp / S;
            const double axd = laplace_cell(g, x, t, xx, y, z, fl, x[base + c]);
            out = precise ? (float)((double)b[base + c] - axd) : __fsub_rn(b[base + c], (float)axd);
        }
        r[base + c] = out;
        m = fmaxf(m, fabsf(out));
    }
    m = block_max(m);
    if (threadIdx.x == 0) partial_max[t] = m;
}

// r = (float)(b - A x) for an FP64 iterate x (the precision form's true
// residual), FP64 throughout; partial max|r|.
__global__ void __launch_bounds__(kNT) residual_f64_kernel(TileGeom g, const float* __restrict__ b,
                                                           const double* __restrict__ x, float* __restrict__ r,
                                                           float* partial_max, Batch B) {
    if (B.active && !B.active[blockIdx.y]) return;
    b += (size_t)blockIdx.y * B.vstride;
    x += (size_t)blockIdx.y * B.vstride;
    r += (size_t)blockIdx.y * B.vstride;
    partial_max += (size_t)blockIdx.y * B.pstride;
    const int t = blockIdx.x;
    const int S = g.sub, TC = S * S * S;
    const size_t base = (size_t)t * TC;
    float m = 0.0f;
    for (int c = threadIdx.x; c < TC; c += kNT) {
        const uint32_t fl = g.flags[base + c];
        float out = 0.0f;
        if (fl & (C_ACTIVE | C_INTERFACE)) {
            const int z = c % S, tmp = c / S, y = tmp % S, xx = tmp / S;
            out = (float)((double)b[base + c] - laplace_cell(g, x, t, xx, y, z, fl, x[base + c]));
        }
        r[base + c] = out;
        m = fmaxf(m, fabsf(out));
    }
    m = block_max(m);
    if (threadIdx.x == 0) partial_max[t] = m;
}

__global__ void __launch_bounds__(kNT) project_dot_kernel(TileGeom g, float* __restrict__ a,
                                                          const float* __restrict__ bv, double* partial,
                                                          size_t vstride, int pstride) {
    a += (size_t)blockIdx.y * vstride;
    bv += (size_t)blockIdx.y * vstride;
    partial += (size_t)blockIdx.y * pstride;
    const int t = blockIdx.x;
    const int TC = g.sub * g.sub * g.sub;
    const size_t base = (size_t)t * TC;
    double acc = 0.0;
    for (int c = threadIdx.x; c < TC; c += kNT) {
        const uint32_t fl = g.flags[base + c];
        float av = a[base + c];
        if (!(fl & (C_ACTIVE | C_INTERFACE))) { av = 0.0f; a[base + c] = 0.0f; }
        acc += (double)(av * bv[base + c]);
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[t] = acc;
}

__global__ void __launch_bounds__(kNT) project_kernel(TileGeom g, float* __restrict__ a) {
    const int t = blockIdx.x;
    const int TC = g.sub * g.sub * g.sub;
    const size_t base = (size_t)t * TC;
    for (int c = threadIdx.x; c < TC; c += kNT)
        if (!(g.flags[base + c] & (C_ACTIVE | C_INTERFACE))) a[base + c] = 0.0f;
}

__global__ void __launch_bounds__(kNT) update_s_kernel(size_t n, float* __restrict__ s,
                                                       const float* __restrict__ z, const PcgScalars* sc,
                                                       int first, int mode, Batch B) {
    const int j = blockIdx.y;
    if (B.active && !B.active[j]) return;
    if (B.first) first = B.first[j];
    s += (size_t)j * B.vstride;
    z += (size_t)j * B.vstride;
    sc += j;
    const float beta = sc->beta;
    const double beta_d = sc->beta_d;
    for (size_t i = blockIdx.x * (size_t)kNT + threadIdx.x; i < n; i += (size_t)gridDim.x * kNT) {
        if (first) s[i] = z[i];
        else if (mode == 0) s[i] = __fadd_rn(__fmul_rn(s[i], beta), z[i]);
        else s[i] = (float)((double)s[i] * beta_d + (double)z[i]);
    }
}

// xd (mode 1, optional): the FP64 iterate, updated as xd += alpha s with x
// its FP32 rounding.
__global__ void __launch_bounds__(kNT) update_xr_kernel(int TC, float* __restrict__ x, float* __restrict__ r,
                                                        const float* __restrict__ s, const float* __restrict__ q,
                                                        const PcgScalars* sc, int mode, float* partial_max,
                                                        double* __restrict__ xd, Batch B) {
    const int j = blockIdx.y;
    if (B.active && !B.active[j]) return;
    const size_t so = (size_t)j * B.vstride;
    x += so; r += so; s += so; q += so;
    if (xd) xd += so;
    partial_max += (size_t)j * B.pstride;
    sc += j;
    const int t = blockIdx.x;
    const size_t base = (size_t)t * TC;
    const float alpha = sc->alpha;
    const double alpha_d = sc->alpha_d;
    float m = 0.0f;
    for (int c = threadIdx.x; c < TC; c += kNT) {
        const size_t i = base + c;
        float xv, rv;
        if (mode == 0) {
            xv = __fadd_rn(__fmul_rn(s[i], alpha), x[i]);
            rv = __fadd_rn(__fmul_rn(q[i], -alpha), r[i]);
        } else if (xd) {
            const double xn = xd[i] + alpha_d * (double)s[i];
            xd[i] = xn;
            xv = (float)xn;
            rv = (float)((double)r[i] - alpha_d * (double)q[i]);
        } else {
            xv = (float)((double)x[i] + alpha_d * (double)s[i]);
            rv = (float)((double)r[i] - alpha_d * (double)q[i]);
        }
        x[i] = xv;
        r[i] = rv;
        m = fmaxf(m, fabsf(rv));
    }
    m = block_max(m);
    if (threadIdx.x == 0) partial_max[t] = m;
}

__global__ void reduce_sum_kernel(const double* partial, int n, double* out, int pstride, int ostride) {
    partial += (size_t)blockIdx.x * pstride;
    out += (size_t)blockIdx.x * ostride;
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

__global__ void reduce_max_kernel(const float* partial, int n, float* out, int pstride, int ostride) {
    partial += (size_t)blockIdx.x * pstride;
    out += (size_t)blockIdx.x * ostride;
    float m = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, partial[i]);
    m = block_max(m);
    if (threadIdx.x == 0) *out = m;
}

__global__ void scalar_rho_kernel(PcgScalars* sc, const double* rho_sum, int first, Batch B, int sstride) {
    const int j = threadIdx.x;
    if (j >= B.k || (B.active && !B.active[j])) return;
    if (B.first) first = B.first[j];
    sc += j;
    rho_sum += (size_t)j * sstride;
    const double rd = *rho_sum;
    sc->rho_d = rd;
    sc->rho = (float)rd;
    if (!first) {
        sc->beta = sc->rho / sc->rho_old;
        sc->beta_d = rd / sc->rho_old_d;
        if (!isfinite(sc->beta) || !isfinite(sc->beta_d)) sc->status = 1;
    }
    if (!isfinite(rd)) sc->status = 1;
}

__global__ void scalar_alpha_kernel(PcgScalars* sc, const double* sdq_sum, Batch B, int sstride) {
    const int j = threadIdx.x;
    if (j >= B.k || (B.active && !B.active[j])) return;
    sc += j;
    sdq_sum += (size_t)j * sstride;
    const double sd = *sdq_sum;
    sc->sdq_d = sd;
    const float sdq = (float)sd;
    sc->alpha = sdq != 0.0f ? sc->rho / sdq : FLT_MAX;  // CONJUGATE_GRADIENT.cpp:57
    sc->alpha_d = sd != 0.0 ? sc->rho_d / sd : (double)FLT_MAX;
    sc->rho_old = sc->rho;
    sc->rho_old_d = sc->rho_d;
    sc->iteration += 1;
    if (!isfinite(sd) || !isfinite(sc->alpha)) sc->status = 1;
}

template <int MODE>
__global__ void __launch_bounds__(kNT) interface_gather_kernel(const long long* slot, const int* nbs, int n,
                                                               const float* r, const float* z, float* b0,
                                                               size_t vstride, size_t istride) {
    r += (size_t)blockIdx.y * vstride;
    z += (size_t)blockIdx.y * vstride;
    b0 += (size_t)blockIdx.y * istride;
    const int i = blockIdx.x * kNT + threadIdx.x;
    if (i >= n) return;
    double result = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int s = nbs[6 * i + q];
        if (s >= 0) result -= (double)z[s];
    }
    if (MODE == kGatherIr) b0[i] = -(float)result;
    else if (MODE == kGatherIrTiled) b0[slot[i]] = -(float)result;
    else if (MODE == kGatherRiAdd) b0[i] = __fadd_rn(b0[i], __fsub_rn(r[slot[i]], (float)result));
    else b0[i] = __fsub_rn(r[slot[i]], (float)result);
}

__global__ void __launch_bounds__(kNT) interface_scatter_kernel(const long long* slot, int n, const float* u0,
                                                                float* z, size_t vstride, size_t istride) {
    u0 += (size_t)blockIdx.y * istride;
    z += (size_t)blockIdx.y * vstride;
    const int i = blockIdx.x * kNT + threadIdx.x;
    if (i < n) z[slot[i]] = u0[i];
}

template <class V>
__global__ void __launch_bounds__(kNT) dense_tiles_kernel(int S, const int* tile_xyz, int sx, int sy, int sz,
                                                          const V* __restrict__ src, V* __restrict__ dst,
                                                          int to_tiles) {
    const int t = blockIdx.x, TC = S * S * S;
    const int ox = tile_xyz[3 * t] * S, oy = tile_xyz[3 * t + 1] * S, oz = tile_xyz[3 * t + 2] * S;
    for (int c = threadIdx.x; c < TC; c += kNT) {
        const int z = c % S, tmp = c / S, y = tmp % S, x = tmp / S;
        const int gx = ox + x, gy = oy + y, gz = oz + z;
        const bool in = gx < sx && gy < sy && gz < sz;
        const size_t di = ((size_t)gx * sy + gy) * sz + gz, ti = (size_t)t * TC + c;
        if (to_tiles) dst[ti] = in ? src[di] : V(0);
        else if (in) dst[di] = src[ti];
    }
}

}  // namespace

cudaError_t launch_dense_to_tiles(const TileGeom& g, const int* txyz, int sx, int sy, int sz, const float* dense,
                                  float* tiled, cudaStream_t st) {
    if (g.ntiles == 0) return cudaSuccess;
    dense_tiles_kernel<<<g.ntiles, kNT, 0, st>>>(g.sub, txyz, sx, sy, sz, dense, tiled, 1);
    return cudaGetLastError();
}
cudaError_t launch_tiles_to_dense(const TileGeom& g, const int* txyz, int sx, int sy, int sz, const float* tiled,
                                  float* dense, cudaStream_t st) {
    if (g.ntiles == 0) return cudaSuccess;
    dense_tiles_kernel<<<g.ntiles, kNT, 0, st>>>(g.sub, txyz, sx, sy, sz, tiled, dense, 0);
    return cudaGetLastError();
}

cudaError_t launch_tiles_to_dense_f64(const TileGeom& g, const int* txyz, int sx, int sy, int sz, const double* tiled,
                                      double* dense, cudaStream_t st) {
    if (g.ntiles == 0) return cudaSuccess;
    dense_tiles_kernel<<<g.ntiles, kNT, 0, st>>>(g.sub, txyz, sx, sy, sz, tiled, dense, 0);
    return cudaGetLastError();
}

// Work units of the marching Laplacian: (tile, slab) pairs, four slabs of 8
// planes per 32^3 tile, so that a 256^3 domain gives 2048 CTAs, 3.5 waves of
// 4 per SM (measured at 256^3: 1, 2 and 4 slabs give 2326, 2442 and 2543
// GB/s; the halo planes a slab reads twice cost less than the tail of fewer,
// longer units).
static int laplace_slabs(int sub) { return sub == 32 ? 4 : 1; }

int laplace_partials(const TileGeom& g) {
    if (g.sub == 8 || g.sub == 16 || g.sub == 32) return g.ntiles * laplace_slabs(g.sub);
    return g.ntiles;
}

template <int S, int SLABS>
static void launch_march(const TileGeom& g, const float* s, float* q, double* partial, cudaStream_t st,
                         const Batch& B) {
    using M = MarchShape<S, SLABS>;
    const long long units = (long long)g.ntiles * SLABS;
    const int grid = (int)((units + M::G - 1) / M::G);
    laplace_dot_march_kernel<S, SLABS><<<dim3(grid, B.k), kNT, 0, st>>>(g, s, q, partial, B.vstride, B.pstride);
}

cudaError_t launch_laplace_dot(const TileGeom& g, const float* s, float* q, double* partial, cudaStream_t st,
                               const Batch& B) {
    if (g.ntiles == 0) return cudaSuccess;
    switch (g.sub) {
        case 32: launch_march<32, 4>(g, s, q, partial, st, B); break;
        case 16: launch_march<16, 1>(g, s, q, partial, st, B); break;
        case 8: launch_march<8, 1>(g, s, q, partial, st, B); break;
        default:
            laplace_dot_kernel<<<dim3(g.ntiles, B.k), kNT, 0, st>>>(g, s, q, partial, B.vstride, B.pstride);
            break;
    }
    return cudaGetLastError();
}
cudaError_t launch_residual(const TileGeom& g, const float* b, const float* x, float* r, float* pm, cudaStream_t st,
                            int precise) {
    if (g.ntiles == 0) return cudaSuccess;
    residual_kernel<<<g.ntiles, kNT, 0, st>>>(g, b, x, r, pm, precise);
    return cudaGetLastError();
}
cudaError_t launch_residual_f64(const TileGeom& g, const float* b, const double* x, float* r, float* pm,
                                cudaStream_t st, const Batch& B) {
    if (g.ntiles == 0) return cudaSuccess;
    residual_f64_kernel<<<dim3(g.ntiles, B.k), kNT, 0, st>>>(g, b, x, r, pm, B);
    return cudaGetLastError();
}
cudaError_t launch_project_dot(const TileGeom& g, float* a, const float* b, double* partial, cudaStream_t st,
                               const Batch& B) {
    if (g.ntiles == 0) return cudaSuccess;
    project_dot_kernel<<<dim3(g.ntiles, B.k), kNT, 0, st>>>(g, a, b, partial, B.vstride, B.pstride);
    return cudaGetLastError();
}
cudaError_t launch_project(const TileGeom& g, float* v, cudaStream_t st) {
    if (g.ntiles == 0) return cudaSuccess;
    project_kernel<<<g.ntiles, kNT, 0, st>>>(g, v);
    return cudaGetLastError();
}
cudaError_t launch_update_s(const TileGeom& g, float* s, const float* z, const PcgScalars* sc, int first, int mode,
                            cudaStream_t st, const Batch& B) {
    const size_t n = (size_t)g.ntiles * g.sub * g.sub * g.sub;
    if (n == 0) return cudaSuccess;
    int blocks = (int)((n + kNT - 1) / kNT);
    if (blocks > 148 * 16) blocks = 148 * 16;
    update_s_kernel<<<dim3(blocks, B.k), kNT, 0, st>>>(n, s, z, sc, first, mode, B);
    return cudaGetLastError();
}
cudaError_t launch_update_xr(const TileGeom& g, float* x, float* r, const float* s, const float* q,
                             const PcgScalars* sc, int mode, float* pm, cudaStream_t st, double* xd, const Batch& B) {
    if (g.ntiles == 0) return cudaSuccess;
    update_xr_kernel<<<dim3(g.ntiles, B.k), kNT, 0, st>>>(g.sub * g.sub * g.sub, x, r, s, q, sc, mode, pm, xd, B);
    return cudaGetLastError();
}
cudaError_t launch_reduce_sum(const double* partial, int n, double* out, cudaStream_t st, const Batch& B,
                              int ostride) {
    reduce_sum_kernel<<<B.k, 1024, 0, st>>>(partial, n, out, B.pstride, ostride);
    return cudaGetLastError();
}
cudaError_t launch_reduce_max(const float* partial, int n, float* out, cudaStream_t st, const Batch& B, int ostride) {
    reduce_max_kernel<<<B.k, 1024, 0, st>>>(partial, n, out, B.pstride, ostride);
    return cudaGetLastError();
}
cudaError_t launch_scalar_rho(PcgScalars* sc, const double* rho_sum, int first, cudaStream_t st, const Batch& B,
                              int sstride) {
    scalar_rho_kernel<<<1, 32, 0, st>>>(sc, rho_sum, first, B, sstride);
    return cudaGetLastError();
}
cudaError_t launch_scalar_alpha(PcgScalars* sc, const double* sdq_sum, cudaStream_t st, const Batch& B,
                                int sstride) {
    scalar_alpha_kernel<<<1, 32, 0, st>>>(sc, sdq_sum, B, sstride);
    return cudaGetLastError();
}
cudaError_t launch_interface_gather(const TileGeom&, const long long* slot, const int* nbs, int n, const float* r,
                                    const float* z, float* b0, cudaStream_t st, const Batch& B, size_t istride,
                                    int mode) {
    if (n == 0) return cudaSuccess;
    const dim3 grid((n + kNT - 1) / kNT, B.k);
    if (mode == kGatherIr)
        interface_gather_kernel<kGatherIr><<<grid, kNT, 0, st>>>(slot, nbs, n, r, z, b0, B.vstride, istride);
    else if (mode == kGatherRiAdd)
        interface_gather_kernel<kGatherRiAdd><<<grid, kNT, 0, st>>>(slot, nbs, n, r, z, b0, B.vstride, istride);
    else if (mode == kGatherIrTiled)
        interface_gather_kernel<kGatherIrTiled><<<grid, kNT, 0, st>>>(slot, nbs, n, r, z, b0, B.vstride, istride);
    else
        interface_gather_kernel<kGatherRi><<<grid, kNT, 0, st>>>(slot, nbs, n, r, z, b0, B.vstride, istride);
    return cudaGetLastError();
}
cudaError_t launch_interface_scatter(const long long* slot, int n, const float* u0, float* z, cudaStream_t st,
                                     const Batch& B, size_t istride) {
    if (n == 0) return cudaSuccess;
    interface_scatter_kernel<<<dim3((n + kNT - 1) / kNT, B.k), kNT, 0, st>>>(slot, n, u0, z, B.vstride, istride);
    return cudaGetLastError();
}

}  // namespace hdd
