// Supernodal triangular solves on the GPU (the device half of the PARDISO
// stand-in, SIGMA_SMOOTHER.cpp:433-449 phase 33).
//
// Every front J of the nested-dissection tree carries Fw = [L_JJ^{-1}; -W],
// W = L_RJ L_JJ^{-1}, so
//   forward   [y_J; v_J] = Fw f_J + [0; f_R]    (f assembled from b and the children's v)
//   backward  x_J        = Fw^T [y_J; x_R]
// are single dense products.
//
// Fronts with at most kSmallM rows (nearly all fronts of the subdomain-interior
// factors) keep Fw column-major with leading dimension m and no padding, and
// are split into warp tasks: 32 rows each in the forward solve (lanes own
// rows), kBwdCols columns each in the backward solve (lanes stride down the
// columns, then reduce by shuffles); the loads of several columns are in
// flight at once.
// Larger fronts are cut into tasks of kTR rows; a task's coefficients are one
// contiguous block (column-major, kTR rows per column) streamed into shared
// memory with 1D bulk async copies (cp.async.bulk, no multicast) through a
// kNS-stage mbarrier pipeline while the CTA assembles its input vector.
// The fronts and tasks of one tree level form one launch of each kernel.
// Every mbarrier wait is bounded; on timeout the kernel raises the plan's error
// word, drains its own copies (bounded) and returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "dev_util.h"
#include "sigma.h"

namespace hdd {
namespace {

constexpr int kTR = 64;   // rows per task = threads per CTA
constexpr int kCB = 32;   // columns per pipeline stage
constexpr int kNS = 4;    // pipeline stages
constexpr long kWaitLimit = 1L << 22;
constexpr int kSmallM = 256;   // rows of a warp-resident front
constexpr int kWarps = 8;      // warps (fronts) per CTA of the warp-front kernels

struct PlanView {
    const int *col0, *ncol, *nrow;
    const int* rows;
    const long long* rows_off;
    const int *child_ptr, *child;
    const long long* relmap_off;
    const int* relmap;
    const long long* upd_off;
    const int* perm;
    const float* val;
    const float* fw;
    float* upd;
    float* ynew;
    float* xnew;
    int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (long i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

template <int DIR>
__global__ void __launch_bounds__(kTR) sn_task_kernel(PlanView P, const SnTask* __restrict__ tasks,
                                                      const float* __restrict__ b_old, float* __restrict__ x_old) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* stage = reinterpret_cast<float*>(smem_raw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(stage + kNS * kCB * kTR);
    float* vec = reinterpret_cast<float*>(bar + kNS);
    const SnTask t = tasks[blockIdx.x];
    const int J = t.front, nj = P.ncol[J], nr = P.nrow[J], c0 = P.col0[J];
    const int tid = threadIdx.x;
    const int nchunks = (t.ncols + kCB - 1) / kCB;
    const float* src = P.val + t.blk;
    if (tid == 0) {
        for (int s = 0; s < kNS; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int k = 0; k < kNS && k < nchunks; ++k) {
            const uint32_t bytes = (uint32_t)min(kCB, t.ncols - k * kCB) * kTR * 4u;
            mbar_expect_tx(&bar[k], bytes);
            bulk_g2s(stage + k * kCB * kTR, src + (size_t)k * kCB * kTR, bytes, &bar[k]);
        }
    }
    // Input vector, assembled while the first stages are in flight.
    if (DIR == 0) {
        for (int i = tid; i < nj; i += kTR) vec[i] = b_old[P.perm[c0 + i]];
        for (int k = tid; k < nr; k += kTR) vec[nj + k] = 0.0f;
        __syncthreads();
        for (int c = P.child_ptr[J]; c < P.child_ptr[J + 1]; ++c) {
            const int C = P.child[c];
            const int mc = P.nrow[C];
            const float* uc = P.upd + P.upd_off[C];
            const int* rm = P.relmap + P.relmap_off[C];
            for (int k = tid; k < mc; k += kTR) vec[rm[k]] += uc[k];
            __syncthreads();
        }
    } else {
        const int* rows = P.rows + P.rows_off[J];
        for (int a = tid; a < nj; a += kTR) vec[a] = P.ynew[c0 + a];
        for (int k = tid; k < nr; k += kTR) vec[nj + k] = P.xnew[rows[k]];
        __syncthreads();
    }
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    int k = 0;
    bool ok = true;
    for (; k < nchunks; ++k) {
        const int st = k % kNS;
        int done = 1;
        if (tid == 0) done = mbar_wait_bounded(&bar[st], (uint32_t)((k / kNS) & 1)) ? 1 : 0;
        if (!__syncthreads_and(done)) { ok = false; break; }
        // The copy has landed for thread 0's observation; every thread reads
        // after the barrier above.
        const int nc = min(kCB, t.ncols - k * kCB);
        const float* sp = stage + st * kCB * kTR + tid;
        const float* vp = vec + t.col_base + k * kCB;
        int j = 0;
        for (; j + 3 < nc; j += 4) {
            s0 = fmaf(sp[(j + 0) * kTR], vp[j + 0], s0);
            s1 = fmaf(sp[(j + 1) * kTR], vp[j + 1], s1);
            s2 = fmaf(sp[(j + 2) * kTR], vp[j + 2], s2);
            s3 = fmaf(sp[(j + 3) * kTR], vp[j + 3], s3);
        }
        for (; j < nc; ++j) s0 = fmaf(sp[j * kTR], vp[j], s0);
        __syncthreads();  // stage st is free again
        if (tid == 0 && k + kNS < nchunks) {
            const uint32_t bytes = (uint32_t)min(kCB, t.ncols - (k + kNS) * kCB) * kTR * 4u;
            fence_proxy_async();
            mbar_expect_tx(&bar[st], bytes);
            bulk_g2s(stage + st * kCB * kTR, src + (size_t)(k + kNS) * kCB * kTR, bytes, &bar[st]);
        }
    }
    if (!ok) {
        if (tid == 0) {
            atomicExch(P.err, 1);
            // Drain the copies this CTA still has in flight (bounded) before leaving.
            for (int q = k; q < nchunks && q < k + kNS; ++q) mbar_wait_bounded(&bar[q % kNS], (uint32_t)((q / kNS) & 1));
        }
        return;
    }
    const float acc = (s0 + s1) + (s2 + s3);
    const int row = t.rb + tid;
    if (row >= t.re) return;
    if (DIR == 0) {
        if (t.kind == 0) P.ynew[c0 + row] = acc;
        else P.upd[P.upd_off[J] + (row - nj)] = vec[row] + acc;
    } else {
        P.xnew[c0 + row] = acc;
        x_old[P.perm[c0 + row]] = acc;
    }
}

constexpr int kBwdCols = 8;   // columns per backward warp task

// Forward rows [32*part, 32*part+32) of a warp-resident front: y (rows < nj)
// or the update vector f_R - W f_J (rows >= nj).  Linv is lower triangular,
// so rows below 32*part+32 need columns < 32*part+32 only.
__global__ void __launch_bounds__(32 * kWarps) sn_front_forward_kernel(PlanView P, const SnFront* __restrict__ fronts,
                                                                      int nf, const float* __restrict__ b_old) {
    __shared__ float sf[kWarps][kSmallM];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int idx = blockIdx.x * kWarps + w;
    if (idx >= nf) return;
    const SnFront F = fronts[idx];
    const int J = F.front, m = F.m, nj = F.nj, c0 = P.col0[J];
    float* f = sf[w];
    for (int i = lane; i < m; i += 32) f[i] = (i < nj) ? b_old[P.perm[c0 + i]] : 0.0f;
    __syncwarp();
    for (int c = P.child_ptr[J]; c < P.child_ptr[J + 1]; ++c) {
        const int C = P.child[c];
        const int mc = P.nrow[C];
        const float* uc = P.upd + P.upd_off[C];
        const int* rm = P.relmap + P.relmap_off[C];
        for (int k = lane; k < mc; k += 32) f[rm[k]] += uc[k];
        __syncwarp();
    }
    const float* A = P.fw + F.off;
    const int r = 32 * F.part + lane;
    const bool rv = r < m;
    const int cend = min(nj, 32 * F.part + 32);
    float acc = 0.0f;
#pragma unroll 2
    for (int c = 0; c < cend; c += 8) {
#pragma unroll
        for (int t = 0; t < 8; ++t)
            if (rv && c + t < cend) acc = fmaf(A[(size_t)(c + t) * m + r], f[c + t], acc);
    }
    if (!rv) return;
    if (r < nj) P.ynew[c0 + r] = acc;
    else P.upd[P.upd_off[J] + (r - nj)] = f[r] + acc;
}

// Backward columns [kBwdCols*part, +kBwdCols) of a warp-resident front:
// x_a = sum_{r >= a} Fw(r, a) g_r with g = [y_J; x_R].
__global__ void __launch_bounds__(32 * kWarps) sn_front_backward_kernel(PlanView P, const SnFront* __restrict__ fronts,
                                                                       int nf, float* __restrict__ x_old) {
    __shared__ float sg[kWarps][kSmallM];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int idx = blockIdx.x * kWarps + w;
    if (idx >= nf) return;
    const SnFront F = fronts[idx];
    const int J = F.front, m = F.m, nj = F.nj, c0 = P.col0[J];
    const int* rows = P.rows + P.rows_off[J];
    float* g = sg[w];
    const int a0 = kBwdCols * F.part;
    for (int i = (a0 & ~31) + lane; i < m; i += 32) g[i] = (i < nj) ? P.ynew[c0 + i] : P.xnew[rows[i - nj]];
    __syncwarp();
    const float* A = P.fw + F.off;
    float sacc[kBwdCols];
#pragma unroll
    for (int t = 0; t < kBwdCols; ++t) sacc[t] = 0.0f;
    for (int r0 = a0 & ~31; r0 < m; r0 += 32) {
        const int r = r0 + lane;
        if (r >= m) continue;
        const float gr = g[r];
#pragma unroll
        for (int t = 0; t < kBwdCols; ++t)
            if (a0 + t < nj && r >= a0 + t) sacc[t] = fmaf(A[(size_t)(a0 + t) * m + r], gr, sacc[t]);
    }
#pragma unroll
    for (int t = 0; t < kBwdCols; ++t)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sacc[t] += __shfl_xor_sync(0xffffffffu, sacc[t], o);
#pragma unroll
    for (int t = 0; t < kBwdCols; ++t) {
        if (lane == t && a0 + t < nj) {
            P.xnew[c0 + a0 + t] = sacc[t];
            x_old[P.perm[c0 + a0 + t]] = sacc[t];
        }
    }
}

size_t task_smem(int max_front) {
    return (size_t)kNS * kCB * kTR * sizeof(float) + kNS * sizeof(uint64_t) + (size_t)max_front * sizeof(float);
}

}  // namespace

void SolvePlan::build(const std::vector<const SnFactor*>& factors, const std::vector<int>& offsets, cudaStream_t s) {
    release();
    std::vector<int> col0, ncol, nrow, rows, child_ptr{0}, child, relmap, perm, height, depth, parent_g;
    std::vector<long long> rows_off, relmap_off, upd_off;
    n = 0;
    for (size_t f = 0; f < factors.size(); ++f) n = std::max(n, offsets[f] + factors[f]->n);
    perm.assign(n, 0);
    std::vector<int> base(factors.size() + 1, 0);
    for (size_t f = 0; f < factors.size(); ++f) base[f + 1] = base[f] + (int)factors[f]->col0.size();
    nsn = base.back();
    parent_g.assign(nsn, -1);
    std::vector<std::vector<int>> kids(nsn);
    std::vector<std::pair<int, int>> where(nsn);
    for (size_t f = 0; f < factors.size(); ++f) {
        const SnFactor& F = *factors[f];
        if (F.Fw.size() != F.col0.size()) throw Error(HDD_ERR_INTERNAL, "solve blocks not built");
        const int off = offsets[f];
        for (int i = 0; i < F.n; ++i) perm[off + i] = off + F.perm[i];
        for (size_t j = 0; j < F.col0.size(); ++j) {
            const int g = base[f] + (int)j;
            where[g] = {(int)f, (int)j};
            if (F.parent[j] >= 0) {
                parent_g[g] = base[f] + F.parent[j];
                kids[parent_g[g]].push_back(g);
            }
        }
    }
    height.assign(nsn, 0);
    depth.assign(nsn, 0);
    for (int g = 0; g < nsn; ++g)
        if (parent_g[g] >= 0) height[parent_g[g]] = std::max(height[parent_g[g]], height[g] + 1);
    for (int g = nsn - 1; g >= 0; --g)
        if (parent_g[g] >= 0) depth[g] = depth[parent_g[g]] + 1;
    long long upd_total = 0;
    max_front = 0;
    for (int g = 0; g < nsn; ++g) {
        const SnFactor& F = *factors[where[g].first];
        const int j = where[g].second, off = offsets[where[g].first];
        const int nj = F.ncol[j], nr = (int)F.rows[j].size();
        col0.push_back(off + F.col0[j]);
        ncol.push_back(nj);
        nrow.push_back(nr);
        max_front = std::max(max_front, nj + nr);
        rows_off.push_back((long long)rows.size());
        for (int r : F.rows[j]) rows.push_back(off + r);
        upd_off.push_back(upd_total);
        upd_total += nr;
    }
    // Tasks per level and their blocks.
    int hmax = 0, dmax = 0;
    for (int g = 0; g < nsn; ++g) { hmax = std::max(hmax, height[g]); dmax = std::max(dmax, depth[g]); }
    std::vector<SnTask> ftasks, btasks;
    long long total = 0;
    auto add = [&](std::vector<SnTask>& v, int g, int rb, int re, int kind, int cb, int nc) {
        SnTask t;
        t.front = g; t.rb = rb; t.re = re; t.kind = kind; t.col_base = cb; t.ncols = nc; t.pad0 = t.pad1 = 0;
        t.blk = total;
        total += (long long)nc * kTR;
        v.push_back(t);
    };
    // Warp-resident fronts: one Fw block each, 16-byte aligned.
    std::vector<long long> small_off(nsn, -1);
    long long fw_total = 0;
    int big_front = 0;
    for (int g = 0; g < nsn; ++g) {
        const int m = ncol[g] + nrow[g];
        if (m <= kSmallM) {
            small_off[g] = fw_total;
            fw_total += ((long long)m * ncol[g] + 3) & ~3LL;
        } else big_front = std::max(big_front, m);
    }
    std::vector<SnFront> sfwd, sbwd;
    auto small_front = [&](int g, int part) {
        SnFront f;
        f.front = g; f.m = ncol[g] + nrow[g]; f.nj = ncol[g]; f.part = part; f.off = small_off[g];
        return f;
    };
    fwd_ptr.assign(1, 0);
    sfwd_ptr.assign(1, 0);
    for (int h = 0; h <= hmax; ++h) {
        for (int g = 0; g < nsn; ++g) {
            if (height[g] != h) continue;
            const int nj = ncol[g], nr = nrow[g];
            if (small_off[g] >= 0) {
                for (int q = 0; q * 32 < nj + nr; ++q) sfwd.push_back(small_front(g, q));
                continue;
            }
            for (int r0 = 0; r0 < nj; r0 += kTR) add(ftasks, g, r0, std::min(r0 + kTR, nj), 0, 0, std::min(r0 + kTR, nj));
            for (int r0 = nj; r0 < nj + nr; r0 += kTR) add(ftasks, g, r0, std::min(r0 + kTR, nj + nr), 1, 0, nj);
        }
        fwd_ptr.push_back((int)ftasks.size());
        sfwd_ptr.push_back((int)sfwd.size());
    }
    bwd_ptr.assign(1, 0);
    sbwd_ptr.assign(1, 0);
    for (int d = 0; d <= dmax; ++d) {
        for (int g = 0; g < nsn; ++g) {
            if (depth[g] != d) continue;
            const int nj = ncol[g], nr = nrow[g];
            if (small_off[g] >= 0) {
                for (int q = 0; q * kBwdCols < nj; ++q) sbwd.push_back(small_front(g, q));
                continue;
            }
            for (int r0 = 0; r0 < nj; r0 += kTR) add(btasks, g, r0, std::min(r0 + kTR, nj), 2, r0, nj + nr - r0);
        }
        bwd_ptr.push_back((int)btasks.size());
        sbwd_ptr.push_back((int)sbwd.size());
    }
    std::vector<float> fw((size_t)std::max<long long>(fw_total, 4), 0.0f);
#pragma omp parallel for schedule(dynamic)
    for (int g = 0; g < nsn; ++g) {
        if (small_off[g] < 0) continue;
        const SnFactor& F = *factors[where[g].first];
        const std::vector<double>& W = F.Fw[where[g].second];
        float* dst = &fw[(size_t)small_off[g]];
        for (size_t i = 0; i < W.size(); ++i) dst[i] = (float)W[i];
    }
    std::vector<float> val((size_t)total, 0.0f);
    auto fill = [&](const std::vector<SnTask>& v, bool forward) {
#pragma omp parallel for schedule(dynamic)
        for (long q = 0; q < (long)v.size(); ++q) {
            const SnTask& t = v[q];
            const SnFactor& F = *factors[where[t.front].first];
            const int j = where[t.front].second;
            const int m = ncol[t.front] + nrow[t.front];
            const std::vector<double>& W = F.Fw[j];  // (m x nj), col-major: W[c*m + r]
            float* blk = &val[(size_t)t.blk];
            for (int c = 0; c < t.ncols; ++c)
                for (int r = t.rb; r < t.re; ++r) {
                    const int a = t.col_base + c;
                    // forward: M(r, a) = Fw(r, a); backward: M(r, a) = Fw(a, r)
                    const double v2 = forward ? W[(size_t)a * m + r] : W[(size_t)r * m + a];
                    blk[(size_t)c * kTR + (r - t.rb)] = (float)v2;
                }
        }
    };
    fill(ftasks, true);
    fill(btasks, false);
    // Children lists and relative maps (child row -> position in parent's front).
    relmap_off.assign(nsn, 0);
    for (int g = 0; g < nsn; ++g) {
        for (int c : kids[g]) child.push_back(c);
        child_ptr.push_back((int)child.size());
    }
    for (int g = 0; g < nsn; ++g) {
        relmap_off[g] = (long long)relmap.size();
        const int p = parent_g[g];
        if (p < 0) continue;
        const int pc0 = col0[p], pnj = ncol[p];
        const int* prow = rows.data() + rows_off[p];
        const int pnr = nrow[p];
        const int* crow = rows.data() + rows_off[g];
        for (int kq = 0; kq < nrow[g]; ++kq) {
            const int r = crow[kq];
            int posn;
            if (r >= pc0 && r < pc0 + pnj) posn = r - pc0;
            else {
                const int* it = std::lower_bound(prow, prow + pnr, r);
                if (it == prow + pnr || *it != r) throw Error(HDD_ERR_INTERNAL, "supernode row not in parent front");
                posn = pnj + (int)(it - prow);
            }
            relmap.push_back(posn);
        }
    }
    if (nsn == 0) return;
    max_front = std::max(big_front, 1);
    if (task_smem(max_front) > 227 * 1024)
        throw Error(HDD_ERR_UNSUPPORTED, "supernodal front too large for shared memory: " + std::to_string(max_front));
    bytes = 0;
    d_col0 = dev::upload(col0, s, bytes);
    d_ncol = dev::upload(ncol, s, bytes);
    d_nrow = dev::upload(nrow, s, bytes);
    d_rows = dev::upload(rows.empty() ? std::vector<int>{0} : rows, s, bytes);
    d_rows_off = dev::upload(rows_off, s, bytes);
    d_child_ptr = dev::upload(child_ptr, s, bytes);
    d_child = dev::upload(child.empty() ? std::vector<int>{0} : child, s, bytes);
    d_relmap_off = dev::upload(relmap_off, s, bytes);
    d_relmap = dev::upload(relmap.empty() ? std::vector<int>{0} : relmap, s, bytes);
    d_upd_off = dev::upload(upd_off, s, bytes);
    d_perm = dev::upload(perm, s, bytes);
    d_fwd = dev::upload(ftasks.empty() ? std::vector<SnTask>(1) : ftasks, s, bytes);
    d_bwd = dev::upload(btasks.empty() ? std::vector<SnTask>(1) : btasks, s, bytes);
    d_val = dev::upload(val.empty() ? std::vector<float>(4, 0.0f) : val, s, bytes);
    d_sfwd = dev::upload(sfwd.empty() ? std::vector<SnFront>(1) : sfwd, s, bytes);
    d_sbwd = dev::upload(sbwd.empty() ? std::vector<SnFront>(1) : sbwd, s, bytes);
    d_fw = dev::upload(fw, s, bytes);
    d_upd = dev::alloc_zero<float>(std::max<long long>(upd_total, 1), bytes);
    d_ynew = dev::alloc_zero<float>(std::max(n, 1), bytes);
    d_xnew = dev::alloc_zero<float>(std::max(n, 1), bytes);
    d_err = dev::alloc_zero<int>(1, bytes);
    dev::ck(cudaStreamSynchronize(s), "plan upload");
}

void SolvePlan::release() {
    dev::release(d_col0); dev::release(d_ncol); dev::release(d_nrow);
    dev::release(d_rows); dev::release(d_rows_off); dev::release(d_child_ptr); dev::release(d_child);
    dev::release(d_relmap_off); dev::release(d_relmap); dev::release(d_upd_off); dev::release(d_perm);
    dev::release(d_fwd); dev::release(d_bwd); dev::release(d_val); dev::release(d_upd); dev::release(d_ynew);
    dev::release(d_xnew); dev::release(d_err);
    dev::release(d_sfwd); dev::release(d_sbwd); dev::release(d_fw);
    nsn = 0;
    n = 0;
}

void SolvePlan::solve(const float* b_old, float* x_old, cudaStream_t s, long long& launches) const {
    if (nsn == 0) return;
    PlanView P{d_col0, d_ncol, d_nrow, d_rows, d_rows_off, d_child_ptr, d_child, d_relmap_off, d_relmap,
               d_upd_off, d_perm, d_val, d_fw, d_upd, d_ynew, d_xnew, d_err};
    const size_t smem = task_smem(max_front);
    if (smem > 48 * 1024) {
        dev::ck(cudaFuncSetAttribute(sn_task_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
        dev::ck(cudaFuncSetAttribute(sn_task_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
    }
    for (size_t h = 0; h + 1 < fwd_ptr.size(); ++h) {
        const int ns = sfwd_ptr[h + 1] - sfwd_ptr[h];
        if (ns) {
            sn_front_forward_kernel<<<(ns + kWarps - 1) / kWarps, 32 * kWarps, 0, s>>>(P, d_sfwd + sfwd_ptr[h], ns, b_old);
            dev::ck(cudaGetLastError(), "sn front forward");
            ++launches;
        }
        const int cnt = fwd_ptr[h + 1] - fwd_ptr[h];
        if (!cnt) continue;
        sn_task_kernel<0><<<cnt, kTR, smem, s>>>(P, d_fwd + fwd_ptr[h], b_old, x_old);
        dev::ck(cudaGetLastError(), "sn forward");
        ++launches;
    }
    for (size_t d = 0; d + 1 < bwd_ptr.size(); ++d) {
        const int ns = sbwd_ptr[d + 1] - sbwd_ptr[d];
        if (ns) {
            sn_front_backward_kernel<<<(ns + kWarps - 1) / kWarps, 32 * kWarps, 0, s>>>(P, d_sbwd + sbwd_ptr[d], ns, x_old);
            dev::ck(cudaGetLastError(), "sn front backward");
            ++launches;
        }
        const int cnt = bwd_ptr[d + 1] - bwd_ptr[d];
        if (!cnt) continue;
        sn_task_kernel<1><<<cnt, kTR, smem, s>>>(P, d_bwd + bwd_ptr[d], b_old, x_old);
        dev::ck(cudaGetLastError(), "sn backward");
        ++launches;
    }
}

int SolvePlan::error_flag(cudaStream_t s) const {
    if (!d_err) return 0;
    int h = 0;
    dev::ck(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, s), "read error flag");
    dev::ck(cudaStreamSynchronize(s), "read error flag");
    return h;
}

}  // namespace hdd
