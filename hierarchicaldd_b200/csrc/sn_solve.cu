// Supernodal triangular solves on the GPU (the device half of the PARDISO
// stand-in; the reference's phase-33 solves are in
// CPU/Interface_Solver/SIGMA_SMOOTHER.cpp:293-324).
//
// Every front J of the nested-dissection forest carries
// Fw = [L_JJ^{-1}; -L_RJ L_JJ^{-1}] (m = nj + nr rows, nj columns), stored once,
// column-major with leading dimension round4(m), so
//   forward   [y_J; v_J] = Fw f_J + [0; f_R]   (f assembled from b and the children's v)
//   backward  x_J        = Fw^T [y_J; x_R]
// are dense products over the same coefficients.  The coefficients are FP32
// (what the HBM stream carries); products are accumulated in FP64 (every
// FP32 x FP32 product is exact in FP64) and the vectors passed between fronts
// (the assembled f, y, x and the update vectors) are FP64, so a solve rounds
// to FP32 once, at its output, like the FP64 substitution it replaces up to
// the rounding of the stored coefficients.
//
// Each direction is ONE persistent launch.  Its work is a list of tasks in
// topological order (forward: children before parents; backward: parents
// before children); CTAs take tasks by ticket and, before starting one, wait
// on per-front completion counters of the fronts it depends on.  A task only
// ever waits on tasks with smaller tickets, which running CTAs already hold,
// so the walk always progresses; every wait is bounded anyway and raises the
// plan's error word when it gives up.  Data produced by other CTAs in the same
// launch is read with L2-coherent loads after an acquire of the counter.
//
// Small fronts (a few row chunks times few columns) go in bundles of one per
// warp, so that many short dependency chains run per CTA.  Other
// forward tasks are row blocks of up to kRB rows; a CTA splits its threads
// into row lanes x column slices and adds the slices in a fixed order.  Tall
// fronts whose row block needs more than kCC columns are split into column
// blocks: each writes its partial sums and the last one to finish adds them in
// column order, so every result is independent of scheduling.  Backward tasks
// are blocks of kBC columns, one warp per column group, lanes striding down
// the contiguous columns.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "dev_util.h"
#include "sigma.h"

namespace hdd {
namespace {

// Threads per CTA: a plan of many independent factors (the subdomain
// interiors) runs 64-thread CTAs, many of them per SM for its many short
// tasks; a plan of one factor (the interface) runs 256-thread CTAs, which do
// its tall fronts in fewer tasks.  Measured at 256^3, level-0 interior plan
// forward / backward: 801 / 836 us with 256 threads, 650 / 760 with 128,
// 577 / 711 with 64; level-0 interface plan: 480 / 596 us with 256 threads,
// 662 / 731 with 128, 703 / 565 with 512.
constexpr int kNTInterior = 64, kNTInterface = 256;
constexpr int kRB = 128;                 // rows per forward row block
constexpr int kCC = 128;                 // columns per forward column block
// Small fronts per bundle (one per warp) and columns per backward task (4 per
// warp), for NT threads.
__host__ __device__ constexpr int warps_of(int nt) { return nt / 32; }
__host__ __device__ constexpr int bc_of(int nt) { return 4 * (nt / 32); }
// CTAs per SM the register budget is sized for (K right-hand sides, NT threads).
__host__ __device__ constexpr int min_blocks(int k, int nt) { return (k == 1 ? 1280 : (k == 2 ? 768 : 512)) / nt; }
constexpr int kSmallM = 256;             // rows of a front solved by one warp
constexpr int kSmallLoads = 128;         // ... when its row chunks x columns stay below this

constexpr int kBundleLevel = 2048;       // bundle only on levels with at least this many small fronts

bool small_front(int m, int nj) { return m <= kSmallM && ((m + 31) / 32) * nj <= kSmallLoads; }

struct PlanView {
    int nsn, max_m;
    const int *col0, *ncol, *nrow, *parent;
    const int* rows;
    const long long* rows_off;
    const int *child_ptr, *child;
    const long long* relmap_off;
    const int* relmap;
    // Gather lists: position p of front J's input vector receives the update
    // entries gent[ge_off[J] + gptr[gp_off[J] + p] .. gptr[gp_off[J] + p + 1])
    // (indices into upd), in child order.
    const long long *gp_off, *ge_off;
    const int *gptr, *gent;
    const long long* upd_off;
    const long long* fw_off;
    const int *ntf, *ntb;
    const int* perm;
    const int *bfwd, *bbwd;
    const float* fw;
    double* part;
    double* upd;
    double* ynew;
    double* xnew;
    int* ctr;
    int* err;
    long long spin_limit;  // polls (with ~128 ns sleeps) before a wait gives up
    // Right-hand side j (of K solved together) uses part + j ld_part,
    // upd + j ld_upd, ynew / xnew + j ld_n, b_old + j ld_b, x_old + j ld_x.
    long long ld_part, ld_upd, ld_n, ld_b, ld_x;
};

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Waits until *p >= target; false when the wait gave up, or at once when an
// earlier wait of this launch already gave up (so one failure cannot turn
// into a long chain of timeouts).
__device__ bool wait_at_least(const int* p, int target, const int* err, long long limit) {
    for (long long i = 0; i < limit; ++i) {
        if (ld_acquire(p) >= target) return true;
        if (ld_acquire(err) != 0) return false;
        __nanosleep(128);
    }
    return false;
}

__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

// Four FP64 fused multiply-adds acc[e] += v.e * x.
__device__ __forceinline__ void fma4(double (&acc)[4], const float4 v, double x) {
    acc[0] = fma((double)v.x, x, acc[0]);
    acc[1] = fma((double)v.y, x, acc[1]);
    acc[2] = fma((double)v.z, x, acc[2]);
    acc[3] = fma((double)v.w, x, acc[3]);
}

// Fw is stored column-major with a leading dimension of round4(m) and
// columns starting on 16-byte boundaries, so four consecutive rows of a column
// are one 16-byte load.  Entries above the diagonal of L_JJ^{-1} and the
// padding rows m .. round4(m) are stored zeros: a load may cover them.
//
// K right-hand sides are solved together: each coefficient load feeds K
// products.  A front's vectors in shared memory hold entry i of right-hand
// side j at i * K + j.  Every right-hand side's arithmetic (which products,
// summed in which order) is the same for every K, so a solve's result does not
// depend on what it was batched with.

// Forward solve of one small front by one warp: the lane owns the row quads
// 4 * (lane + 32 q), q < MQ.
template <int MQ, int K>
__device__ __forceinline__ void warp_forward_rows(const PlanView& P, int J, int m, int nj, const double* f, int lane) {
    const size_t ld = (size_t)((m + 3) & ~3);
    const float* A = P.fw + P.fw_off[J];
    double acc[MQ][K][4];
#pragma unroll
    for (int q = 0; q < MQ; ++q)
#pragma unroll
        for (int j = 0; j < K; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[q][j][e] = 0.0;
#pragma unroll 4
    for (int c = 0; c < nj; ++c) {
        double fc[K];
#pragma unroll
        for (int j = 0; j < K; ++j) fc[j] = f[(size_t)c * K + j];
        const float* col = A + (size_t)c * ld;
#pragma unroll
        for (int q = 0; q < MQ; ++q) {
            const int r = 4 * (lane + 32 * q);
            if (r < m && r + 3 >= c) {
                const float4 v = ldg4(col + r);
#pragma unroll
                for (int j = 0; j < K; ++j) fma4(acc[q][j], v, fc[j]);
            }
        }
    }
    const int c0 = P.col0[J];
    const long long uo = P.upd_off[J];
#pragma unroll
    for (int q = 0; q < MQ; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int r = 4 * (lane + 32 * q) + e;
            if (r >= m) continue;
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (r < nj) P.ynew[j * P.ld_n + c0 + r] = acc[q][j][e];
                else P.upd[j * P.ld_upd + uo + (r - nj)] = f[(size_t)r * K + j] + acc[q][j][e];
            }
        }
}

template <int K>
__device__ void warp_forward(const PlanView& P, int J, double* f, int lane, const float* b_old, int* done) {
    const int nj = P.ncol[J], m = nj + P.nrow[J], c0 = P.col0[J];
    const int cb = P.child_ptr[J], ce = P.child_ptr[J + 1];
    for (int i = lane; i < m; i += 32) {
        const int po = i < nj ? P.perm[c0 + i] : 0;
#pragma unroll
        for (int j = 0; j < K; ++j) f[(size_t)i * K + j] = (i < nj) ? (double)b_old[j * P.ld_b + po] : 0.0;
    }
    if (lane == 0) {
        bool ok = true;
        for (int c = cb; c < ce; ++c) ok &= wait_at_least(done + P.child[c], P.ntf[P.child[c]], P.err, P.spin_limit);
        if (!ok) atomicExch(P.err, 1);
    }
    __syncwarp();
    for (int c = cb; c < ce; ++c) {
        const int C = P.child[c];
        const int mc = P.nrow[C];
        const double* uc = P.upd + P.upd_off[C];
        const int* rm = P.relmap + P.relmap_off[C];
        for (int k = lane; k < mc; k += 32) {
            const int t = rm[k];
#pragma unroll
            for (int j = 0; j < K; ++j) f[(size_t)t * K + j] += __ldcg(uc + j * P.ld_upd + k);
        }
        __syncwarp();
    }
    if (m <= 128) warp_forward_rows<1, K>(P, J, m, nj, f, lane);
    else warp_forward_rows<2, K>(P, J, m, nj, f, lane);
    __threadfence();
    __syncwarp();
    if (lane == 0) atomicAdd(done + J, 1);
}

// Backward solve of one small front by one warp: x_a = sum_{r >= a} Fw(r, a) g_r,
// four columns at a time, the lane summing the row quads a + 4 lane + 128 k.
template <int K>
__device__ void warp_backward(const PlanView& P, int J, double* g, int lane, float* x_old, int* done) {
    const int nj = P.ncol[J], m = nj + P.nrow[J], c0 = P.col0[J];
    const int m4 = (m + 3) & ~3;
    const int* rows = P.rows + P.rows_off[J];
    for (int i = lane; i < nj; i += 32)  // from the forward launch
#pragma unroll
        for (int j = 0; j < K; ++j) g[(size_t)i * K + j] = P.ynew[j * P.ld_n + c0 + i];
    for (int i = m + lane; i < m4; i += 32)  // padding rows
#pragma unroll
        for (int j = 0; j < K; ++j) g[(size_t)i * K + j] = 0.0;
    if (lane == 0) {
        const int p = P.parent[J];
        if (p >= 0 && !wait_at_least(done + p, P.ntb[p], P.err, P.spin_limit)) atomicExch(P.err, 1);
    }
    __syncwarp();
    for (int i = nj + lane; i < m; i += 32) {
        const int t = rows[i - nj];
#pragma unroll
        for (int j = 0; j < K; ++j) g[(size_t)i * K + j] = __ldcg(P.xnew + j * P.ld_n + t);
    }
    __syncwarp();
    const size_t ld = (size_t)m4;
    const float* A = P.fw + P.fw_off[J];
    for (int a = 0; a < nj; a += 4) {
        double s4[K][4];
#pragma unroll
        for (int j = 0; j < K; ++j)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) s4[j][jj] = 0.0;
#pragma unroll 2
        for (int r = a + 4 * lane; r < m; r += 128) {
            double gg[K][4];
#pragma unroll
            for (int j = 0; j < K; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) gg[j][e] = g[(size_t)(r + e) * K + j];
#pragma unroll
            for (int jj = 0; jj < 4; ++jj)
                if (a + jj < nj) {
                    const float4 v = ldg4(A + (size_t)(a + jj) * ld + r);
#pragma unroll
                    for (int j = 0; j < K; ++j) {
                        s4[j][jj] = fma((double)v.x, gg[j][0], s4[j][jj]);
                        s4[j][jj] = fma((double)v.y, gg[j][1], s4[j][jj]);
                        s4[j][jj] = fma((double)v.z, gg[j][2], s4[j][jj]);
                        s4[j][jj] = fma((double)v.w, gg[j][3], s4[j][jj]);
                    }
                }
        }
#pragma unroll
        for (int j = 0; j < K; ++j)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s4[j][jj] += __shfl_xor_sync(0xffffffffu, s4[j][jj], o);
        if (lane == 0) {
#pragma unroll
            for (int jj = 0; jj < 4; ++jj)
                if (a + jj < nj) {
                    const int po = P.perm[c0 + a + jj];
#pragma unroll
                    for (int j = 0; j < K; ++j) {
                        P.xnew[j * P.ld_n + c0 + a + jj] = s4[j][jj];
                        x_old[j * P.ld_x + po] = (float)s4[j][jj];
                    }
                }
        }
    }
    __threadfence();
    __syncwarp();
    if (lane == 0) atomicAdd(done + J, 1);
}

template <int K, int NT>
__global__ void __launch_bounds__(NT, min_blocks(K, NT))
    sn_forward_kernel(PlanView P, const SnTask* __restrict__ tasks, int ntasks, const float* __restrict__ b_old) {
    extern __shared__ double sh[];
    double* f = sh;                    // the front's input vectors, m x K entries
    double* red = sh + P.max_m * K;    // column-slice partial sums, 4 K NT entries
    __shared__ int s_ticket, s_last;
    int* done = P.ctr + 2;
    int* chunk_ctr = P.ctr + 2 + 2 * P.nsn;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_ticket = atomicAdd(P.ctr + 0, 1);
        __syncthreads();
        const int t = s_ticket;
        if (t >= ntasks) break;
        const SnTask T = tasks[t];
        if (T.front < 0) {
            const int w = tid >> 5;
            if (w < T.rows) warp_forward<K>(P, P.bfwd[T.r0 + w], sh + (size_t)w * kSmallM * K, tid & 31, b_old, done);
            __syncthreads();
            continue;
        }
        const int J = T.front, nj = P.ncol[J], m = nj + P.nrow[J], c0 = P.col0[J];
        const int cb = P.child_ptr[J], ce = P.child_ptr[J + 1];
        // Row quads x column slices: the block's rows in quads of four (one
        // 16-byte load per column), mq quad lanes per slice, ks slices.  Each
        // thread's first four coefficient loads are issued before the
        // dependency wait and the assembly.
        const int nq = (T.rows + 3) >> 2;
        const int mq = nq <= 8 ? 8 : (nq <= 16 ? 16 : 32);
        const int ks = NT / mq;
        const int sl = tid / mq, lq = tid - sl * mq;
        const int row = T.r0 + 4 * lq;
        const bool active = lq < nq;
        int cbeg = 0, cend = 0;
        const size_t ld = (size_t)((m + 3) & ~3);
        const float* A = P.fw + P.fw_off[J] + row;
        if (active) {
            const int cs = (T.ncols + ks - 1) / ks;
            cbeg = T.c0 + sl * cs;
            cend = min(T.c0 + T.ncols, cbeg + cs);
            if (row < nj) cend = min(cend, row + 4);  // L_JJ^{-1} is lower triangular
        }
        float4 v0[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            v0[u] = (cbeg + u < cend) ? ldg4(A + (size_t)(cbeg + u) * ld) : make_float4(0.f, 0.f, 0.f, 0.f);
        if constexpr (NT < 128) {
            // Small fronts (the interior plans' 64-thread CTAs): the whole
            // input vectors, b's part before the wait, then each child's
            // update scattered in, child by child.
            for (int i = tid; i < m; i += NT) {
                const int po = i < nj ? P.perm[c0 + i] : 0;
#pragma unroll
                for (int j = 0; j < K; ++j) f[(size_t)i * K + j] = (i < nj) ? (double)b_old[j * P.ld_b + po] : 0.0;
            }
            if (tid == 0) {
                bool ok = true;
                for (int c = cb; c < ce; ++c)
                    ok &= wait_at_least(done + P.child[c], P.ntf[P.child[c]], P.err, P.spin_limit);
                if (!ok) atomicExch(P.err, 1);
            }
            __syncthreads();
            for (int c = cb; c < ce; ++c) {
                const int C = P.child[c];
                const int mc = P.nrow[C];
                const double* uc = P.upd + P.upd_off[C];
                const int* rm = P.relmap + P.relmap_off[C];
                for (int k = tid; k < mc; k += NT) {
                    const int tr = rm[k];
#pragma unroll
                    for (int j = 0; j < K; ++j) f[(size_t)tr * K + j] += __ldcg(uc + j * P.ld_upd + k);
                }
                __syncthreads();
            }
        } else {
            // Tall fronts (the interface plans): only the positions this task
            // reads, its columns [T.c0, T.c0 + T.ncols) and its update rows
            // [max(T.r0, nj), rend); b's part before the wait, then each
            // position adds its children's update entries in child order,
            // the same sums as the whole-front scatter above.  Measured: the
            // level-0 interface forward drops from 485 to 436 us.
            const int rlo = max(T.r0, nj), nrn = max(0, T.r0 + T.rows - rlo);
            const int nneed = T.ncols + nrn;
            for (int q = tid; q < nneed; q += NT) {
                const int p = q < T.ncols ? T.c0 + q : rlo + (q - T.ncols);
                const int po = p < nj ? P.perm[c0 + p] : 0;
#pragma unroll
                for (int j = 0; j < K; ++j) f[(size_t)p * K + j] = (p < nj) ? (double)b_old[j * P.ld_b + po] : 0.0;
            }
            if (tid == 0) {
                bool ok = true;
                for (int c = cb; c < ce; ++c)
                    ok &= wait_at_least(done + P.child[c], P.ntf[P.child[c]], P.err, P.spin_limit);
                if (!ok) atomicExch(P.err, 1);
            }
            __syncthreads();
            if (ce > cb) {
                const int* gp = P.gptr + P.gp_off[J];
                const int* ge = P.gent + P.ge_off[J];
                for (int q = tid; q < nneed; q += NT) {
                    const int p = q < T.ncols ? T.c0 + q : rlo + (q - T.ncols);
                    double v[K];
#pragma unroll
                    for (int j = 0; j < K; ++j) v[j] = f[(size_t)p * K + j];
                    for (int e = gp[p]; e < gp[p + 1]; ++e) {
                        const int ui = ge[e];
#pragma unroll
                        for (int j = 0; j < K; ++j) v[j] += __ldcg(P.upd + j * P.ld_upd + ui);
                    }
#pragma unroll
                    for (int j = 0; j < K; ++j) f[(size_t)p * K + j] = v[j];
                }
                __syncthreads();
            }
        }
        double acc[K][4];
#pragma unroll
        for (int j = 0; j < K; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[j][e] = 0.0;
        if (active) {
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (cbeg + u < cend)
#pragma unroll
                    for (int j = 0; j < K; ++j) fma4(acc[j], v0[u], f[(size_t)(cbeg + u) * K + j]);
            int c = cbeg + 4;
            for (; c + 4 <= cend; c += 4) {
#pragma unroll
                for (int u = 0; u < 4; ++u) v0[u] = ldg4(A + (size_t)(c + u) * ld);
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int j = 0; j < K; ++j) fma4(acc[j], v0[u], f[(size_t)(c + u) * K + j]);
            }
            for (; c < cend; ++c) {
                const float4 v = ldg4(A + (size_t)c * ld);
#pragma unroll
                for (int j = 0; j < K; ++j) fma4(acc[j], v, f[(size_t)c * K + j]);
            }
        }
        if (ks > 1) {
#pragma unroll
            for (int j = 0; j < K; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) red[(size_t)(j * 4 + e) * NT + tid] = acc[j][e];
            __syncthreads();
            if (sl == 0 && active) {
#pragma unroll
                for (int j = 0; j < K; ++j)
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        double s2 = red[(size_t)(j * 4 + e) * NT + lq];
                        for (int q = 1; q < ks; ++q) s2 += red[(size_t)(j * 4 + e) * NT + q * mq + lq];
                        acc[j][e] = s2;
                    }
            }
        }
        const bool mine = sl == 0 && active;
        const int rend = T.r0 + T.rows;
        if (T.nk == 1) {
            if (mine) {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = row + e;
                    if (r >= rend) break;
#pragma unroll
                    for (int j = 0; j < K; ++j) {
                        if (r < nj) P.ynew[j * P.ld_n + c0 + r] = acc[j][e];
                        else P.upd[j * P.ld_upd + P.upd_off[J] + (r - nj)] = f[(size_t)r * K + j] + acc[j][e];
                    }
                }
            }
        } else {
            if (mine) {
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    double* pp = P.part + j * P.ld_part + T.part + (size_t)T.k * kRB + 4 * lq;
#pragma unroll
                    for (int e = 0; e < 4; ++e) pp[e] = acc[j][e];
                }
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) s_last = (atomicAdd(chunk_ctr + T.chunk, 1) == T.nk - 1);
            __syncthreads();
            if (s_last) {
                __threadfence();
                if (mine) {
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int r = row + e;
                        if (r >= rend) break;
#pragma unroll
                        for (int j = 0; j < K; ++j) {
                            const double* pj = P.part + j * P.ld_part + T.part + 4 * lq + e;
                            double s2 = 0.0;
                            for (int k = 0; k < T.nk; ++k) s2 += __ldcg(pj + (size_t)k * kRB);
                            if (r < nj) P.ynew[j * P.ld_n + c0 + r] = s2;
                            else P.upd[j * P.ld_upd + P.upd_off[J] + (r - nj)] = f[(size_t)r * K + j] + s2;
                        }
                    }
                }
            }
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) atomicAdd(done + J, 1);
    }
}

template <int K, int NT>
__global__ void __launch_bounds__(NT, min_blocks(K, NT))
    sn_backward_kernel(PlanView P, const SnTask* __restrict__ tasks, int ntasks, float* __restrict__ x_old) {
    extern __shared__ double g[];  // [y_J; x_R] x K, m4 x K entries (zero padding rows)
    __shared__ int s_ticket, s_last;
    int* done = P.ctr + 2 + P.nsn;
    int* chunk_ctr = P.ctr + 2 + 2 * P.nsn;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    for (;;) {
        if (tid == 0) s_ticket = atomicAdd(P.ctr + 1, 1);
        __syncthreads();
        const int t = s_ticket;
        if (t >= ntasks) break;
        const SnTask T = tasks[t];
        if (T.front < 0) {
            if (w < T.rows) warp_backward<K>(P, P.bbwd[T.r0 + w], g + (size_t)w * kSmallM * K, lane, x_old, done);
            __syncthreads();
            continue;
        }
        const int J = T.front, nj = P.ncol[J], m = nj + P.nrow[J], c0 = P.col0[J];
        const int m4 = (m + 3) & ~3;
        const int a0 = T.r0, na = T.rows;
        // This task's rows [rlo, rhi): all rows from a0 (the first any of its
        // columns needs, a multiple of 4), or one chunk of them when a tall
        // column block is split (chunks start at multiples of 4; partial sums
        // of the chunks are added in chunk order by the last one to finish).
        const int rlo = T.c0, rhi = T.c0 + T.ncols;
        const int* rows = P.rows + P.rows_off[J];
        const size_t ld = (size_t)m4;
        const float* A = P.fw + P.fw_off[J];
        double s4[K][4];
#pragma unroll
        for (int j = 0; j < K; ++j)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) s4[j][jj] = 0.0;
        const int amin = a0 + w;
        // Row quads wholly below nj (the L_JJ^{-T} y part) need only this
        // front's forward result, so they are summed before waiting on the
        // parent; each lane adds its quads in ascending order.
        const int yhi = min(rhi, nj);
        for (int i = rlo + tid; i < yhi; i += NT)  // from the forward launch
#pragma unroll
            for (int j = 0; j < K; ++j) g[(size_t)i * K + j] = P.ynew[j * P.ld_n + c0 + i];
        if (rhi == m)
            for (int i = m + tid; i < m4; i += NT)  // padding rows
#pragma unroll
                for (int j = 0; j < K; ++j) g[(size_t)i * K + j] = 0.0;
        __syncthreads();
        int r = rlo + 4 * lane;
        auto quad = [&](int rr) {
            double gg[K][4];
#pragma unroll
            for (int j = 0; j < K; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) gg[j][e] = g[(size_t)(rr + e) * K + j];
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                const int a = amin + warps_of(NT) * jj;
                if (a < a0 + na) {
                    const float4 v = ldg4(A + (size_t)a * ld + rr);
#pragma unroll
                    for (int j = 0; j < K; ++j) {
                        s4[j][jj] = fma((double)v.x, gg[j][0], s4[j][jj]);
                        s4[j][jj] = fma((double)v.y, gg[j][1], s4[j][jj]);
                        s4[j][jj] = fma((double)v.z, gg[j][2], s4[j][jj]);
                        s4[j][jj] = fma((double)v.w, gg[j][3], s4[j][jj]);
                    }
                }
            }
        };
        if (amin < a0 + na) {
#pragma unroll 2
            for (; r + 4 <= yhi; r += 128) quad(r);
        }
        if (rhi > nj) {
            // The update rows need the parent's solution.
            if (tid == 0) {
                const int p = P.parent[J];
                if (p >= 0 && !wait_at_least(done + p, P.ntb[p], P.err, P.spin_limit)) atomicExch(P.err, 1);
            }
            __syncthreads();
            for (int i = max(rlo, nj) + tid; i < rhi; i += NT) {
                const int tr = rows[i - nj];
#pragma unroll
                for (int j = 0; j < K; ++j) g[(size_t)i * K + j] = __ldcg(P.xnew + j * P.ld_n + tr);
            }
            __syncthreads();
        }
        // The rest: the update rows, and the quad that straddles nj (its rows
        // past m are the zero padding).
        if (amin < a0 + na) {
#pragma unroll 2
            for (; r < rhi; r += 128) quad(r);
        }
#pragma unroll
        for (int j = 0; j < K; ++j)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s4[j][jj] += __shfl_xor_sync(0xffffffffu, s4[j][jj], o);
        auto write_x = [&](int a, int j, double v) {
            P.xnew[j * P.ld_n + c0 + a] = v;
            x_old[j * P.ld_x + P.perm[c0 + a]] = (float)v;
        };
        if (T.nk == 1) {
            if (lane == 0) {
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    const int a = amin + warps_of(NT) * jj;
                    if (a < a0 + na)
#pragma unroll
                        for (int j = 0; j < K; ++j) write_x(a, j, s4[j][jj]);
                }
            }
        } else {
            // Partial sums of this chunk: column (a - a0) of chunk k.
            if (lane == 0) {
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    const int a = amin + warps_of(NT) * jj;
                    if (a < a0 + na)
#pragma unroll
                        for (int j = 0; j < K; ++j)
                            P.part[j * P.ld_part + T.part + (size_t)T.k * bc_of(NT) + (a - a0)] = s4[j][jj];
                }
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) s_last = (atomicAdd(chunk_ctr + T.chunk, 1) == T.nk - 1);
            __syncthreads();
            if (s_last) {
                __threadfence();
                for (int q = tid; q < na * K; q += NT) {
                    const int c = q / K, j = q - c * K;
                    const double* pj = P.part + j * P.ld_part + T.part + c;
                    double v = 0.0;
                    for (int k = 0; k < T.nk; ++k) v += __ldcg(pj + (size_t)k * bc_of(NT));
                    write_x(a0 + c, j, v);
                }
            }
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) atomicAdd(done + J, 1);
    }
}

size_t forward_smem(int max_m, int k, int nt) {
    return (size_t)std::max((max_m + 4 * nt) * k, warps_of(nt) * kSmallM * k) * sizeof(double);
}
size_t backward_smem(int max_m, int k, int nt) {
    return (size_t)std::max(((max_m + 3) & ~3) * k, warps_of(nt) * kSmallM * k) * sizeof(double);
}

// Right-hand-side counts a launch can take (template instances), and the
// shared memory any of them may use.
constexpr int kBatches[3] = {1, 2, 4};
constexpr size_t kSmemMax = 227 * 1024;

// The dynamic shared-memory limit of each kernel instance only ever grows,
// so a plan built later with smaller fronts cannot invalidate an earlier
// plan's launches.
std::mutex g_smem_mu;
int g_smem_limit[64][6] = {};
template <int K, int NT>
void raise_limit_k(int device, int bytes, int slot) {
    if (bytes <= g_smem_limit[device][slot]) return;
    dev::ck(cudaFuncSetAttribute(sn_forward_kernel<K, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
            "smem attr");
    dev::ck(cudaFuncSetAttribute(sn_backward_kernel<K, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
            "smem attr");
    g_smem_limit[device][slot] = bytes;
}
template <int NT>
void raise_limit_nt(int device, int k, int bytes, int base) {
    if (k == 1) raise_limit_k<1, NT>(device, bytes, base);
    else if (k == 2) raise_limit_k<2, NT>(device, bytes, base + 1);
    else raise_limit_k<4, NT>(device, bytes, base + 2);
}
void raise_smem_limit(int device, int k, int nt, int bytes) {
    std::lock_guard<std::mutex> lock(g_smem_mu);
    if (device < 0 || device >= 64) throw Error(HDD_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    if (nt == kNTInterior) raise_limit_nt<kNTInterior>(device, k, bytes, 0);
    else raise_limit_nt<kNTInterface>(device, k, bytes, 3);
}

template <int K, int NT>
int occupancy_k(size_t smf, size_t smb) {
    int bf = 0, bb = 0;
    dev::ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf, sn_forward_kernel<K, NT>, NT, smf), "occupancy");
    dev::ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bb, sn_backward_kernel<K, NT>, NT, smb), "occupancy");
    return std::max(1, std::min(bf, bb));
}
template <int NT>
int occupancy_nt(int k, size_t smf, size_t smb) {
    return k == 1 ? occupancy_k<1, NT>(smf, smb) : (k == 2 ? occupancy_k<2, NT>(smf, smb) : occupancy_k<4, NT>(smf, smb));
}

}  // namespace

void SolvePlan::build(const std::vector<const SnFactor*>& factors, const std::vector<int>& offsets, cudaStream_t s,
                      int* shared_err) {
    release();
    const bool verbose = std::getenv("HDD_VERBOSE") != nullptr;
    const auto t_start = std::chrono::steady_clock::now();
    auto stamp = [&](const char* what) {
        if (verbose)
            std::fprintf(stderr, "[hdd setup]   plan (%zu factors): %s at %.3f s\n", factors.size(), what,
                         std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count());
    };
    std::vector<int> col0, ncol, nrow, rows, child_ptr{0}, child, relmap, perm, height, depth, parent_g;
    std::vector<long long> rows_off, relmap_off, upd_off, fw_off;
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
    if (nsn == 0) return;
    nt = factors.size() >= 2 ? kNTInterior : kNTInterface;
    const int kWarps = warps_of(nt), kBC = bc_of(nt);
    // Rows per backward task: about 16K coefficients per task, as a forward
    // task's 128 x 128 block (512 rows of 32 columns, 2048 of 8).
    const int kBRows = 16384 / kBC;
    height.assign(nsn, 0);
    depth.assign(nsn, 0);
    for (int g = 0; g < nsn; ++g)
        if (parent_g[g] >= 0) height[parent_g[g]] = std::max(height[parent_g[g]], height[g] + 1);
    for (int g = nsn - 1; g >= 0; --g)
        if (parent_g[g] >= 0) depth[g] = depth[parent_g[g]] + 1;
    long long upd_total = 0, fw_total = 0;
    max_front = 0;
    for (int g = 0; g < nsn; ++g) {
        const SnFactor& F = *factors[where[g].first];
        const int j = where[g].second, off = offsets[where[g].first];
        const int nj = F.ncol[j], nr = (int)F.rows[j].size(), m = nj + nr;
        col0.push_back(off + F.col0[j]);
        ncol.push_back(nj);
        nrow.push_back(nr);
        max_front = std::max(max_front, m);
        rows_off.push_back((long long)rows.size());
        for (int r : F.rows[j]) rows.push_back(off + r);
        upd_off.push_back(upd_total);
        upd_total += nr;
        fw_off.push_back(fw_total);
        fw_total += (long long)((m + 3) & ~3) * nj;
    }
    // Tasks in topological order.
    std::vector<int> order(nsn);
    for (int g = 0; g < nsn; ++g) order[g] = g;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return height[a] < height[b]; });
    std::vector<SnTask> ftasks, btasks;
    std::vector<int> ntf(nsn, 0), ntb(nsn, 0), bfwd, bbwd;
    int nchunk = 0;
    long long part_total = 0;
    // Small fronts of one level go in bundles of kWarps, one warp each.
    auto flush = [](std::vector<SnTask>& tasks, std::vector<int>& list, int& first) {
        if ((int)list.size() == first) return;
        SnTask t;
        t.front = -1; t.r0 = first; t.rows = (int)list.size() - first; t.c0 = 0; t.ncols = 0;
        t.k = 0; t.nk = 1; t.chunk = -1; t.part = 0;
        tasks.push_back(t);
        first = (int)list.size();
    };
    // Bundles pay off where a level has many small fronts (throughput); on
    // narrow levels a whole CTA per front keeps the dependency chain short.
    std::vector<int> small_h(nsn + 1, 0), small_d(nsn + 1, 0);
    for (int g = 0; g < nsn; ++g)
        if (small_front(ncol[g] + nrow[g], ncol[g])) { ++small_h[height[g]]; ++small_d[depth[g]]; }
    int bfirst = 0, blevel = -1;
    for (int g : order) {
        const int nj = ncol[g], m = nj + nrow[g];
        if (height[g] != blevel) { flush(ftasks, bfwd, bfirst); blevel = height[g]; }
        if (small_front(m, nj) && small_h[height[g]] >= kBundleLevel) {
            bfwd.push_back(g);
            ntf[g] = 1;
            if ((int)bfwd.size() - bfirst == kWarps) flush(ftasks, bfwd, bfirst);
            continue;
        }
        for (int r0 = 0; r0 < m; r0 += kRB) {
            const int rowsb = std::min(kRB, m - r0);
            const int cend = std::min(nj, r0 + kRB);
            const int nk = std::max(1, (cend + kCC - 1) / kCC);
            const int chunk = nk > 1 ? nchunk++ : -1;
            const long long part = nk > 1 ? part_total : 0;
            if (nk > 1) part_total += (long long)nk * kRB;
            for (int k = 0; k < nk; ++k) {
                SnTask t;
                t.front = g; t.r0 = r0; t.rows = rowsb; t.c0 = k * kCC;
                t.ncols = std::min(kCC, cend - k * kCC); t.k = k; t.nk = nk; t.chunk = chunk; t.part = part;
                ftasks.push_back(t);
                ++ntf[g];
            }
        }
    }
    flush(ftasks, bfwd, bfirst);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return depth[a] < depth[b]; });
    bfirst = 0;
    blevel = -1;
    for (int g : order) {
        const int nj = ncol[g], m = nj + nrow[g];
        if (depth[g] != blevel) { flush(btasks, bbwd, bfirst); blevel = depth[g]; }
        if (small_front(m, nj) && small_d[depth[g]] >= kBundleLevel) {
            bbwd.push_back(g);
            ntb[g] = 1;
            if ((int)bbwd.size() - bfirst == kWarps) flush(btasks, bbwd, bfirst);
            continue;
        }
        // Column blocks of kBC columns over rows a0 .. m-1; a tall block is
        // split into row chunks of kBRows (c0, ncols: the chunk's rows) whose
        // partial sums the last chunk adds, so that the wide update part of a
        // tall front is read by several CTAs at once.
        for (int a0 = 0; a0 < nj; a0 += kBC) {
            const int span = m - a0;
            const int nk = std::max(1, (span + kBRows - 1) / kBRows);
            const int chunk = nk > 1 ? nchunk++ : -1;
            const long long part = nk > 1 ? part_total : 0;
            if (nk > 1) part_total += (long long)nk * kBC;
            for (int k = 0; k < nk; ++k) {
                SnTask t;
                t.front = g; t.r0 = a0; t.rows = std::min(kBC, nj - a0);
                t.c0 = a0 + k * kBRows; t.ncols = std::min(kBRows, m - t.c0);
                t.k = k; t.nk = nk; t.chunk = chunk; t.part = part;
                btasks.push_back(t);
                ++ntb[g];
            }
        }
    }
    flush(btasks, bbwd, bfirst);
    // Algorithmic bytes: each stored coefficient of L_JJ^{-1} (lower triangle)
    // and of -L_RJ L_JJ^{-1} read once per direction, plus b read and x written.
    double coef = 0;
    for (int g = 0; g < nsn; ++g) coef += 0.5 * ncol[g] * (ncol[g] + 1.0) + (double)nrow[g] * ncol[g];
    fwd_bytes = 4.0 * coef + 8.0 * n;
    bwd_bytes = 4.0 * coef + 8.0 * n;
    n_fwd = (int)ftasks.size();
    n_bwd = (int)btasks.size();
    n_ctr = 2 + 2 * nsn + nchunk;
    stamp("fronts and tasks");
    // Coefficient blocks (FP64 -> FP32, padding rows zero), packed front by
    // front into two pinned staging buffers in turn, each copied to the device
    // while the next is packed: the gigabytes of a level-0 plan then cross at
    // pinned-copy speed and the packing overlaps the copy.
    size_t bytes_fw = 0;
    {
        const long long total = std::max<long long>(fw_total, 4);
        d_fw = nullptr;
        if (cudaMalloc(&d_fw, (size_t)total * sizeof(float)) != cudaSuccess)
            throw Error(HDD_ERR_OUT_OF_MEMORY, "cudaMalloc: supernodal coefficients");
        long long biggest = 4;
        for (int g = 0; g < nsn; ++g) biggest = std::max(biggest, (long long)((ncol[g] + nrow[g] + 3) & ~3) * ncol[g]);
        // Floats per staging buffer: 32 MB (pinning costs about as much as the
        // copy, so the buffers stay small), or the largest front.
        const long long chunk = std::max<long long>(biggest, 8ll << 20);
        float* stage[2] = {nullptr, nullptr};
        cudaEvent_t copied[2] = {nullptr, nullptr};
        auto cleanup = [&]() {
            for (int i = 0; i < 2; ++i) {
                if (copied[i]) { cudaEventSynchronize(copied[i]); cudaEventDestroy(copied[i]); }
                if (stage[i]) cudaFreeHost(stage[i]);
            }
        };
        try {
            for (int i = 0; i < 2; ++i) {
                dev::ck(cudaMallocHost(&stage[i], (size_t)std::min(chunk, total) * sizeof(float)), "pinned staging");
                dev::ck(cudaEventCreateWithFlags(&copied[i], cudaEventDisableTiming), "event");
            }
            int g0 = 0, buf = 0;
            bool used[2] = {false, false};
            while (g0 < nsn) {
                // Fronts g0 .. g1-1 fill this chunk (at least one front).
                int g1 = g0 + 1;
                while (g1 < nsn && fw_off[g1] + (long long)((ncol[g1] + nrow[g1] + 3) & ~3) * ncol[g1] -
                                           fw_off[g0] <= chunk)
                    ++g1;
                const long long base = fw_off[g0];
                const long long end = g1 < nsn ? fw_off[g1] : fw_total;
                if (used[buf]) dev::ck(cudaEventSynchronize(copied[buf]), "staging reuse");
                float* st = stage[buf];
#pragma omp parallel for schedule(dynamic)
                for (int g = g0; g < g1; ++g) {
                    const SnFactor& F = *factors[where[g].first];
                    const BlockVec& W = F.Fw[where[g].second];  // m x nj, col-major
                    const int nj = ncol[g], m = nj + nrow[g], ld = (m + 3) & ~3;
                    float* dst = st + (fw_off[g] - base);
                    for (int c = 0; c < nj; ++c) {
                        for (int r = 0; r < m; ++r) dst[(size_t)c * ld + r] = (float)W[(size_t)c * m + r];
                        for (int r = m; r < ld; ++r) dst[(size_t)c * ld + r] = 0.0f;
                    }
                }
                if (end > base)
                    dev::ck(cudaMemcpyAsync(d_fw + base, st, (size_t)(end - base) * sizeof(float),
                                            cudaMemcpyHostToDevice, s), "coefficient upload");
                dev::ck(cudaEventRecord(copied[buf], s), "event");
                used[buf] = true;
                buf ^= 1;
                g0 = g1;
            }
            if (fw_total < total)  // an empty plan's placeholder
                dev::ck(cudaMemsetAsync(d_fw + fw_total, 0, (size_t)(total - fw_total) * sizeof(float), s), "memset");
        } catch (...) {
            cleanup();
            throw;
        }
        cleanup();
        bytes_fw = (size_t)total * sizeof(float);
    }
    stamp("coefficients packed and uploaded");
    // Children lists and relative maps (child row -> position in parent's front).
    relmap_off.assign(nsn, 0);
    for (int g = 0; g < nsn; ++g) {
        for (int c : kids[g]) child.push_back(c);
        child_ptr.push_back((int)child.size());
    }
    {
        long long total = 0;
        for (int g = 0; g < nsn; ++g) {
            relmap_off[g] = total;
            if (parent_g[g] >= 0) total += nrow[g];
        }
        relmap.resize((size_t)total);
        int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
        for (int g = 0; g < nsn; ++g) {
            const int p = parent_g[g];
            if (p < 0) continue;
            const int pc0 = col0[p], pnj = ncol[p];
            const int* prow = rows.data() + rows_off[p];
            const int pnr = nrow[p];
            const int* crow = rows.data() + rows_off[g];
            int* out = relmap.data() + relmap_off[g];
            for (int kq = 0; kq < nrow[g]; ++kq) {
                const int r = crow[kq];
                int posn = 0;
                if (r >= pc0 && r < pc0 + pnj) posn = r - pc0;
                else {
                    const int* it = std::lower_bound(prow, prow + pnr, r);
                    if (it == prow + pnr || *it != r) bad = 1;
                    else posn = pnj + (int)(it - prow);
                }
                out[kq] = posn;
            }
        }
        if (bad) throw Error(HDD_ERR_INTERNAL, "supernode row not in parent front");
    }
    // Gather lists (the relative maps inverted per parent position, children
    // in their order).
    if (upd_total >= (long long)INT32_MAX) throw Error(HDD_ERR_UNSUPPORTED, "update vectors too large for 32-bit indices");
    std::vector<long long> gp_off(nsn, 0), ge_off(nsn, 0);
    std::vector<int> gptr, gent;
    {
        long long np = 0, ne = 0;
        for (int g = 0; g < nsn; ++g) {
            gp_off[g] = np;
            ge_off[g] = ne;
            np += ncol[g] + nrow[g] + 1;
            for (int c = child_ptr[g]; c < child_ptr[g + 1]; ++c) ne += nrow[child[c]];
        }
        gptr.resize((size_t)np);
        gent.resize((size_t)ne);
#pragma omp parallel for schedule(dynamic, 64)
        for (int g = 0; g < nsn; ++g) {
            const int m = ncol[g] + nrow[g];
            int* cnt = gptr.data() + gp_off[g];  // m + 1 entries
            std::fill(cnt, cnt + m + 1, 0);
            for (int c = child_ptr[g]; c < child_ptr[g + 1]; ++c) {
                const int C = child[c];
                for (int k = 0; k < nrow[C]; ++k) ++cnt[relmap[relmap_off[C] + k] + 1];
            }
            for (int q = 0; q < m; ++q) cnt[q + 1] += cnt[q];
            std::vector<int> fill(cnt, cnt + m);
            int* ent = gent.data() + ge_off[g];
            for (int c = child_ptr[g]; c < child_ptr[g + 1]; ++c) {
                const int C = child[c];
                for (int k = 0; k < nrow[C]; ++k) {
                    const int q = relmap[relmap_off[C] + k];
                    ent[fill[q]++] = (int)(upd_off[C] + k);
                }
            }
        }
    }
    stamp("relative maps and gather lists");
    if (forward_smem(max_front, 1, nt) > 200 * 1024)
        throw Error(HDD_ERR_UNSUPPORTED, "supernodal front too large for shared memory: " + std::to_string(max_front));
    bytes = bytes_fw;
    d_col0 = dev::upload(col0, s, bytes);
    d_ncol = dev::upload(ncol, s, bytes);
    d_nrow = dev::upload(nrow, s, bytes);
    d_parent = dev::upload(parent_g, s, bytes);
    d_rows = dev::upload(rows.empty() ? std::vector<int>{0} : rows, s, bytes);
    d_rows_off = dev::upload(rows_off, s, bytes);
    d_child_ptr = dev::upload(child_ptr, s, bytes);
    d_child = dev::upload(child.empty() ? std::vector<int>{0} : child, s, bytes);
    d_relmap_off = dev::upload(relmap_off, s, bytes);
    d_gp_off = dev::upload(gp_off, s, bytes);
    d_ge_off = dev::upload(ge_off, s, bytes);
    d_gptr = dev::upload(gptr.empty() ? std::vector<int>{0} : gptr, s, bytes);
    d_gent = dev::upload(gent.empty() ? std::vector<int>{0} : gent, s, bytes);
    d_relmap = dev::upload(relmap.empty() ? std::vector<int>{0} : relmap, s, bytes);
    d_upd_off = dev::upload(upd_off, s, bytes);
    d_fw_off = dev::upload(fw_off, s, bytes);
    d_ntf = dev::upload(ntf, s, bytes);
    d_ntb = dev::upload(ntb, s, bytes);
    d_perm = dev::upload(perm, s, bytes);
    d_fwd = dev::upload(ftasks, s, bytes);
    d_bwd = dev::upload(btasks, s, bytes);
    d_bfwd = dev::upload(bfwd.empty() ? std::vector<int>{0} : bfwd, s, bytes);
    d_bbwd = dev::upload(bbwd.empty() ? std::vector<int>{0} : bbwd, s, bytes);
    stamp("uploads issued");
    part_len = std::max<long long>(part_total, 1);
    upd_len = std::max<long long>(upd_total, 1);
    {
        PlanScratch sc;
        alloc_scratch(sc, shared_err, s, bytes);
        d_part = sc.part; d_upd = sc.upd; d_ynew = sc.ynew; d_xnew = sc.xnew; d_ctr = sc.ctr;
        d_err = sc.err;
        own_err = sc.own_err;
    }
    stamp("scratch allocated");
    // A front with a parent, for stall_dependency (the wait of its parent's
    // forward tasks on it can be made unsatisfiable).
    stall_front = -1;
    stall_ntf = 0;
    for (int g = 0; g < nsn; ++g)
        if (parent_g[g] >= 0) { stall_front = g; stall_ntf = ntf[g]; break; }
    ntasks_f = n_fwd;
    ntasks_b = n_bwd;
    // Persistent grid: as many CTAs as fit on the device, per right-hand-side
    // count whose shared memory fits; no more than tasks at launch.
    int dev_id = 0, nsm = 0;
    dev::ck(cudaGetDevice(&dev_id), "cudaGetDevice");
    dev::ck(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev_id), "SM count");
    kmax = 1;
    for (int i = 0; i < 3; ++i) {
        const int k = kBatches[i];
        const size_t smf = forward_smem(max_front, k, nt), smb = backward_smem(max_front, k, nt);
        grids[i] = 0;
        if (std::max(smf, smb) > kSmemMax) break;
        raise_smem_limit(dev_id, k, nt, (int)std::max(smf, smb));
        const int occ = nt == kNTInterior ? occupancy_nt<kNTInterior>(k, smf, smb) : occupancy_nt<kNTInterface>(k, smf, smb);
        grids[i] = std::max(1, nsm * occ);
        kmax = k;
    }
    grid = grids[0];
    stamp("grids sized");
    dev::ck(cudaStreamSynchronize(s), "plan upload");
    stamp("uploaded");
}

void SolvePlan::release() {
    dev::release(d_col0); dev::release(d_ncol); dev::release(d_nrow); dev::release(d_parent);
    dev::release(d_rows); dev::release(d_rows_off); dev::release(d_child_ptr); dev::release(d_child);
    dev::release(d_relmap_off); dev::release(d_relmap);
    dev::release(d_gp_off); dev::release(d_ge_off); dev::release(d_gptr); dev::release(d_gent); dev::release(d_upd_off); dev::release(d_fw_off);
    dev::release(d_ntf); dev::release(d_ntb); dev::release(d_perm);
    dev::release(d_fwd); dev::release(d_bwd); dev::release(d_bfwd); dev::release(d_bbwd); dev::release(d_fw); dev::release(d_part); dev::release(d_upd);
    dev::release(d_ynew); dev::release(d_xnew); dev::release(d_ctr);
    if (own_err) dev::release(d_err);
    d_err = nullptr;
    own_err = false;
    nsn = 0;
    n = 0;
    n_fwd = n_bwd = n_ctr = 0;
}

void SolvePlan::alloc_scratch(PlanScratch& sc, int* shared_err, cudaStream_t s, size_t& b, int nrhs) const {
    if (nrhs != 1 && nrhs != 2 && nrhs != 4) throw Error(HDD_ERR_INVALID_ARGUMENT, "right-hand sides per solve: 1, 2 or 4");
    sc.nrhs = nrhs;
    sc.part = dev::alloc_zero<double>(part_len * nrhs, b, s);
    sc.upd = dev::alloc_zero<double>(upd_len * nrhs, b, s);
    sc.ynew = dev::alloc_zero<double>((long long)std::max(n, 1) * nrhs, b, s);
    sc.xnew = dev::alloc_zero<double>((long long)std::max(n, 1) * nrhs, b, s);
    sc.ctr = dev::alloc_zero<int>(std::max(n_ctr, 1), b, s);
    if (shared_err) {
        sc.err = shared_err;
        sc.own_err = false;
    } else {
        sc.err = dev::alloc_zero<int>(1, b, s);
        sc.own_err = true;
    }
}

void SolvePlan::free_scratch(PlanScratch& sc) {
    dev::release(sc.part); dev::release(sc.upd); dev::release(sc.ynew); dev::release(sc.xnew); dev::release(sc.ctr);
    if (sc.own_err) dev::release(sc.err);
    sc.err = nullptr;
    sc.own_err = false;
}

PlanScratch SolvePlan::primary() const {
    PlanScratch sc;
    sc.part = d_part; sc.upd = d_upd; sc.ynew = d_ynew; sc.xnew = d_xnew; sc.ctr = d_ctr; sc.err = d_err;
    sc.own_err = false;
    sc.nrhs = 1;
    return sc;
}

void SolvePlan::solve(const float* b_old, float* x_old, cudaStream_t s, long long& launches, PhaseHook* hook) const {
    solve(primary(), b_old, x_old, s, launches, hook);
}

template <int K, int NT>
static void launch_pair(const PlanView& P, int g, int n_fwd, int n_bwd, int max_front, const SnTask* fwd,
                        const SnTask* bwd, const float* b_old, float* x_old, cudaStream_t s, PhaseHook* hook,
                        double fwd_bytes, double bwd_bytes) {
    if (hook) hook->begin(kPhaseSnForward);
    sn_forward_kernel<K, NT><<<std::min(g, n_fwd), NT, forward_smem(max_front, K, NT), s>>>(P, fwd, n_fwd, b_old);
    dev::ck(cudaGetLastError(), "sn forward");
    if (hook) hook->end(kPhaseSnForward, fwd_bytes);
    if (hook) hook->begin(kPhaseSnBackward);
    sn_backward_kernel<K, NT><<<std::min(g, n_bwd), NT, backward_smem(max_front, K, NT), s>>>(P, bwd, n_bwd,
                                                                                          x_old);
    dev::ck(cudaGetLastError(), "sn backward");
    if (hook) hook->end(kPhaseSnBackward, bwd_bytes);
}

void SolvePlan::solve(const PlanScratch& sc, const float* b_old, float* x_old, cudaStream_t s, long long& launches,
                      PhaseHook* hook, int nrhs, long long ld_b, long long ld_x) const {
    if (nsn == 0) return;
    if ((nrhs != 1 && nrhs != 2 && nrhs != 4) || nrhs > sc.nrhs || nrhs > kmax)
        throw Error(HDD_ERR_INVALID_ARGUMENT, "right-hand sides per solve: 1, 2 or 4, within the scratch and the plan");
    PlanView P{nsn, max_front, d_col0, d_ncol, d_nrow, d_parent, d_rows, d_rows_off, d_child_ptr, d_child,
               d_relmap_off, d_relmap, d_gp_off, d_ge_off, d_gptr, d_gent, d_upd_off, d_fw_off, d_ntf, d_ntb, d_perm,
               d_bfwd, d_bbwd, d_fw, sc.part, sc.upd,
               sc.ynew, sc.xnew, sc.ctr, sc.err, spin_limit,
               part_len, upd_len, (long long)std::max(n, 1), ld_b, ld_x};
    dev::ck(cudaMemsetAsync(sc.ctr, 0, sizeof(int) * n_ctr, s), "reset counters");
    const int slot = nrhs == 1 ? 0 : (nrhs == 2 ? 1 : 2);
    const int full = grids[slot];
    const int g = sc.grid_div > 1 ? std::max(1, (full + sc.grid_div - 1) / sc.grid_div) : full;
    const double fb = fwd_bytes + 8.0 * n * (nrhs - 1), bb = bwd_bytes + 8.0 * n * (nrhs - 1);
    if (nt == kNTInterior) {
        if (nrhs == 1) launch_pair<1, kNTInterior>(P, g, n_fwd, n_bwd, max_front, d_fwd, d_bwd, b_old, x_old, s, hook, fb, bb);
        else if (nrhs == 2) launch_pair<2, kNTInterior>(P, g, n_fwd, n_bwd, max_front, d_fwd, d_bwd, b_old, x_old, s, hook, fb, bb);
        else launch_pair<4, kNTInterior>(P, g, n_fwd, n_bwd, max_front, d_fwd, d_bwd, b_old, x_old, s, hook, fb, bb);
    } else {
        if (nrhs == 1) launch_pair<1, kNTInterface>(P, g, n_fwd, n_bwd, max_front, d_fwd, d_bwd, b_old, x_old, s, hook, fb, bb);
        else if (nrhs == 2) launch_pair<2, kNTInterface>(P, g, n_fwd, n_bwd, max_front, d_fwd, d_bwd, b_old, x_old, s, hook, fb, bb);
        else launch_pair<4, kNTInterface>(P, g, n_fwd, n_bwd, max_front, d_fwd, d_bwd, b_old, x_old, s, hook, fb, bb);
    }
    launches += 2;
}

void SolvePlan::stall_dependency(bool on, cudaStream_t s) {
    if (stall_front < 0) return;
    const int v = on ? stall_ntf + 1 : stall_ntf;
    dev::ck(cudaMemcpyAsync(d_ntf + stall_front, &v, sizeof(int), cudaMemcpyHostToDevice, s), "stall dependency");
    dev::ck(cudaStreamSynchronize(s), "stall dependency");
}

int SolvePlan::error_flag(cudaStream_t s) const {
    if (!d_err) return 0;
    int h = 0;
    dev::ck(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, s), "read error flag");
    dev::ck(cudaStreamSynchronize(s), "read error flag");
    return h;
}

}  // namespace hdd
