// Device-side sigma (interface Schur complement) V-cycle, sm_100a.
//
// Restates CPU/Interface_Solver/SIGMA_MULTIGRID_SOLVER.cpp:70-82 and
// SIGMA_SMOOTHER.cpp:418-478 on the GPU:
//   Smooth:   u <- (Arr+eps)^{-1} (b + sum_s Air_s^T (Aii_s+eps)^{-1} Air_s u)
//   Residual: r <- b + sum_s Air_s^T (Aii_s+eps)^{-1} Air_s u - Arr u
// * Every SpMV is a row-per-thread CSR walk in a fixed order (the transposed
//   products use an explicitly transposed CSR), so all sums are deterministic
//   and follow the order of the host restatement.
// * The PARDISO solves are supernodal triangular solves over nested-dissection
//   fronts: one CTA per front, fronts of one tree level per launch, inverted
//   diagonal blocks so each front is two dense GEMVs.
// * The coarsest level's 200 smoothing steps (SIGMA_MULTIGRID_SOLVER.cpp:78)
//   form a contraction whose fixed point is the Schur complement solve
//   S^{-1} b with S = Arr+eps - sum_s Air_s^T (Aii_s+eps)^{-1} Air_s; setup
//   estimates the contraction factor rho and checks rho^200 < 1e-7, and the
//   device applies the dense S^{-1} in one GEMV.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>

#include "sigma.h"

namespace hdd {

namespace {

constexpr int kNT = 256;

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(HDD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
T* dev_upload(const std::vector<T>& h, cudaStream_t s, size_t& bytes) {
    if (h.empty()) return nullptr;
    T* p = nullptr;
    cudaError_t e = cudaMalloc(&p, h.size() * sizeof(T));
    if (e != cudaSuccess) throw Error(HDD_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    ck(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
    bytes += h.size() * sizeof(T);
    return p;
}
template <class T>
T* dev_alloc(size_t n, size_t& bytes) {
    if (n == 0) return nullptr;
    T* p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) throw Error(HDD_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    ck(cudaMemset(p, 0, n * sizeof(T)), "memset");
    bytes += n * sizeof(T);
    return p;
}
template <class T>
void dev_free(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// y = A x            (mode 0)
// y = b + A x        (mode 1)
// y = b - A x        (mode 2)
// y = y + A x        (mode 3)
__global__ void __launch_bounds__(kNT) csr_kernel(int rows, const int* __restrict__ ptr, const int* __restrict__ col,
                                                  const float* __restrict__ val, const float* __restrict__ x,
                                                  const float* __restrict__ b, float* __restrict__ y, int mode) {
    const int r = blockIdx.x * kNT + threadIdx.x;
    if (r >= rows) return;
    float acc = (mode == 1) ? b[r] : 0.0f;
    for (int p = ptr[r]; p < ptr[r + 1]; ++p) acc = __fadd_rn(acc, __fmul_rn(val[p], x[col[p]]));
    if (mode == 2) acc = __fsub_rn(b[r], acc);
    else if (mode == 3) acc = __fadd_rn(y[r], acc);
    y[r] = acc;
}

__global__ void fill_kernel(float* p, size_t n, float v) {
    for (size_t i = blockIdx.x * (size_t)kNT + threadIdx.x; i < n; i += (size_t)gridDim.x * kNT) p[i] = v;
}

// y = A x for dense row-major A (n x n): one warp per row.
__global__ void __launch_bounds__(kNT) dense_gemv_kernel(int n, const float* __restrict__ A,
                                                         const float* __restrict__ x, float* __restrict__ y) {
    const int warp = (blockIdx.x * kNT + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const float* row = A + (size_t)warp * n;
    float acc = 0.0f;
    for (int j = lane; j < n; j += 32) acc = fmaf(row[j], x[j], acc);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) y[warp] = acc;
}

struct PlanView {
    const int *col0, *ncol, *nrow;
    const long long *linv, *lrj;   // value offsets: linv[j] -> Linv, Linv+nj*nj -> LinvT
    const int* rows;
    const long long* rows_off;
    const int *child_ptr, *child;
    const long long* relmap_off;
    const int* relmap;
    const long long* upd_off;
    const int* perm;
    const float* val;
    float* upd;
    float* ynew;
};

// Forward substitution for the fronts of one tree height (leaves first).
__global__ void __launch_bounds__(kNT) sn_forward_kernel(PlanView P, const int* __restrict__ nodes,
                                                         const float* __restrict__ b_old) {
    extern __shared__ float sh[];
    const int J = nodes[blockIdx.x];
    const int nj = P.ncol[J], nr = P.nrow[J], c0 = P.col0[J];
    float* f = sh;            // nj + nr
    float* y = sh + nj + nr;  // nj
    for (int i = threadIdx.x; i < nj; i += kNT) f[i] = b_old[P.perm[c0 + i]];
    for (int k = threadIdx.x; k < nr; k += kNT) f[nj + k] = 0.0f;
    __syncthreads();
    for (int c = P.child_ptr[J]; c < P.child_ptr[J + 1]; ++c) {
        const int C = P.child[c];
        const int m = P.nrow[C];
        const float* uc = P.upd + P.upd_off[C];
        const int* rm = P.relmap + P.relmap_off[C];
        for (int k = threadIdx.x; k < m; k += kNT) f[rm[k]] = __fadd_rn(f[rm[k]], uc[k]);
        __syncthreads();
    }
    const float* Linv = P.val + P.linv[J];
    for (int i = threadIdx.x; i < nj; i += kNT) {
        float acc = 0.0f;
        for (int a = 0; a < nj; ++a) acc = fmaf(Linv[(size_t)a * nj + i], f[a], acc);
        y[i] = acc;
        P.ynew[c0 + i] = acc;
    }
    __syncthreads();
    if (nr > 0) {
        const float* Lrj = P.val + P.lrj[J];
        float* uo = P.upd + P.upd_off[J];
        for (int k = threadIdx.x; k < nr; k += kNT) {
            float acc = f[nj + k];
            for (int a = 0; a < nj; ++a) acc = fmaf(-Lrj[(size_t)a * nr + k], y[a], acc);
            uo[k] = acc;
        }
    }
}

// Backward substitution for the fronts of one tree depth (roots first).
__global__ void __launch_bounds__(kNT) sn_backward_kernel(PlanView P, const int* __restrict__ nodes,
                                                          float* __restrict__ x_old) {
    extern __shared__ float sh[];
    const int J = nodes[blockIdx.x];
    const int nj = P.ncol[J], nr = P.nrow[J], c0 = P.col0[J];
    float* g = sh;
    const float* Lrj = P.val + P.lrj[J];
    const float* LrjT = Lrj + (size_t)nr * nj;
    const int* rows = P.rows + P.rows_off[J];
    for (int a = threadIdx.x; a < nj; a += kNT) {
        float acc = P.ynew[c0 + a];
        for (int k = 0; k < nr; ++k) acc = fmaf(-LrjT[(size_t)k * nj + a], P.ynew[rows[k]], acc);
        g[a] = acc;
    }
    __syncthreads();
    const float* LinvT = P.val + P.linv[J] + (size_t)nj * nj;
    for (int i = threadIdx.x; i < nj; i += kNT) {
        float acc = 0.0f;
        for (int a = 0; a < nj; ++a) acc = fmaf(LinvT[(size_t)a * nj + i], g[a], acc);
        P.ynew[c0 + i] = acc;
        x_old[P.perm[c0 + i]] = acc;
    }
}

void launch_csr(const DeviceCsr& A, const float* x, const float* b, float* y, int mode, cudaStream_t s,
                long long& launches) {
    if (A.rows == 0) return;
    csr_kernel<<<(A.rows + kNT - 1) / kNT, kNT, 0, s>>>(A.rows, A.ptr, A.col, A.val, x, b, y, mode);
    ck(cudaGetLastError(), "csr_kernel");
    ++launches;
}

void launch_fill(float* p, size_t n, float v, cudaStream_t s, long long& launches) {
    if (!n) return;
    int blocks = (int)std::min<size_t>((n + kNT - 1) / kNT, 148 * 8);
    fill_kernel<<<blocks, kNT, 0, s>>>(p, n, v);
    ck(cudaGetLastError(), "fill_kernel");
    ++launches;
}

CsrF transpose(const CsrF& A) {
    CsrF T;
    T.rows = A.cols;
    T.cols = A.rows;
    T.ptr.assign(T.rows + 1, 0);
    for (int c : A.col) T.ptr[c + 1]++;
    for (int r = 0; r < T.rows; ++r) T.ptr[r + 1] += T.ptr[r];
    T.col.resize(A.col.size());
    T.val.resize(A.val.size());
    std::vector<int> fill(T.ptr.begin(), T.ptr.end() - 1);
    for (int r = 0; r < A.rows; ++r)
        for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) {
            const int q = fill[A.col[p]]++;
            T.col[q] = r;
            T.val[q] = A.val[p];
        }
    return T;
}

}  // namespace

// ---------------------------------------------------------------------------
// DeviceCsr / SolvePlan
// ---------------------------------------------------------------------------
void DeviceCsr::upload(const CsrF& m, cudaStream_t s) {
    release();
    size_t bytes = 0;
    rows = m.rows;
    cols = m.cols;
    nnz = (int)m.col.size();
    ptr = dev_upload(m.ptr, s, bytes);
    col = dev_upload(m.col, s, bytes);
    val = dev_upload(m.val, s, bytes);
}
void DeviceCsr::release() {
    dev_free(ptr);
    dev_free(col);
    dev_free(val);
    rows = cols = nnz = 0;
}

void SolvePlan::build(const std::vector<const SnFactor*>& factors, const std::vector<int>& offsets, cudaStream_t s) {
    release();
    std::vector<int> col0, ncol, nrow, rows, child_ptr{0}, child, relmap, perm, height, depth, parent_g;
    std::vector<long long> linv, lrj, rows_off, relmap_off, upd_off;
    std::vector<float> val;
    long long upd_total = 0;
    n = 0;
    for (size_t f = 0; f < factors.size(); ++f) n = std::max(n, offsets[f] + factors[f]->n);
    perm.assign(n, 0);
    // Global supernode ids: factor by factor in post-order.
    std::vector<int> base(factors.size() + 1, 0);
    for (size_t f = 0; f < factors.size(); ++f) base[f + 1] = base[f] + (int)factors[f]->col0.size();
    nsn = base.back();
    parent_g.assign(nsn, -1);
    std::vector<std::vector<int>> kids(nsn);
    for (size_t f = 0; f < factors.size(); ++f) {
        const SnFactor& F = *factors[f];
        const int off = offsets[f];
        for (int i = 0; i < F.n; ++i) perm[off + i] = off + F.perm[i];
        for (size_t j = 0; j < F.col0.size(); ++j) {
            const int g = base[f] + (int)j;
            if (F.parent[j] >= 0) {
                parent_g[g] = base[f] + F.parent[j];
                kids[parent_g[g]].push_back(g);
            }
        }
    }
    height.assign(nsn, 0);
    depth.assign(nsn, 0);
    // Post-order inside each factor: children precede parents.
    for (int g = 0; g < nsn; ++g)
        if (parent_g[g] >= 0) height[parent_g[g]] = std::max(height[parent_g[g]], height[g] + 1);
    for (int g = nsn - 1; g >= 0; --g)
        if (parent_g[g] >= 0) depth[g] = depth[parent_g[g]] + 1;
    max_front = 0;
    for (size_t f = 0; f < factors.size(); ++f) {
        const SnFactor& F = *factors[f];
        const int off = offsets[f];
        for (size_t j = 0; j < F.col0.size(); ++j) {
            const int nj = F.ncol[j], nr = (int)F.rows[j].size();
            col0.push_back(off + F.col0[j]);
            ncol.push_back(nj);
            nrow.push_back(nr);
            max_front = std::max(max_front, 2 * nj + nr);
            // Linv (col-major) and its transpose, then Lrj (col-major) and its transpose.
            std::vector<double> Li((size_t)nj * nj, 0.0);
            const std::vector<double>& L = F.Ljj[j];
            for (int c = 0; c < nj; ++c) {  // solve L * Li(:,c) = e_c
                Li[(size_t)c * nj + c] = 1.0 / L[(size_t)c * nj + c];
                for (int i = c + 1; i < nj; ++i) {
                    double acc = 0;
                    for (int p = c; p < i; ++p) acc -= L[(size_t)p * nj + i] * Li[(size_t)c * nj + p];
                    Li[(size_t)c * nj + i] = acc / L[(size_t)i * nj + i];
                }
            }
            linv.push_back((long long)val.size());
            for (size_t q = 0; q < Li.size(); ++q) val.push_back((float)Li[q]);
            for (int c = 0; c < nj; ++c)
                for (int i = 0; i < nj; ++i) val.push_back((float)Li[(size_t)i * nj + c]);
            lrj.push_back((long long)val.size());
            const std::vector<double>& R = F.Lrj[j];
            for (size_t q = 0; q < R.size(); ++q) val.push_back((float)R[q]);
            for (int k = 0; k < nr; ++k)
                for (int a = 0; a < nj; ++a) val.push_back((float)R[(size_t)a * nr + k]);
            rows_off.push_back((long long)rows.size());
            for (int r : F.rows[j]) rows.push_back(off + r);
            upd_off.push_back(upd_total);
            upd_total += nr;
        }
    }
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
        for (int k = 0; k < nrow[g]; ++k) {
            const int r = crow[k];
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
    // Schedules.
    int hmax = 0, dmax = 0;
    for (int g = 0; g < nsn; ++g) { hmax = std::max(hmax, height[g]); dmax = std::max(dmax, depth[g]); }
    height_ptr.assign(hmax + 2, 0);
    depth_ptr.assign(dmax + 2, 0);
    for (int g = 0; g < nsn; ++g) { height_ptr[height[g] + 1]++; depth_ptr[depth[g] + 1]++; }
    for (int h = 0; h <= hmax; ++h) height_ptr[h + 1] += height_ptr[h];
    for (int d = 0; d <= dmax; ++d) depth_ptr[d + 1] += depth_ptr[d];
    height_nodes.assign(nsn, 0);
    depth_nodes.assign(nsn, 0);
    {
        std::vector<int> fh(height_ptr.begin(), height_ptr.end() - 1), fd(depth_ptr.begin(), depth_ptr.end() - 1);
        for (int g = 0; g < nsn; ++g) { height_nodes[fh[height[g]]++] = g; depth_nodes[fd[depth[g]]++] = g; }
    }
    if (nsn == 0) return;
    bytes = 0;
    d_col0 = dev_upload(col0, s, bytes);
    d_ncol = dev_upload(ncol, s, bytes);
    d_nrow = dev_upload(nrow, s, bytes);
    d_linv = dev_upload(linv, s, bytes);
    d_lrj = dev_upload(lrj, s, bytes);
    d_rows = dev_upload(rows.empty() ? std::vector<int>{0} : rows, s, bytes);
    d_rows_off = dev_upload(rows_off, s, bytes);
    d_child_ptr = dev_upload(child_ptr, s, bytes);
    d_child = dev_upload(child.empty() ? std::vector<int>{0} : child, s, bytes);
    d_relmap_off = dev_upload(relmap_off, s, bytes);
    d_relmap = dev_upload(relmap.empty() ? std::vector<int>{0} : relmap, s, bytes);
    d_upd_off = dev_upload(upd_off, s, bytes);
    d_perm = dev_upload(perm, s, bytes);
    d_height_nodes = dev_upload(height_nodes, s, bytes);
    d_depth_nodes = dev_upload(depth_nodes, s, bytes);
    d_val = dev_upload(val, s, bytes);
    d_upd = dev_alloc<float>(std::max<long long>(upd_total, 1), bytes);
    d_ynew = dev_alloc<float>(std::max(n, 1), bytes);
}

void SolvePlan::release() {
    dev_free(d_col0); dev_free(d_ncol); dev_free(d_nrow); dev_free(d_linv); dev_free(d_lrj);
    dev_free(d_rows); dev_free(d_rows_off); dev_free(d_child_ptr); dev_free(d_child);
    dev_free(d_relmap_off); dev_free(d_relmap); dev_free(d_upd_off); dev_free(d_perm);
    dev_free(d_height_nodes); dev_free(d_depth_nodes); dev_free(d_val); dev_free(d_upd); dev_free(d_ynew);
    nsn = 0;
    n = 0;
}

void SolvePlan::solve(const float* b_old, float* x_old, cudaStream_t s, long long& launches) const {
    if (nsn == 0) return;
    PlanView P{d_col0, d_ncol, d_nrow, d_linv, d_lrj, d_rows, d_rows_off, d_child_ptr, d_child,
               d_relmap_off, d_relmap, d_upd_off, d_perm, d_val, d_upd, d_ynew};
    const size_t smem = (size_t)max_front * sizeof(float);
    if (smem > 48 * 1024) {
        ck(cudaFuncSetAttribute(sn_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
        ck(cudaFuncSetAttribute(sn_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attr");
    }
    const int H = (int)height_ptr.size() - 1;
    for (int h = 0; h < H; ++h) {
        const int cnt = height_ptr[h + 1] - height_ptr[h];
        if (!cnt) continue;
        sn_forward_kernel<<<cnt, kNT, smem, s>>>(P, d_height_nodes + height_ptr[h], b_old);
        ck(cudaGetLastError(), "sn_forward_kernel");
        ++launches;
    }
    const int D = (int)depth_ptr.size() - 1;
    for (int d = 0; d < D; ++d) {
        const int cnt = depth_ptr[d + 1] - depth_ptr[d];
        if (!cnt) continue;
        sn_backward_kernel<<<cnt, kNT, smem, s>>>(P, d_depth_nodes + depth_ptr[d], x_old);
        ck(cudaGetLastError(), "sn_backward_kernel");
        ++launches;
    }
}

// ---------------------------------------------------------------------------
// SigmaGpu
// ---------------------------------------------------------------------------
void SigmaGpu::release() {
    for (auto& L : lv) {
        L.air.release(); L.airT.release(); L.arr.release(); L.prr.release(); L.prrT.release();
        L.aii.release(); L.arr_solve.release();
        dev_free(L.u); dev_free(L.r); dev_free(L.b); dev_free(L.tmp); dev_free(L.vb); dev_free(L.vx);
    }
    lv.clear();
    dev_free(bottom_inv);
    device_bytes = 0;
}

void SigmaGpu::setup(const InterfaceHost& ih, int smoothing_iterations, cudaStream_t s) {
    release();
    M = ih.M;
    smoothing = smoothing_iterations;
    const double eps = 1e-5;  // SIGMA_SMOOTHER.cpp:176 default epsilon
    lv.resize(M);
    for (int l = 0; l < M; ++l) {
        SigmaLevel& L = lv[l];
        L.n_iface = ih.n_iface[l];
        // Concatenated Air (rows: interior DOFs of subdomain 0, 1, ...).
        std::vector<int> off(ih.n_sub + 1, 0);
        for (int sd = 0; sd < ih.n_sub; ++sd) off[sd + 1] = off[sd] + ih.Air[l][sd].rows;
        L.n_int = off[ih.n_sub];
        CsrF air;
        air.rows = L.n_int;
        air.cols = L.n_iface;
        air.ptr.assign(1, 0);
        for (int sd = 0; sd < ih.n_sub; ++sd) {
            const CsrF& A = ih.Air[l][sd];
            for (int r = 0; r < A.rows; ++r) {
                for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) { air.col.push_back(A.col[p]); air.val.push_back(A.val[p]); }
                air.ptr.push_back((int)air.col.size());
            }
        }
        L.air.upload(air, s);
        L.airT.upload(transpose(air), s);
        L.arr.upload(ih.Arr[l], s);
        if (l + 1 < M) {
            L.prr.upload(ih.Prr[l], s);
            L.prrT.upload(transpose(ih.Prr[l]), s);
        }
        size_t bytes = 0;
        L.u = dev_alloc<float>(std::max(L.n_iface, 1), bytes);
        L.r = dev_alloc<float>(std::max(L.n_iface, 1), bytes);
        L.b = dev_alloc<float>(std::max(L.n_iface, 1), bytes);
        L.tmp = dev_alloc<float>(std::max(L.n_iface, 1), bytes);
        L.vb = dev_alloc<float>(std::max(L.n_int, 1), bytes);
        L.vx = dev_alloc<float>(std::max(L.n_int, 1), bytes);
        device_bytes += bytes;

        // Factorisations.
        std::vector<SnFactor> aii(ih.n_sub);
        std::vector<std::string> err(ih.n_sub);
#pragma omp parallel for schedule(dynamic)
        for (int sd = 0; sd < ih.n_sub; ++sd) {
            try {
                if (ih.Aii[l][sd].rows == 0) continue;
                aii[sd].analyze(ih.Aii[l][sd]);
                aii[sd].factor(ih.Aii[l][sd], eps);
            } catch (const std::exception& e) { err[sd] = e.what(); }
        }
        for (auto& e : err)
            if (!e.empty()) throw Error(HDD_ERR_INTERNAL, "subdomain factorisation: " + e);
        SnFactor arrf;
        arrf.analyze(ih.Arr[l]);
        arrf.factor(ih.Arr[l], eps);
        if (l + 1 < M) {
            std::vector<const SnFactor*> fs;
            std::vector<int> offs;
            for (int sd = 0; sd < ih.n_sub; ++sd)
                if (aii[sd].n > 0) { fs.push_back(&aii[sd]); offs.push_back(off[sd]); }
            L.aii.build(fs, offs, s);
            L.arr_solve.build({&arrf}, {0}, s);
            device_bytes += L.aii.bytes + L.arr_solve.bytes;
        } else {
            // Coarsest level: dense S = (Arr+eps I) - sum_s Air_s^T (Aii_s+eps I)^{-1} Air_s.
            const int nb = L.n_iface;
            n_bottom = nb;
            std::vector<double> S((size_t)nb * nb, 0.0);
            const CsrF& A = ih.Arr[l];
            for (int r = 0; r < nb; ++r) {
                for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) S[(size_t)r * nb + A.col[p]] += A.val[p];
                S[(size_t)r * nb + r] += eps;
            }
            std::vector<std::vector<std::pair<int, int>>> touch(ih.n_sub);
#pragma omp parallel for schedule(dynamic)
            for (int sd = 0; sd < ih.n_sub; ++sd) {
                const CsrF& Air = ih.Air[l][sd];
                if (Air.rows == 0) continue;
                std::vector<int> cols(Air.col.begin(), Air.col.end());
                std::sort(cols.begin(), cols.end());
                cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
                const int nc = (int)cols.size(), ni = Air.rows;
                // G = (Aii+eps)^{-1} Air(:, cols), column by column.
                std::vector<double> G((size_t)nc * ni, 0.0);
                for (int c = 0; c < nc; ++c) {
                    double* g = &G[(size_t)c * ni];
                    for (int r = 0; r < ni; ++r)
                        for (int p = Air.ptr[r]; p < Air.ptr[r + 1]; ++p)
                            if (Air.col[p] == cols[c]) g[r] += Air.val[p];
                    aii[sd].solve(g);
                }
                // K = Air(:,cols)^T G, subtracted from S (serialised per subdomain).
                std::vector<double> K((size_t)nc * nc, 0.0);
                for (int r = 0; r < ni; ++r)
                    for (int p = Air.ptr[r]; p < Air.ptr[r + 1]; ++p) {
                        const int ci = (int)(std::lower_bound(cols.begin(), cols.end(), Air.col[p]) - cols.begin());
                        for (int c = 0; c < nc; ++c) K[(size_t)ci * nc + c] += (double)Air.val[p] * G[(size_t)c * ni + r];
                    }
#pragma omp critical
                for (int a = 0; a < nc; ++a)
                    for (int c = 0; c < nc; ++c) S[(size_t)cols[a] * nb + cols[c]] -= K[(size_t)a * nc + c];
            }
            // Contraction factor of the bottom smoother M = (Arr+eps)^{-1}(Arr+eps - S),
            // by power iteration.
            {
                std::vector<double> x(nb), y(nb);
                for (int i = 0; i < nb; ++i) x[i] = 1.0 + 0.001 * ((i * 7919) % 1000);
                double rho = 0;
                for (int it = 0; it < 60 && nb > 0; ++it) {
                    double nx = 0;
                    for (double v : x) nx += v * v;
                    nx = std::sqrt(nx);
                    for (double& v : x) v /= nx;
                    // y = (Arr+eps)x - S x
                    std::fill(y.begin(), y.end(), 0.0);
                    for (int r = 0; r < nb; ++r) {
                        double acc = eps * x[r];
                        for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) acc += A.val[p] * x[A.col[p]];
                        const double* Sr = &S[(size_t)r * nb];
                        for (int c = 0; c < nb; ++c) acc -= Sr[c] * x[c];
                        y[r] = acc;
                    }
                    arrf.solve(y.data());
                    double ny = 0;
                    for (double v : y) ny += v * v;
                    rho = std::sqrt(ny);
                    x.swap(y);
                }
                bottom_contraction = rho;
                if (std::pow(rho, 200.0) > 1e-7)
                    throw Error(HDD_ERR_UNSUPPORTED,
                                "coarsest sigma smoother does not converge in 200 steps (rho=" + std::to_string(rho) + ")");
            }
            dense_spd_inverse(S, nb);
            std::vector<float> Sf(S.begin(), S.end());
            size_t b2 = 0;
            bottom_inv = dev_upload(Sf, s, b2);
            device_bytes += b2;
        }
    }
    ck(cudaStreamSynchronize(s), "sigma setup");
}

void SigmaGpu::vcycle(cudaStream_t s, long long& launches) {
    auto schur_apply = [&](int l, const float* u, float* out_tmp) {
        SigmaLevel& L = lv[l];
        launch_csr(L.air, u, nullptr, L.vb, 0, s, launches);
        L.aii.solve(L.vb, L.vx, s, launches);
        launch_csr(L.airT, L.vx, L.b, out_tmp, 1, s, launches);  // tmp = b + Air^T vx
    };
    auto smooth = [&](int l) {
        SigmaLevel& L = lv[l];
        schur_apply(l, L.u, L.tmp);
        L.arr_solve.solve(L.tmp, L.u, s, launches);
    };
    for (int l = 0; l + 1 < M; ++l) {
        SigmaLevel& L = lv[l];
        for (int i = 0; i < smoothing; ++i) smooth(l);
        schur_apply(l, L.u, L.tmp);
        launch_csr(L.arr, L.u, L.tmp, L.r, 2, s, launches);           // r = tmp - Arr u
        launch_fill(lv[l + 1].u, lv[l + 1].n_iface, 0.0f, s, launches);
        launch_csr(L.prrT, L.r, nullptr, lv[l + 1].b, 0, s, launches); // b_{l+1} = Prr^T r
    }
    {
        SigmaLevel& B = lv[M - 1];
        if (n_bottom > 0) {
            const int blocks = (int)(((size_t)n_bottom * 32 + kNT - 1) / kNT);
            dense_gemv_kernel<<<blocks, kNT, 0, s>>>(n_bottom, bottom_inv, B.b, B.u);
            ck(cudaGetLastError(), "dense_gemv_kernel");
            ++launches;
        }
    }
    for (int l = M - 2; l >= 0; --l) {
        SigmaLevel& L = lv[l];
        launch_csr(L.prr, lv[l + 1].u, nullptr, L.u, 3, s, launches);  // u += Prr u_{l+1}
        for (int i = 0; i < smoothing; ++i) smooth(l);
    }
}

}  // namespace hdd
