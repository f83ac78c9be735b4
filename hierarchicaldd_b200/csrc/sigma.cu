// Device-side sigma (interface Schur complement) V-cycle, sm_100a.
//
// Restates CPU/Interface_Solver/SIGMA_MULTIGRID_SOLVER.cpp:35-47 and
// SIGMA_SMOOTHER.cpp:290-352 on the GPU:
//   Smooth:   u <- (Arr+eps)^{-1} (b + sum_s Air_s^T (Aii_s+eps)^{-1} Air_s u)
//   Residual: r <- b + sum_s Air_s^T (Aii_s+eps)^{-1} Air_s u - Arr u
// * Every SpMV is a row-per-thread CSR walk in a fixed order (the transposed
//   products use an explicitly transposed CSR), so all sums are deterministic
//   and follow the order of the host restatement.
// * The PARDISO solves are supernodal triangular solves over nested-dissection
//   fronts (sn_solve.cu): one persistent launch per solve direction walks the
//   fronts in dependency order.
// * The coarsest level's 200 smoothing steps (SIGMA_MULTIGRID_SOLVER.cpp:43)
//   form a contraction whose fixed point is the Schur complement solve
//   S^{-1} b with S = Arr+eps - sum_s Air_s^T (Aii_s+eps)^{-1} Air_s; setup
//   estimates the contraction factor rho.  When rho^200 <= 1e-7 the steps
//   have converged, and S^{-1} b is computed as the interface block of the
//   solution of K [x_i; x_G] = [0; b] with K = [Aii+eps, -Air; -Air^T, Arr+eps]:
//   one sparse supernodal solve of K instead of 200 dependent smoothing steps.
//   Otherwise the 200 steps run as written.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "dev_util.h"
#include "sigma.h"

namespace hdd {

namespace {

constexpr int kNT = 256;

using dev::ck;

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// y = A x            (mode 0)
// y = b + A x        (mode 1)
// y = b - A x        (mode 2)
// y = y + A x        (mode 3)
// for system blockIdx.y: x, b, y at + blockIdx.y * (xs, bs, ys).
__global__ void __launch_bounds__(kNT) csr_kernel(int rows, const int* __restrict__ ptr, const int* __restrict__ col,
                                                  const float* __restrict__ val, const float* __restrict__ x,
                                                  const float* __restrict__ b, float* __restrict__ y, int mode,
                                                  size_t xs, size_t bs, size_t ys) {
    x += (size_t)blockIdx.y * xs;
    if (b) b += (size_t)blockIdx.y * bs;
    y += (size_t)blockIdx.y * ys;
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

void launch_csr(const DeviceCsr& A, const float* x, const float* b, float* y, int mode, cudaStream_t s,
                long long& launches, int k = 1, size_t xs = 0, size_t bs = 0, size_t ys = 0) {
    if (A.rows == 0) return;
    csr_kernel<<<dim3((A.rows + kNT - 1) / kNT, k), kNT, 0, s>>>(A.rows, A.ptr, A.col, A.val, x, b, y, mode, xs, bs,
                                                                 ys);
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
    ptr = dev::upload(m.ptr, s, bytes);
    col = dev::upload(m.col, s, bytes);
    val = dev::upload(m.val, s, bytes);
}
void DeviceCsr::release() {
    dev::release(ptr);
    dev::release(col);
    dev::release(val);
    rows = cols = nnz = 0;
}

// ---------------------------------------------------------------------------
// SigmaGpu
// ---------------------------------------------------------------------------
void SigmaGpu::release() {
    for (auto& L : lv) {
        L.air.release(); L.airT.release(); L.arr.release(); L.prr.release(); L.prrT.release();
        L.aii.release(); L.arr_solve.release();
        dev::release(L.u); dev::release(L.r); dev::release(L.b); dev::release(L.tmp); dev::release(L.vb); dev::release(L.vx);
    }
    lv.clear();
    bottom.release();
    dev::release(kb);
    dev::release(kx);
    dev::release(d_err);
    device_bytes = 0;
}

void SigmaGpu::setup(const InterfaceHost& ih, int smoothing_iterations, cudaStream_t s, bool force_exact) {
    release();
    const bool verbose = std::getenv("HDD_VERBOSE") != nullptr;
    auto t_start = std::chrono::steady_clock::now();
    auto stamp = [&](const char* what, int l) {
        if (!verbose) return;
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
        std::fprintf(stderr, "[hdd setup] sigma level %d: %s at %.2f s\n", l, what, sec);
    };
    M = ih.M;
    smoothing = smoothing_iterations;
    {
        size_t b0 = 0;
        d_err = dev::alloc_zero<int>(1, b0, s);
        device_bytes += b0;
    }
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
        L.u = dev::alloc_zero<float>(std::max(L.n_iface, 1), bytes, s);
        L.r = dev::alloc_zero<float>(std::max(L.n_iface, 1), bytes, s);
        L.b = dev::alloc_zero<float>(std::max(L.n_iface, 1), bytes, s);
        L.tmp = dev::alloc_zero<float>(std::max(L.n_iface, 1), bytes, s);
        L.vb = dev::alloc_zero<float>(std::max(L.n_int, 1), bytes, s);
        L.vx = dev::alloc_zero<float>(std::max(L.n_int, 1), bytes, s);
        device_bytes += bytes;

        // Factorisations.
        std::vector<SnFactor> aii(ih.n_sub);
        std::vector<std::string> err(ih.n_sub);
#pragma omp parallel for schedule(dynamic)
        for (int sd = 0; sd < ih.n_sub; ++sd) {
            try {
                if (ih.Aii[l][sd].rows == 0) continue;
                aii[sd].analyze(ih.Aii[l][sd], interior_positions(ih, l, sd));
                aii[sd].factor(ih.Aii[l][sd], eps);
                if (l + 1 < M) aii[sd].build_solve_blocks();
            } catch (const std::exception& e) { err[sd] = e.what(); }
        }
        for (auto& e : err)
            if (!e.empty()) throw Error(HDD_ERR_INTERNAL, "subdomain factorisation: " + e);
        stamp("subdomain factors", l);
        SnFactor arrf;
        const std::vector<std::array<int, 3>>* ixyz = interface_positions(ih, l);
        arrf.analyze(ih.Arr[l], ixyz);
        arrf.factor(ih.Arr[l], eps);
        if (l + 1 < M) arrf.build_solve_blocks();
        stamp("interface factor", l);
        if (l + 1 < M) {
            std::vector<const SnFactor*> fs;
            std::vector<int> offs;
            for (int sd = 0; sd < ih.n_sub; ++sd)
                if (aii[sd].n > 0) { fs.push_back(&aii[sd]); offs.push_back(off[sd]); }
            L.aii.build(fs, offs, s, d_err);
            L.arr_solve.build({&arrf}, {0}, s, d_err);
            device_bytes += L.aii.bytes + L.arr_solve.bytes;
            stamp("device plans", l);
        } else {
            // Coarsest level.  The 200 smoothing steps (SIGMA_MULTIGRID_SOLVER.cpp:43)
            // contract towards u = S^{-1} b, S = (Arr+eps) - sum_s Air_s^T (Aii_s+eps)^{-1} Air_s;
            // estimate the contraction factor on the host first.
            const int nb = L.n_iface;
            {
                std::vector<double> xv(nb), yv(nb), tv;
                for (int i = 0; i < nb; ++i) xv[i] = 1.0 + 0.001 * ((i * 7919) % 1000);
                double rho = 0;
                for (int it = 0; it < 60 && nb > 0; ++it) {
                    double nx = 0;
                    for (double v : xv) nx += v * v;
                    nx = std::sqrt(nx);
                    for (double& v : xv) v /= nx;
                    std::fill(yv.begin(), yv.end(), 0.0);
                    for (int sd = 0; sd < ih.n_sub; ++sd) {
                        const CsrF& Air = ih.Air[l][sd];
                        if (Air.rows == 0) continue;
                        tv.assign(Air.rows, 0.0);
                        for (int r = 0; r < Air.rows; ++r)
                            for (int p = Air.ptr[r]; p < Air.ptr[r + 1]; ++p) tv[r] += Air.val[p] * xv[Air.col[p]];
                        aii[sd].solve(tv.data());
                        for (int r = 0; r < Air.rows; ++r)
                            for (int p = Air.ptr[r]; p < Air.ptr[r + 1]; ++p) yv[Air.col[p]] += Air.val[p] * tv[r];
                    }
                    arrf.solve(yv.data());
                    double ny = 0;
                    for (double v : yv) ny += v * v;
                    rho = std::sqrt(ny);
                    xv.swap(yv);
                }
                bottom_contraction = rho;
                bottom_exact = force_exact || std::pow(rho, 200.0) <= 1e-7;
                if (verbose)
                    std::fprintf(stderr, "[hdd setup] coarsest sigma smoother: rho %.4f, %s\n", rho,
                                 bottom_exact ? (force_exact ? "exact Schur solve (requested)" : "exact Schur solve")
                                              : "200 literal smoothing steps");
            }
            if (!bottom_exact) {
                // The 200 steps have not converged to S^{-1} b: run them as the
                // reference does, with this level's solve plans.
                std::vector<std::string> err2(ih.n_sub);
#pragma omp parallel for schedule(dynamic)
                for (int sd = 0; sd < ih.n_sub; ++sd) {
                    try {
                        if (aii[sd].n > 0) aii[sd].build_solve_blocks();
                    } catch (const std::exception& e) { err2[sd] = e.what(); }
                }
                for (auto& e : err2)
                    if (!e.empty()) throw Error(HDD_ERR_INTERNAL, "subdomain solve blocks: " + e);
                arrf.build_solve_blocks();
                std::vector<const SnFactor*> fs;
                std::vector<int> offs;
                for (int sd = 0; sd < ih.n_sub; ++sd)
                    if (aii[sd].n > 0) { fs.push_back(&aii[sd]); offs.push_back(off[sd]); }
                L.aii.build(fs, offs, s, d_err);
                L.arr_solve.build({&arrf}, {0}, s, d_err);
                device_bytes += L.aii.bytes + L.arr_solve.bytes;
                stamp("device plans (coarsest level, literal smoothing)", l);
                continue;
            }
            // K = [Aii (block diagonal) , -Air ; -Air^T , Arr]; factor() adds eps to the diagonal.
            const int ni = L.n_int;
            CsrF K;
            K.rows = K.cols = ni + nb;
            std::vector<std::vector<std::pair<int, float>>> rowsK(ni + nb);
            for (int sd = 0; sd < ih.n_sub; ++sd) {
                const CsrF& A = ih.Aii[l][sd];
                const CsrF& B = ih.Air[l][sd];
                for (int r = 0; r < A.rows; ++r) {
                    for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) rowsK[off[sd] + r].push_back({off[sd] + A.col[p], A.val[p]});
                    for (int p = B.ptr[r]; p < B.ptr[r + 1]; ++p) {
                        rowsK[off[sd] + r].push_back({ni + B.col[p], -B.val[p]});
                        rowsK[ni + B.col[p]].push_back({off[sd] + r, -B.val[p]});
                    }
                }
            }
            const CsrF& Ar = ih.Arr[l];
            for (int r = 0; r < nb; ++r)
                for (int p = Ar.ptr[r]; p < Ar.ptr[r + 1]; ++p) rowsK[ni + r].push_back({ni + Ar.col[p], Ar.val[p]});
            K.ptr.assign(1, 0);
            for (auto& row : rowsK) {
                std::sort(row.begin(), row.end());
                for (auto& e : row) { K.col.push_back(e.first); K.val.push_back(e.second); }
                K.ptr.push_back((int)K.col.size());
            }
            // Positions of K's DOFs: subdomain interiors, then the interface.
            std::vector<std::array<int, 3>> kxyz;
            bool have_xyz = ixyz != nullptr;
            for (int sd = 0; sd < ih.n_sub && have_xyz; ++sd) {
                const auto* px = interior_positions(ih, l, sd);
                if (!px) have_xyz = false;
                else kxyz.insert(kxyz.end(), px->begin(), px->end());
            }
            if (have_xyz) kxyz.insert(kxyz.end(), ixyz->begin(), ixyz->end());
            SnFactor kf;
            kf.analyze(K, have_xyz ? &kxyz : nullptr);
            kf.factor(K, eps);
            kf.build_solve_blocks();
            bottom.build({&kf}, {0}, s, d_err);
            n_bottom = nb;
            n_bottom_int = ni;
            size_t b2 = 0;
            kb = dev::alloc_zero<float>(std::max(ni + nb, 1), b2, s);
            kx = dev::alloc_zero<float>(std::max(ni + nb, 1), b2, s);
            device_bytes += b2 + bottom.bytes;
        }
    }
    ck(cudaStreamSynchronize(s), "sigma setup");
}

SigmaScratch SigmaGpu::primary() const {
    SigmaScratch sc;
    sc.lv.resize(lv.size());
    for (size_t l = 0; l < lv.size(); ++l) {
        const SigmaLevel& L = lv[l];
        SigmaScratch::Level& S = sc.lv[l];
        S.u = L.u; S.r = L.r; S.b = L.b; S.tmp = L.tmp; S.vb = L.vb; S.vx = L.vx;
        S.si = (size_t)std::max(L.n_iface, 1);
        S.sn = (size_t)std::max(L.n_int, 1);
        S.aii = L.aii.primary();
        S.arr = L.arr_solve.primary();
    }
    sc.bottom = bottom.primary();
    sc.kb = kb;
    sc.kx = kx;
    sc.kbs = (size_t)std::max(n_bottom_int + n_bottom, 1);
    sc.err = d_err;
    sc.nrhs = 1;
    return sc;
}

int SigmaGpu::max_rhs() const {
    int k = 4;
    for (const SigmaLevel& L : lv) {
        if (L.aii.nsn > 0) k = std::min(k, L.aii.kmax);
        if (L.arr_solve.nsn > 0) k = std::min(k, L.arr_solve.kmax);
    }
    if (bottom.nsn > 0) k = std::min(k, bottom.kmax);
    return k;
}

void SigmaGpu::alloc_scratch(SigmaScratch& sc, cudaStream_t s, int nrhs) const {
    free_scratch(sc);
    if (nrhs != 1 && nrhs != 2 && nrhs != 4) throw Error(HDD_ERR_INVALID_ARGUMENT, "systems per batch: 1, 2 or 4");
    if (nrhs > max_rhs())
        throw Error(HDD_ERR_UNSUPPORTED, "the interface solver's largest fronts leave no room for that many systems");
    size_t& b = sc.bytes;
    sc.nrhs = nrhs;
    sc.err = dev::alloc_zero<int>(1, b, s);
    sc.lv.resize(lv.size());
    for (size_t l = 0; l < lv.size(); ++l) {
        const SigmaLevel& L = lv[l];
        SigmaScratch::Level& S = sc.lv[l];
        S.si = (size_t)std::max(L.n_iface, 1);
        S.sn = (size_t)std::max(L.n_int, 1);
        S.u = dev::alloc_zero<float>(S.si * nrhs, b, s);
        S.r = dev::alloc_zero<float>(S.si * nrhs, b, s);
        S.b = dev::alloc_zero<float>(S.si * nrhs, b, s);
        S.tmp = dev::alloc_zero<float>(S.si * nrhs, b, s);
        S.vb = dev::alloc_zero<float>(S.sn * nrhs, b, s);
        S.vx = dev::alloc_zero<float>(S.sn * nrhs, b, s);
        if (L.aii.nsn > 0) L.aii.alloc_scratch(S.aii, sc.err, s, b, nrhs);
        if (L.arr_solve.nsn > 0) L.arr_solve.alloc_scratch(S.arr, sc.err, s, b, nrhs);
    }
    if (bottom.nsn > 0) bottom.alloc_scratch(sc.bottom, sc.err, s, b, nrhs);
    sc.kbs = (size_t)std::max(n_bottom_int + n_bottom, 1);
    if (kb) {
        sc.kb = dev::alloc_zero<float>(sc.kbs * nrhs, b, s);
        sc.kx = dev::alloc_zero<float>(sc.kbs * nrhs, b, s);
    }
}

size_t SigmaGpu::scratch_bytes(int nrhs) const {
    size_t t = 4;
    for (const SigmaLevel& L : lv) {
        t += nrhs * (16 * (size_t)std::max(L.n_iface, 1) + 8 * (size_t)std::max(L.n_int, 1));
        t += L.aii.scratch_bytes(nrhs) + L.arr_solve.scratch_bytes(nrhs);
    }
    t += bottom.scratch_bytes(nrhs);
    if (kb) t += 8 * (size_t)std::max(n_bottom_int + n_bottom, 1) * nrhs;
    return t;
}

void SigmaGpu::free_scratch(SigmaScratch& sc) {
    for (SigmaScratch::Level& S : sc.lv) {
        dev::release(S.u); dev::release(S.r); dev::release(S.b); dev::release(S.tmp); dev::release(S.vb);
        dev::release(S.vx);
        SolvePlan::free_scratch(S.aii);
        SolvePlan::free_scratch(S.arr);
    }
    sc.lv.clear();
    SolvePlan::free_scratch(sc.bottom);
    dev::release(sc.kb);
    dev::release(sc.kx);
    dev::release(sc.err);
    sc.bytes = 0;
}

void SigmaGpu::vcycle(cudaStream_t s, long long& launches, PhaseHook* hook) { vcycle(primary(), s, launches, hook); }

void SigmaGpu::vcycle(const SigmaScratch& sc, cudaStream_t s, long long& launches, PhaseHook* hook) {
    const int k = sc.nrhs;
    auto schur_apply = [&](int l, const float* u, float* out_tmp) {
        const SigmaLevel& L = lv[l];
        const SigmaScratch::Level& S = sc.lv[l];
        launch_csr(L.air, u, nullptr, S.vb, 0, s, launches, k, S.si, 0, S.sn);
        L.aii.solve(S.aii, S.vb, S.vx, s, launches, hook, k, (long long)S.sn, (long long)S.sn);
        launch_csr(L.airT, S.vx, S.b, out_tmp, 1, s, launches, k, S.sn, S.si, S.si);  // tmp = b + Air^T vx
    };
    auto smooth = [&](int l) {
        const SigmaScratch::Level& S = sc.lv[l];
        schur_apply(l, S.u, S.tmp);
        lv[l].arr_solve.solve(S.arr, S.tmp, S.u, s, launches, hook, k, (long long)S.si, (long long)S.si);
    };
    for (int l = 0; l + 1 < M; ++l) {
        const SigmaLevel& L = lv[l];
        const SigmaScratch::Level& S = sc.lv[l];
        const SigmaScratch::Level& N = sc.lv[l + 1];
        for (int i = 0; i < smoothing; ++i) smooth(l);
        schur_apply(l, S.u, S.tmp);
        launch_csr(L.arr, S.u, S.tmp, S.r, 2, s, launches, k, S.si, S.si, S.si);  // r = tmp - Arr u
        launch_fill(N.u, N.si * k, 0.0f, s, launches);
        launch_csr(L.prrT, S.r, nullptr, N.b, 0, s, launches, k, S.si, 0, N.si);  // b_{l+1} = Prr^T r
    }
    if (!bottom_exact) {
        for (int i = 0; i < kBottomSmoothing; ++i) smooth(M - 1);
    } else {
        const SigmaScratch::Level& B = sc.lv[M - 1];
        if (n_bottom > 0) {
            // Right-hand sides [0; b], solutions' interface blocks -> u.
            const size_t p = sc.kbs * sizeof(float);
            if (n_bottom_int > 0)
                ck(cudaMemset2DAsync(sc.kb, p, 0, sizeof(float) * n_bottom_int, k, s), "memset kb");
            ck(cudaMemcpy2DAsync(sc.kb + n_bottom_int, p, B.b, B.si * sizeof(float), sizeof(float) * n_bottom, k,
                                 cudaMemcpyDeviceToDevice, s),
               "copy b");
            bottom.solve(sc.bottom, sc.kb, sc.kx, s, launches, hook, k, (long long)sc.kbs, (long long)sc.kbs);
            ck(cudaMemcpy2DAsync(B.u, B.si * sizeof(float), sc.kx + n_bottom_int, p, sizeof(float) * n_bottom, k,
                                 cudaMemcpyDeviceToDevice, s),
               "copy u");
        }
    }
    for (int l = M - 2; l >= 0; --l) {
        const SigmaLevel& L = lv[l];
        const SigmaScratch::Level& S = sc.lv[l];
        const SigmaScratch::Level& N = sc.lv[l + 1];
        launch_csr(L.prr, N.u, nullptr, S.u, 3, s, launches, k, N.si, 0, S.si);  // u += Prr u_{l+1}
        for (int i = 0; i < smoothing; ++i) smooth(l);
    }
}

int SigmaGpu::error_flag(const SigmaScratch& sc, cudaStream_t s) {
    if (!sc.err) return 0;
    int h = 0;
    ck(cudaMemcpyAsync(&h, sc.err, sizeof(int), cudaMemcpyDeviceToHost, s), "read error word");
    ck(cudaStreamSynchronize(s), "read error word");
    return h;
}

void SigmaGpu::clear_error(const SigmaScratch& sc, cudaStream_t s) {
    if (sc.err) ck(cudaMemsetAsync(sc.err, 0, sizeof(int), s), "clear error word");
}

int SigmaGpu::error_flag(cudaStream_t s) const {
    if (!d_err) return 0;
    int h = 0;
    ck(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, s), "read error word");
    ck(cudaStreamSynchronize(s), "read error word");
    return h;
}

void SigmaGpu::clear_error(cudaStream_t s) {
    if (d_err) ck(cudaMemsetAsync(d_err, 0, sizeof(int), s), "clear error word");
}

void SigmaGpu::set_wait_limit(long long polls) {
    for (SigmaLevel& L : lv) { L.aii.spin_limit = polls; L.arr_solve.spin_limit = polls; }
    bottom.spin_limit = polls;
}

void SigmaGpu::stall_dependency(bool on, cudaStream_t s) {
    if (lv.empty()) return;
    SolvePlan& p = lv[0].arr_solve.nsn > 0 ? lv[0].arr_solve : bottom;
    p.stall_dependency(on, s);
}

}  // namespace hdd
