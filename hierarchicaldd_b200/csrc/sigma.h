// Interface (Schur complement, "sigma") solver: host assembly of the
// adaptive-hierarchy Galerkin matrices, supernodal Cholesky factorisations and
// the device-side sigma V-cycle.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <vector>

#include "hdd_common.h"

namespace hdd {

struct DomainLayout;

struct CsrF {
    int rows = 0, cols = 0;
    std::vector<int> ptr, col;
    std::vector<float> val;
};

// Interface system in the reference's DOF numbering
// (CPU/Interface_Solver/INTERFACE_MATRIX_GENERATOR.h:130-735).
struct InterfaceHost {
    int M = 0, n_sub = 0;
    std::vector<int> n_iface;                       // [level]
    std::vector<std::array<int, 3>> iface_map;      // level-0 interface DOF -> cell
    std::vector<CsrF> Arr, Prr;                     // [level]
    std::vector<std::vector<CsrF>> Aii, Air;        // [level][subdomain]
    // DOF positions in finest-level grid units (used only for the fill-reducing
    // ordering of the factorisations).
    std::vector<std::vector<std::array<int, 3>>> iface_xyz;             // [level][dof]
    std::vector<std::vector<std::vector<std::array<int, 3>>>> aii_xyz;  // [level][subdomain][dof]
};

// Builds the interface system from the caller's flags (before the global
// Domain_Divider pass, as the reference splits first), in parallel over
// subdomains.
void build_interface(const DomainLayout& L, int sigma_levels, InterfaceHost& out);

// Supernodal Cholesky of (A + eps I) (zero rows get eps), the stand-in for
// the reference's MKL PARDISO phases 11/22 (SIGMA_SMOOTHER.cpp:241-414).
// Supernodes are the fronts of a nested-dissection separator tree.
struct SnFactor {
    int n = 0;
    std::vector<int> perm;                     // new -> old
    std::vector<int> col0, ncol, parent;       // per supernode, post-order
    std::vector<std::vector<int>> rows;        // below-diagonal rows (new indices), sorted
    std::vector<std::vector<double>> Ljj, Lrj; // col-major dense blocks
    std::vector<std::vector<double>> Fw;       // [Linv; -L_RJ Linv], (nj+nr) x nj col-major
    // Nested-dissection ordering and symbolic factorisation.  With DOF
    // positions the separators are planes cut at the median along the axis
    // that gives the smallest separator; without them, breadth-first level sets.
    void analyze(const CsrF& A, const std::vector<std::array<int, 3>>* xyz = nullptr);
    void factor(const CsrF& A, double eps);
    void build_solve_blocks();
    void solve(double* x) const;               // host reference solve (tests)
};

// One unit of device work of a supernodal solve: rows [rb, re) of one front,
// streamed as a contiguous block of ncols columns x kTaskRows rows.
struct SnTask {
    int front, rb, re, kind;  // kind 0: forward L^{-1} rows, 1: forward update rows, 2: backward
    int col_base, ncols, pad0, pad1;
    long long blk;            // float offset of the task's block
};

// One warp task of a small front: its Fw block (m x nj, column-major, leading
// dimension m) at float offset `off`; `part` selects the rows (forward) or
// columns (backward) the warp computes.
struct SnFront {
    int front, m, nj, part;
    long long off;
};

// Device plan for a batch of independent supernodal triangular solves
// (sn_solve.cu).
struct SolvePlan {
    int n = 0;                       // total unknowns (concatenated)
    int nsn = 0;
    int max_front = 0;
    std::vector<int> fwd_ptr, bwd_ptr;           // task ranges per tree level
    std::vector<int> sfwd_ptr, sbwd_ptr;         // warp-front ranges per tree level
    SnFront *d_sfwd = nullptr, *d_sbwd = nullptr;
    float* d_fw = nullptr;                       // warp-front coefficient blocks
    int *d_col0 = nullptr, *d_ncol = nullptr, *d_nrow = nullptr;
    int *d_rows = nullptr; long long *d_rows_off = nullptr;
    int *d_child_ptr = nullptr, *d_child = nullptr;
    long long* d_relmap_off = nullptr; int* d_relmap = nullptr;
    long long* d_upd_off = nullptr;
    int* d_perm = nullptr;           // new -> old (concatenated)
    SnTask *d_fwd = nullptr, *d_bwd = nullptr;
    float* d_val = nullptr;          // task blocks
    float* d_upd = nullptr;          // update vectors
    float* d_ynew = nullptr;         // forward result in new order
    float* d_xnew = nullptr;         // backward result in new order
    int* d_err = nullptr;            // set when a bounded wait gives up
    size_t bytes = 0;
    void build(const std::vector<const SnFactor*>& factors, const std::vector<int>& offsets, cudaStream_t s);
    void release();
    // x_old = (A+eps I)^{-1} b_old (both in the concatenated original order).
    void solve(const float* b_old, float* x_old, cudaStream_t s, long long& launches) const;
    int error_flag(cudaStream_t s) const;
    ~SolvePlan() { release(); }
};

struct DeviceCsr {
    int rows = 0, cols = 0, nnz = 0;
    int *ptr = nullptr, *col = nullptr;
    float* val = nullptr;
    void upload(const CsrF& m, cudaStream_t s);
    void release();
};

struct SigmaLevel {
    int n_iface = 0, n_int = 0;
    DeviceCsr air;      // concatenated Air (rows: interior DOFs of all subdomains)
    DeviceCsr airT;     // its transpose (rows: interface DOFs)
    DeviceCsr arr;      // Arr (for residuals)
    DeviceCsr prr;      // Prr (fine x coarse)
    DeviceCsr prrT;     // Prr^T
    SolvePlan aii, arr_solve;
    float *u = nullptr, *r = nullptr, *b = nullptr, *tmp = nullptr, *vb = nullptr, *vx = nullptr;
};

struct SigmaGpu {
    int M = 0, smoothing = 3;
    std::vector<SigmaLevel> lv;
    // Coarsest level: sparse Cholesky of K = [Aii+eps, -Air; -Air^T, Arr+eps]
    // (all subdomain interiors first, then the interface), whose interface block
    // solves the Schur complement S exactly.
    SolvePlan bottom;
    float *kb = nullptr, *kx = nullptr;
    int n_bottom = 0, n_bottom_int = 0;
    double bottom_contraction = 0;   // estimated spectral radius of the bottom smoother
    size_t device_bytes = 0;
    void setup(const InterfaceHost& ih, int smoothing_iterations, cudaStream_t s);
    void release();
    // u[0] = sigma V-cycle(b[0]) (SIGMA_MULTIGRID_SOLVER.cpp:70-82), u[0] starting at 0.
    void vcycle(cudaStream_t s, long long& launches);
    // Nonzero when a bounded wait inside a supernodal solve gave up.
    int error_flag(cudaStream_t s) const;
    float* b0() const { return lv.empty() ? nullptr : lv[0].b; }
    float* u0() const { return lv.empty() ? nullptr : lv[0].u; }
    ~SigmaGpu() { release(); }
};

}  // namespace hdd
