// ORACLE (test infrastructure only) -- interface (Schur complement, "sigma")
// system: adaptive subdomain hierarchies, Galerkin assembly of Arr/Aii/Air,
// interface prolongation Prr, sparse Cholesky solves and the sigma V-cycle.
//
// Restates CPU/Interface_Solver/{INTERFACE_MATRIX_GENERATOR.h,GALERKIN_PROCESS.h,
// CELL_PROLONGATION_BAKER.h,STRIDE_GENERATOR.h,PROLONGATION_MATRIX_HELPER.cpp,
// SIGMA_SMOOTHER.cpp,SIGMA_MULTIGRID_SOLVER.cpp,EIGEN_INTERFACE.cpp} and the
// subdomain flag extraction of CPU/SPGrid_Domain_Decomposition_Solver/
// {SPGrid_Subdomain_Splitter.h:123-154,SPGrid_Subdomain_Rasterizer.h}.
//
// Third-party arithmetic that the reference delegates: MKL PARDISO (Intel
// Parallel Studio XE 2017; SPD mtype=2, METIS ordering, single precision) for
// (A + 1e-5 I)^{-1}, and Eigen 3.3.3 sparse storage/SpMV.  Both are absent here;
// the oracle restates the PARDISO solve as an exact sparse Cholesky solve of
// A + 1e-5 I (zero rows get a 1e-5 diagonal, SIGMA_SMOOTHER.cpp:175-237), with
// its own nested-dissection ordering and an up-looking factorisation in FP64.
#pragma once
#include <cstdint>
#include <vector>
#include <array>
#include <unordered_map>

#include "oracle_core.h"

namespace oracle {

template <class T>
struct Csr {
    int rows = 0, cols = 0;
    std::vector<int> ptr, col;
    std::vector<T> val;
    void spmv(const T* x, T* y) const;            // y = A x
    void spmv_t_add(const T* x, T* y) const;      // y += A^T x
};

// Sparse Cholesky of (A + eps I) with zero rows replaced by eps on the diagonal.
struct Cholesky {
    int n = 0;
    std::vector<int> perm;          // new -> old
    std::vector<int> Lp, Li;        // CSC of L, diagonal first in each column
    std::vector<double> Lx;
    // xyz: DOF positions for the fill-reducing ordering (optional).
    template <class T>
    void factor(const Csr<T>& A, double eps, const std::vector<std::array<int, 3>>* xyz = nullptr);
    void solve(double* x) const;    // x <- (A+eps I)^{-1} x
    size_t nnz() const { return Li.size(); }
};

template <class T>
struct InterfaceSystem {
    int M = 0;                         // sigma levels
    int n_sub = 0;
    std::vector<int> n_iface;          // per level
    std::vector<std::array<int, 3>> iface_map;   // level-0 interface DOF -> cell
    std::vector<Csr<T>> Arr;           // [level]
    std::vector<std::vector<Csr<T>>> Aii, Air;   // [level][subdomain]
    std::vector<Csr<T>> Prr;           // [level] (fine rows, coarse cols)
    std::vector<std::vector<int>> n_interior;    // [level][subdomain]
    // DOF positions (finest-level units), used only to order the factorisations.
    std::vector<std::vector<std::array<int, 3>>> iface_xyz;               // [level][dof]
    std::vector<std::vector<std::vector<std::array<int, 3>>>> aii_xyz;    // [level][subdomain][dof]
};

// Build the interface system.  gflags_in are the caller's flags before the
// global Domain_Divider pass (the reference splits before dividing,
// SPGrid_Domain_Decomposition_Solver.h:121-127).
template <class T>
void build_interface_system(const Dims& gd, const uint32_t* gflags_in, const int sub[3], int M,
                            InterfaceSystem<T>& out);

template <class T>
struct SigmaSolver {
    const InterfaceSystem<T>* sys = nullptr;
    int smoothing = 3;
    std::vector<Cholesky> arr;                    // [level]
    std::vector<std::vector<Cholesky>> aii;       // [level][sub]
    std::vector<std::vector<T>> u, r, b;
    void initialize(const InterfaceSystem<T>& s, int smoothing_iterations);
    void smooth(int l, std::vector<T>& u, std::vector<T>& tmp, const std::vector<T>& b) const;
    void compute_residual(int l, const std::vector<T>& u, std::vector<T>& r,
                          const std::vector<T>& b) const;
    void v_cycle();
};

}  // namespace oracle
