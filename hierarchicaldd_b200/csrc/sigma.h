// Interface (Schur complement, "sigma") solver: host assembly of the
// adaptive-hierarchy Galerkin matrices, supernodal Cholesky factorisations and
// the device-side sigma V-cycle.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdint>
#include <string>
#include <vector>
#include <utility>
#include <type_traits>
#include <memory>

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

// Two-level DD: the second-level interface systems of every first-level
// subdomain of sub cells (L.opt.size and L.flags_in are read), stacked into
// one block-diagonal system on boxes of sub/2.
void build_second_level(const DomainLayout& L, const int sub[3], int sigma_levels, InterfaceHost& out);

// Interface dump and reload, the reference's -iomode output / input
// (CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Solver.h:121-161);
// host_interface_io.cpp.  read_interface_dir throws HDD_ERR_IO on a missing or
// malformed file; check_interface throws HDD_ERR_INVALID_ARGUMENT when a
// reloaded system does not fit the domain (levels, subdomain count, sizes,
// interface cells).
void write_interface_dir(const InterfaceHost& ih, const std::string& dir);
void read_interface_dir(const std::string& dir, InterfaceHost& ih);
void check_interface(const DomainLayout& L, int sigma_levels, const InterfaceHost& ih);

// Allocator whose resize leaves new elements uninitialised, for blocks that are
// written in full right after (by several threads, instead of one thread
// zeroing them first).
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind { using other = NoInitAlloc<U>; };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... Args>
    void construct(U* p, Args&&... args) {
        ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
    }
};
using BlockVec = std::vector<double, NoInitAlloc<double>>;

// Supernodal Cholesky of (A + eps I) (zero rows get eps), the stand-in for
// the reference's MKL PARDISO phases 11/22 (SIGMA_SMOOTHER.cpp:115-288).
// Supernodes are the fronts of a nested-dissection separator tree.
struct SnFactor {
    int n = 0;
    std::vector<int> perm;                     // new -> old
    std::vector<int> col0, ncol, parent;       // per supernode, post-order
    std::vector<std::vector<int>> rows;        // below-diagonal rows (new indices), sorted
    std::vector<BlockVec> Ljj, Lrj;            // col-major dense blocks (L_JJ: lower triangle only)
    std::vector<BlockVec> Fw;                  // [Linv; -L_RJ Linv], (nj+nr) x nj col-major
    // Nested-dissection ordering and symbolic factorisation.  With DOF
    // positions the separators are planes cut at the median along the axis
    // that gives the smallest separator; without them, breadth-first level sets.
    void analyze(const CsrF& A, const std::vector<std::array<int, 3>>* xyz = nullptr);
    void factor(const CsrF& A, double eps);
    void build_solve_blocks();
    void solve(double* x) const;               // host reference solve (tests)
};

// Optional per-phase device timing: the caller records events around the
// launches of a phase and accumulates the phase's algorithmic bytes.
struct PhaseHook {
    virtual void begin(int phase) = 0;
    virtual void end(int phase, double bytes) = 0;

protected:
    ~PhaseHook() = default;
};

// Timing phases of the supernodal solve kernels.
constexpr int kPhaseSnForward = 6;
constexpr int kPhaseSnBackward = 7;

// Host reference of a solve plan (sn_plan.cpp): the fronts of a batch of
// independent factorisations with concatenated unknowns and the FP32
// coefficient blocks Fw the device plan stores, solved front by front in
// post-order with FP64 accumulation and FP64 vectors between fronts (the
// device kernels' arithmetic, up to the order of FP64 sums).  Test
// infrastructure for the device plan: CPU tests check it against the FP64
// factorisation, GPU tests check the device solve against it.
struct PlanHost {
    int n = 0, nsn = 0;
    std::vector<int> perm;                        // new -> old (concatenated)
    std::vector<int> col0, ncol, nrow, parent, rows;
    std::vector<long long> rows_off, fw_off;
    std::vector<float> fw;                        // Fw blocks, m x nj col-major, ld round4(m)
    void build(const std::vector<const SnFactor*>& factors, const std::vector<int>& offsets);
    void emulate(const float* b_old, float* x_old) const;
};

// DOF positions (for the fill-reducing ordering) of level l's interface
// system and of subdomain sd's interior system, or null when assembly did not
// record them.
const std::vector<std::array<int, 3>>* interface_positions(const InterfaceHost& ih, int l);
const std::vector<std::array<int, 3>>* interior_positions(const InterfaceHost& ih, int l, int sd);

// Factorisations of one interface solve as the sigma solver builds them
// (A + 1e-5 I, ordering from the positions, explicit solve blocks) and the
// plan over them: kind 0 = Arr of level l, kind 1 = Aii of every subdomain of
// level l with the unknowns concatenated in subdomain order.
void interface_solve_plan(const InterfaceHost& ih, int kind, int l, std::vector<SnFactor>& factors, PlanHost& plan);

// One unit of device work of a supernodal solve, taken by a CTA of the
// persistent solve kernels (sn_solve.cu).  With front >= 0, forward: rows
// [r0, r0+rows) of front `front` times its columns [c0, c0+ncols); when a row
// block is split into nk > 1 column blocks, the partial sums go to `part` and
// the last task of the block (counter `chunk`) adds them in order; backward:
// columns [r0, r0+rows) of the front.  With front < 0, a bundle of `rows`
// small fronts (listed from index r0 of the plan's bundle list), one per warp.
struct SnTask {
    int front, r0, rows, c0, ncols, k, nk, chunk;
    long long part;
};

// The device buffers one supernodal solve writes (split-block partial sums,
// update vectors, forward and backward results, task counters, error word):
// every solve context of a plan has its own, so solves of one plan on
// different streams can run at the same time.
struct PlanScratch {
    double *part = nullptr, *upd = nullptr, *ynew = nullptr, *xnew = nullptr;
    int* ctr = nullptr;
    int* err = nullptr;
    bool own_err = false;
    // The persistent launches use 1/grid_div of the plan's CTAs (rounded up),
    // leaving room on the device for concurrent solves; the results do not
    // depend on it.
    int grid_div = 1;
    int nrhs = 1;  // right-hand sides the buffers hold (1, 2 or 4)
};

// Device plan for a batch of independent supernodal triangular solves.
struct SolvePlan {
    int n = 0;                       // total unknowns (concatenated)
    int nsn = 0;
    int max_front = 0;
    int n_fwd = 0, n_bwd = 0;        // task counts
    int n_ctr = 0;                   // ints in the counter block
    int grid = 0;                    // persistent CTAs per launch (one right-hand side)
    int grids[3] = {0, 0, 0};        // ... for 1, 2 and 4 right-hand sides (0: shared memory too small)
    int kmax = 1;                    // most right-hand sides one launch takes
    int nt = 256;                    // threads per CTA (128 for plans of many factors)
    int ntasks_f = 0, ntasks_b = 0;  // tasks, forward / backward
    double fwd_bytes = 0, bwd_bytes = 0;  // algorithmic bytes of one forward / backward launch
    int *d_col0 = nullptr, *d_ncol = nullptr, *d_nrow = nullptr, *d_parent = nullptr;
    int *d_rows = nullptr; long long *d_rows_off = nullptr;
    int *d_child_ptr = nullptr, *d_child = nullptr;
    long long* d_relmap_off = nullptr; int* d_relmap = nullptr;
    long long *d_gp_off = nullptr, *d_ge_off = nullptr;  // per front: gather-list offsets
    int *d_gptr = nullptr, *d_gent = nullptr;           // gather lists (see sn_solve.cu)
    long long* d_upd_off = nullptr;
    long long* d_fw_off = nullptr;   // per front: float offset of Fw (leading dimension round4(m))
    int *d_ntf = nullptr, *d_ntb = nullptr;  // tasks per front, forward / backward
    int* d_perm = nullptr;           // new -> old (concatenated)
    SnTask *d_fwd = nullptr, *d_bwd = nullptr;
    int *d_bfwd = nullptr, *d_bbwd = nullptr;  // fronts of the forward / backward bundles
    float* d_fw = nullptr;           // Fw blocks of all fronts
    double* d_part = nullptr;        // partial sums of split row blocks
    double* d_upd = nullptr;         // update vectors
    double* d_ynew = nullptr;        // forward result in new order
    double* d_xnew = nullptr;        // backward result in new order
    int* d_ctr = nullptr;            // tickets, completion and chunk counters
    int* d_err = nullptr;            // set when a bounded wait gives up
    bool own_err = false;            // d_err allocated by this plan (else shared)
    long long spin_limit = 1LL << 22;  // polls of a bounded wait before it gives up
    int stall_front = -1, stall_ntf = 0;  // front used by stall_dependency and its task count
    size_t bytes = 0;
    // shared_err: an error word shared with other plans (owned by the caller),
    // or null for a word of the plan's own.
    void build(const std::vector<const SnFactor*>& factors, const std::vector<int>& offsets, cudaStream_t s,
               int* shared_err = nullptr);
    void release();
    long long part_len = 0, upd_len = 0;  // doubles in a scratch's partial-sum and update buffers
    // x_old = (A+eps I)^{-1} b_old (both in the concatenated original order),
    // with the plan's own scratch or a context's.
    void solve(const float* b_old, float* x_old, cudaStream_t s, long long& launches,
               PhaseHook* hook = nullptr) const;
    // With nrhs = 2 or 4 it solves that many systems at once: right-hand side
    // j at b_old + j ld_b, solution at x_old + j ld_x, each coefficient read
    // once for all of them; each solution is bit-identical to its solve alone.
    void solve(const PlanScratch& sc, const float* b_old, float* x_old, cudaStream_t s, long long& launches,
               PhaseHook* hook = nullptr, int nrhs = 1, long long ld_b = 0, long long ld_x = 0) const;
    // Scratch for another solve context (error word shared_err, or its own),
    // for up to nrhs right-hand sides per solve.
    void alloc_scratch(PlanScratch& sc, int* shared_err, cudaStream_t s, size_t& bytes, int nrhs = 1) const;
    static void free_scratch(PlanScratch& sc);
    PlanScratch primary() const;
    // Device bytes alloc_scratch takes (without a shared error word).
    size_t scratch_bytes() const {
        if (nsn == 0) return 0;
        return 8 * (size_t)(part_len + upd_len) + 16 * (size_t)std::max(n, 1) + 4 * (size_t)std::max(n_ctr, 1) + 4;
    }
    size_t scratch_bytes(int nrhs) const {
        if (nsn == 0) return 0;
        return nrhs * (8 * (size_t)(part_len + upd_len) + 16 * (size_t)std::max(n, 1)) +
               4 * (size_t)std::max(n_ctr, 1) + 4;
    }
    int error_flag(cudaStream_t s) const;
    // Test seam: on = raise the forward task count that one front's parent
    // waits for by one, so that wait can never be satisfied and runs into its
    // poll limit; off = restore it.
    void stall_dependency(bool on, cudaStream_t s);
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

// The device buffers one sigma V-cycle writes: every level's vectors, the
// scratch of its solve plans, the coarsest level's [0; b] / solution pair and
// the error word.  The solver's first solve context uses the SigmaGpu's own;
// further contexts (concurrent solves of one resident domain) allocate theirs.
struct SigmaScratch {
    // Level vectors for nrhs systems: system j's interface vectors (u, r, b,
    // tmp) at + j * si, its interior vectors (vb, vx) at + j * sn.
    struct Level {
        float *u = nullptr, *r = nullptr, *b = nullptr, *tmp = nullptr, *vb = nullptr, *vx = nullptr;
        size_t si = 0, sn = 0;
        PlanScratch aii, arr;
    };
    int nrhs = 1;
    size_t kbs = 0;  // stride of the coarsest level's [0; b] / solution pair
    std::vector<Level> lv;
    PlanScratch bottom;
    void set_grid_div(int div) {
        for (Level& L : lv) L.aii.grid_div = L.arr.grid_div = div;
        bottom.grid_div = div;
    }
    float *kb = nullptr, *kx = nullptr;
    int* err = nullptr;
    size_t bytes = 0;
    float* b0() const { return lv.empty() ? nullptr : lv[0].b; }
    float* u0() const { return lv.empty() ? nullptr : lv[0].u; }
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
    // True when 200 bottom smoothing steps have converged to S^{-1} b (rho^200 <=
    // 1e-7), so the coarsest level is one solve of K; false runs the 200 steps.
    bool bottom_exact = true;
    static constexpr int kBottomSmoothing = 200;  // SIGMA_MULTIGRID_SOLVER.cpp:43
    size_t device_bytes = 0;
    // Error word shared by every solve plan of this solver: nonzero once a
    // bounded wait gave up (then later waits return at once).
    int* d_err = nullptr;
    // force_exact: solve the coarsest level exactly even where the 200
    // smoothing steps have not converged (HDD_COARSE_EXACT).
    void setup(const InterfaceHost& ih, int smoothing_iterations, cudaStream_t s, bool force_exact = false);
    void release();
    // u[0] = sigma V-cycle(b[0]) (SIGMA_MULTIGRID_SOLVER.cpp:35-47), u[0] starting at 0,
    // in the given scratch (default: the SigmaGpu's own).
    void vcycle(cudaStream_t s, long long& launches, PhaseHook* hook = nullptr);
    // With sc.nrhs = 2 or 4 it runs that many V-cycles at once (each
    // bit-identical to its V-cycle alone), every supernodal solve taking all
    // right-hand sides in one launch pair.
    void vcycle(const SigmaScratch& sc, cudaStream_t s, long long& launches, PhaseHook* hook = nullptr);
    SigmaScratch primary() const;
    void alloc_scratch(SigmaScratch& sc, cudaStream_t s, int nrhs = 1) const;
    // Most right-hand sides every plan of this hierarchy takes in one launch.
    int max_rhs() const;
    size_t scratch_bytes(int nrhs = 1) const;
    static void free_scratch(SigmaScratch& sc);
    // Nonzero when a bounded wait inside a supernodal solve gave up.
    int error_flag(cudaStream_t s) const;
    void clear_error(cudaStream_t s);
    static int error_flag(const SigmaScratch& sc, cudaStream_t s);
    static void clear_error(const SigmaScratch& sc, cudaStream_t s);
    // Poll limit of every bounded wait (default 1 << 22).
    void set_wait_limit(long long polls);
    // Test seam (SolvePlan::stall_dependency) on the level-0 interface plan.
    void stall_dependency(bool on, cudaStream_t s);
    float* b0() const { return lv.empty() ? nullptr : lv[0].b; }
    float* u0() const { return lv.empty() ? nullptr : lv[0].u; }
    ~SigmaGpu() { release(); }
};

}  // namespace hdd
