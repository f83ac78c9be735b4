// ORACLE (test infrastructure only).
//
// CPU restatement of the reference's CPU dd_pcg path
// (demos/Domain_Decomposition_CPU_Only, "CPU/" below) used as the checker for the
// CUDA product path.  Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg load this code; the product library never links it.
//
// Parity status: the reference ships no golden vectors for the solver (its only
// fixture is the 2D SPGrid directory under
// demos/SPGrid_Create_Simple_Domain/Create_2D_Domain/output), and the reference
// cannot be built here (Intel icc, MKL PARDISO and Eigen are absent).  The
// oracle's solver arithmetic is therefore "parity unpinned": it is pinned only by
// self-consistency checks (known-answer stencil tests, preconditioner symmetry,
// FP64 exact discrete solves) and by the file-format fixture.
//
// Data layout: every grid level is a dense x-slowest / z-fastest array, which
// is equivalent to the reference's page-sparse SPGrid because every operation is
// masked by flags and unallocated SPGrid pages read as zero.
#pragma once
#include <cstdint>
#include <cstddef>
#include <cstdlib>
#include <cmath>
#include <vector>
#include <array>

namespace oracle {

// Cell flag bits, PB/Common_Libraries/SPGrid_Fluids/Solvers/Domain_Decomposition/
// SPGRID_MULTIGRID_FLAGS.h:13-30 (same values in CPU/SPGrid_Library/SPGRID_MULTIGRID_FLAGS.h:13-28).
enum : uint32_t {
    ACTIVE    = 0x00010000u,
    DIRICHLET = 0x00020000u,
    BOUNDARY  = 0x00040000u,
    INTERFACE = 0x00080000u,
    FACE_MX   = 0x00100000u,   // face bit k = FACE_MX << k, k in (-x,+x,-y,+y,-z,+z)
    FACE_ALL  = 0x03f00000u,
    PARTITION = 0x0000ffffu,
};

struct Dims {
    int n[3] = {0, 0, 0};
    size_t count() const { return (size_t)n[0] * n[1] * n[2]; }
    size_t at(int i, int j, int k) const { return ((size_t)i * n[1] + j) * n[2] + k; }
    bool in(int i, int j, int k) const {
        return i >= 0 && j >= 0 && k >= 0 && i < n[0] && j < n[1] && k < n[2];
    }
};

// Face neighbour offsets in the reference order (-x,+x,-y,+y,-z,+z),
// GRID_TOPOLOGY_HELPER::Face_Neighbor_Offsets as used in CPU/SPGrid_Library/SPGrid_Residual_Legacy.h:45.
static const int FACE_D[6][3] = {{-1,0,0},{1,0,0},{0,-1,0},{0,1,0},{0,0,-1},{0,0,1}};

inline uint32_t flag_at(const Dims& d, const uint32_t* f, int i, int j, int k) {
    return d.in(i, j, k) ? f[d.at(i, j, k)] : 0u;
}
template <class T>
inline T val_at(const Dims& d, const T* v, int i, int j, int k) {
    return d.in(i, j, k) ? v[d.at(i, j, k)] : T(0);
}

// ----------------------------------------------------------------------------
// Flag construction
// ----------------------------------------------------------------------------

// CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Flag_Helper.h:74-106: an
// Active|Interface cell gets face bit k iff its neighbour k is
// Active|Interface|Dirichlet.  Bits are OR-ed in, as in the reference.
void flag_faces(const Dims& d, uint32_t* f);

// CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Flag_Boundary_Helper.h:38-107:
// an Active cell within Manhattan distance <= 3 of a cell whose flag is 0 or
// Interface or Dirichlet (cells outside the grid count as flag 0) is Boundary.
// The reference computes this with three in-place relaxation passes over a
// block plus a 4-cell halo; for distances <= 3 that equals the exact L1
// distance, which is what is restated here.
void flag_boundary(const Dims& d, uint32_t* f);

// CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Divider_Helper.h:31-74.
// Active cells with any index % sub == 0 become Interface; the others get the
// 1-based partition id in the low 16 bits.
void divide_domain(const Dims& d, uint32_t* f, const int sub[3]);
void number_of_subdomains(const int size[3], const int sub[3], int out[3]);

// CPU/SPGrid_Library/SPGrid_V_Cycle_Topology.h:35-67 (Topology_Downsample):
// children (fine c*2-1 .. c*2) visited in SPGrid address order; an unset
// coarse cell takes Active from an Active child and Dirichlet from a
// Dirichlet one (an Interface child leaves it unset); a set one becomes
// Dirichlet on a Dirichlet or Interface child.
void downsample_topology(const Dims& fd, const uint32_t* ff, const Dims& cd, uint32_t* cf);

// ----------------------------------------------------------------------------
// V-cycle stencil operations (CPU/SPGrid_Library/*_Legacy.h)
// ----------------------------------------------------------------------------

// CPU/SPGrid_Library/SPGrid_Residual_Legacy.h:52-61.  r = b - sum_faces(u_c - u_n)
// at Active cells, accumulated as result -= (n - c) in face order.
template <class T>
void residual(const Dims& d, const uint32_t* f, const T* u, T* r, const T* b);

// CPU/SPGrid_Library/SPGrid_Correction_Legacy.h:47-80.  Damped Jacobi update
// u += (omega/face_count) r on Active cells, split by the Boundary bit.
template <class T>
void correction(const Dims& d, const uint32_t* f, T* u, const T* r, bool write_interior,
                bool write_boundary);

// CPU/SPGrid_Library/SPGrid_Restriction_Legacy.h:47-186.
template <class T>
void restriction(const Dims& cd, const uint32_t* cf, T* cb, const Dims& fd, const T* fr);

// CPU/SPGrid_Library/SPGrid_Prolongation_Legacy.h:46-128.
template <class T>
void prolongation(const Dims& fd, const uint32_t* ff, T* fu, const Dims& cd, const T* cu);

// CPU/SPGrid_Library/SPGrid_V_Cycle_Helper.h:156-195 for one level hierarchy.
template <class T>
struct MGLevel {
    Dims d;
    std::vector<uint32_t> flags;
    std::vector<T> u, r, b;
};

template <class T>
void v_cycle(std::vector<MGLevel<T>>& lv, T* u0, T* r0, const T* b0, int interior_itr,
             int boundary_itr);

// CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Gemini_Arithmetic_Helpers.h:241-262
// (SPGrid_Laplace with active_flag = Active|Interface): double accumulation.
template <class T>
void laplace_ai(const Dims& d, const uint32_t* f, const T* u, T* lu);

// CPU/SPGrid_Library/SPGrid_Laplace_Legacy.h:70-117 (Laplace_ri): at Interface
// cells, Lu -= (T)(-sum over active-face Active neighbours of u_n).
template <class T>
void laplace_ri(const Dims& d, const uint32_t* f, const T* u, T* lu);

// Two-level DD (demos/Domain_Decomposition_CPU_Only_Two_Levels, "TWO/"):
// a cell is on a first-level plane when any index is a multiple of sub.
// TWO/SPGrid_Library/SPGrid_Laplace_Legacy.h:120-178 (Laplace_ri_Subdomain):
// at Active|Interface cells on a first-level plane, Lu -= (T)(-sum over
// active-face Active|Interface neighbours off the planes of u_n).
template <class T>
void laplace_ri_subdomain(const Dims& d, const uint32_t* f, const T* u, T* lu, const int sub[3]);

// TWO/SPGrid_Library/SPGrid_Laplace_Legacy.h:232-290 (Laplace_ir_Subdomain):
// at Active|Interface cells off the first-level planes, Lu = -(T)(-sum over
// active-face Active|Interface neighbours on the planes of u_n).
template <class T>
void laplace_ir_subdomain(const Dims& d, const uint32_t* f, const T* u, T* lu, const int sub[3]);

}  // namespace oracle
