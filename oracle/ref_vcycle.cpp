// ORACLE (test infrastructure only) -- a driver that runs the reference's own
// CPU V-cycle code, compiled from the reference tree where it lies (recipe:
// oracle/Makefile.ref, output oracle/_ref/libref_vcycle.so), so the tests can
// pin the oracle's restatement of the level-0 flag pipeline, the V-cycle
// topology and the V-cycle to the reference's code bit for bit.
//
// Reference code run here (nothing of it is copied):
//   CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Divider_Helper.h (Domain_Divider)
//   CPU/SPGrid_Library/SPGrid_Flag_Helper.h (Flaging)
//   CPU/SPGrid_Library/SPGrid_V_Cycle_Topology.h (V_Cycle_Topology: Initialize, Flaging)
//   CPU/SPGrid_Library/SPGrid_V_Cycle_Helper.h (V_Cycle_Helper::v_cycle) and the
//   Residual/Correction/Restriction/Prolongation legacy stencils it calls,
//   CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Gemini_Arithmetic_Helpers.h (SPGrid_Laplace,
//   the operator of CG_SYSTEM::Multiply) and CPU/SPGrid_Library/SPGrid_Laplace_Legacy.h
//   (Laplace_ri, the interface right-hand side of Apply_Preconditioner),
//   CPU/Interface_Solver/STRIDE_GENERATOR.h (Generate_Adaptive_Stride, the graded
//   node spacing of the interface hierarchy),
// in the order CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Solver.h:121-155
// runs them (divider, Flaging, topology).  The SPGrid containers come from
// PB/Common_Libraries/SPGrid.  PhysBAM's logging and debug-reporting functions,
// which those headers call, are defined below as minimal stand-ins.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include <SPGrid/Core/SPGrid_Allocator.h>
#include <SPGrid/Core/SPGrid_Set.h>
#include <SPGrid/Tools/SPGrid_Block_Iterator.h>
#include <SPGrid_Fluids/Grids/GRID_TOPOLOGY_HELPER.h>
#include "SPGRID_MULTIGRID_FLAGS.h"
#include "SPGRID_MULTIGRID_DATA.h"

// V_Cycle_Helper's global_smoothing (not called by v_cycle) names a
// Correction_Global that the reference tree never defines.
namespace SPGrid_Computations {
template <class A, class B, class C, int D> class Correction_Global;
}
using namespace PhysBAM;
using namespace SPGrid;
// The legacy headers call SPGrid_Mask's member templates without the
// "template" disambiguator, which only icc accepts; with SPGrid_Mask.h already
// in, these spell it for them.
#define Packed_OffsetXdim template Packed_OffsetXdim
#define Packed_OffsetYdim template Packed_OffsetYdim
#define Packed_OffsetZdim template Packed_OffsetZdim
#define Packed_Offset template Packed_Offset
#include "SPGrid_V_Cycle_Helper.h"
#include "SPGrid_V_Cycle_Topology.h"
#include "SPGrid_Laplace_Legacy.h"
#include "SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Divider_Helper.h"
#include "SPGrid_Domain_Decomposition_Solver/SPGrid_Gemini_Arithmetic_Helpers.h"
#include "Interface_Solver/STRIDE_GENERATOR.h"
#undef Packed_OffsetXdim
#undef Packed_OffsetYdim
#undef Packed_OffsetZdim
#undef Packed_Offset

// The thread pool the reference's threading helpers use (this driver runs
// them serially, number_of_threads = 0, so it stays null).
PTHREAD_QUEUE* pthread_queue = nullptr;

// Stand-ins for PhysBAM's logging and assertion reporting.
namespace PhysBAM {
namespace LOG {
std::ostream& cout_Helper() { return std::cout; }
std::ostream& cerr_Helper() { return std::cerr; }
SCOPE::~SCOPE() {}
void LOG_CLASS::Push_Scope(const std::string&, const std::string&, const int) {}
}  // namespace LOG
namespace DEBUG_UTILITIES {
void Assertion_Failed(const char* function, const char* file, unsigned int line, const char* condition) {
    std::fprintf(stderr, "reference assertion failed: %s (%s, %s:%u)\n", condition, function, file, line);
    std::abort();
}
void Fatal_Error(const char* function, const char* file, unsigned int line) {
    std::fprintf(stderr, "reference fatal error (%s, %s:%u)\n", function, file, line);
    std::abort();
}
}  // namespace DEBUG_UTILITIES
}  // namespace PhysBAM

namespace {
typedef SPGRID_MULTIGRID_DATA<float> T_STRUCT;
typedef SPGrid_Allocator<T_STRUCT, 3> Alloc;
typedef Alloc::Array<unsigned>::type Flags;
typedef SPGrid_Set<Flags> Set;
}  // namespace

extern "C" {

// Dense x-slowest arrays over size[0..2] cells.  Builds the domain from
// flags_in (cells with a nonzero flag), runs the reference's divider, Flaging
// and V-cycle topology with `levels` levels, writes every level's flags to
// level_flags (level l at offset sum of the earlier levels' cell counts, each
// level (n/2+1) per axis of the previous; cells of inactive pages 0), then one
// v_cycle(u, r, b) from u_in (r starting at 0) and writes u to u_out.
// Returns 0.
int refv_vcycle(const int size[3], const int sub[3], const uint32_t* flags_in, int levels, int interior,
                int boundary, const float* u_in, const float* b_in, uint32_t* level_flags, float* u_out) {
    typedef VECTOR<int, 3> T_INDEX;
    std_array<int, 3> sz(size[0], size[1], size[2]);
    Alloc allocator(sz);
    Set set(allocator.Get_Array(&T_STRUCT::flags));
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                const uint32_t f = flags_in[((size_t)i * size[1] + j) * size[2] + k];
                if (f) set.Mask(std_array<unsigned int, 3>(i, j, k), f);
            }
    set.Refresh_Block_Offsets();
    SPGrid_Computations::Domain_Divider<T_STRUCT, 3>(allocator, set.Get_Blocks(), &T_STRUCT::flags, set,
                                                     T_INDEX(size[0], size[1], size[2]), T_INDEX(),
                                                     T_INDEX(sub[0], sub[1], sub[2]));
    SPGrid_Computations::Flaging<T_STRUCT, 3>(allocator, set.Get_Blocks(), &T_STRUCT::flags, set);
    SPGrid_Computations::V_Cycle_Topology<T_STRUCT, float, 3> topo(allocator, set, sz, levels, &T_STRUCT::flags);
    topo.Initialize(0);
    topo.Flaging(0);
    size_t off = 0;
    for (int l = 0; l < levels; ++l) {
        const std_array<unsigned, 3> n = topo.Get_Size(l);
        Alloc& A = topo.Get_Allocator(l);
        Set& S = topo.Get_Set(l);
        Flags fl = A.Get_Array(&T_STRUCT::flags);
        for (unsigned i = 0; i < n(0); ++i)
            for (unsigned j = 0; j < n(1); ++j)
                for (unsigned k = 0; k < n(2); ++k) {
                    const std_array<unsigned int, 3> c(i, j, k);
                    level_flags[off + ((size_t)i * n(1) + j) * n(2) + k] = S.IsPageActive(c) ? fl(c) : 0u;
                }
        off += (size_t)n(0) * n(1) * n(2);
    }
    Alloc::Array<float>::type u = allocator.Get_Array(&T_STRUCT::ch0), r = allocator.Get_Array(&T_STRUCT::ch1),
                              b = allocator.Get_Array(&T_STRUCT::ch2);
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                const std_array<unsigned int, 3> c(i, j, k);
                if (!set.IsPageActive(c)) continue;
                const size_t x = ((size_t)i * size[1] + j) * size[2] + k;
                u(c) = u_in[x];
                b(c) = b_in[x];
                r(c) = 0.0f;
            }
    SPGrid_Computations::V_Cycle_Helper<T_STRUCT, float, 3>::v_cycle(&T_STRUCT::ch0, &T_STRUCT::ch1, &T_STRUCT::ch2,
                                                                      &T_STRUCT::flags, topo, 0, interior, boundary);
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                const std_array<unsigned int, 3> c(i, j, k);
                const size_t x = ((size_t)i * size[1] + j) * size[2] + k;
                u_out[x] = set.IsPageActive(c) ? u(c) : 0.0f;
            }
    return 0;
}

// The CG operator and the interface gather on the same domain (built as
// refv_vcycle does): lu_out = SPGrid_Laplace(u) at Active|Interface cells
// (CG_SYSTEM.cpp:28-44, before Project; other cells 0), and ri_out =
// b_in with Laplace_ri(u) applied (Lu -= (T)(-sum of Active neighbours) at
// Interface cells; other cells keep b).  Returns 0.
int refv_laplace(const int size[3], const int sub[3], const uint32_t* flags_in, const float* u_in, const float* b_in,
                 float* lu_out, float* ri_out) {
    typedef VECTOR<int, 3> T_INDEX;
    std_array<int, 3> sz(size[0], size[1], size[2]);
    Alloc allocator(sz);
    Set set(allocator.Get_Array(&T_STRUCT::flags));
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                const uint32_t f = flags_in[((size_t)i * size[1] + j) * size[2] + k];
                if (f) set.Mask(std_array<unsigned int, 3>(i, j, k), f);
            }
    set.Refresh_Block_Offsets();
    SPGrid_Computations::Domain_Divider<T_STRUCT, 3>(allocator, set.Get_Blocks(), &T_STRUCT::flags, set,
                                                     T_INDEX(size[0], size[1], size[2]), T_INDEX(),
                                                     T_INDEX(sub[0], sub[1], sub[2]));
    SPGrid_Computations::Flaging<T_STRUCT, 3>(allocator, set.Get_Blocks(), &T_STRUCT::flags, set);
    Alloc::Array<float>::type u = allocator.Get_Array(&T_STRUCT::ch0), lu = allocator.Get_Array(&T_STRUCT::ch1),
                              t = allocator.Get_Array(&T_STRUCT::ch2);
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                const std_array<unsigned int, 3> c(i, j, k);
                if (!set.IsPageActive(c)) continue;
                const size_t x = ((size_t)i * size[1] + j) * size[2] + k;
                u(c) = u_in[x];
                lu(c) = 0.0f;
                t(c) = b_in[x];
            }
    SPGrid_Computations::SPGrid_Laplace<T_STRUCT, float, unsigned, 3>(
        allocator, set.Get_Blocks(), allocator, allocator, &T_STRUCT::ch0, &T_STRUCT::ch1, &T_STRUCT::flags,
        SPGrid_Solver_Cell_Type_Active | SPGrid_Solver_Cell_Type_Interface);
    SPGrid_Computations::Laplace_ri<T_STRUCT, float, unsigned, 3>(allocator, set.Get_Blocks(), &T_STRUCT::ch0,
                                                                  &T_STRUCT::ch2, &T_STRUCT::flags);
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                const std_array<unsigned int, 3> c(i, j, k);
                const size_t x = ((size_t)i * size[1] + j) * size[2] + k;
                const bool on = set.IsPageActive(c);
                lu_out[x] = on ? lu(c) : 0.0f;
                ri_out[x] = on ? t(c) : b_in[x];
            }
    return 0;
}

// STRIDE_GENERATOR<3>::Generate_Adaptive_Stride over the box [lo, hi]: the
// stride of every index per axis, axis 0 first (hi - lo + 1 entries each),
// into q_out.  Returns the adaptation level.
int refv_adaptive_stride(const int lo[3], const int hi[3], int* q_out) {
    typedef VECTOR<int, 3> T_INDEX;
    RANGE<T_INDEX> range(T_INDEX(lo[0], lo[1], lo[2]), T_INDEX(hi[0], hi[1], hi[2]));
    VECTOR<ARRAY<int, VECTOR<int, 1> >, 3> q;
    const int level = STRIDE_GENERATOR<3>::Generate_Adaptive_Stride(range, q);
    size_t o = 0;
    for (int a = 1; a <= 3; ++a)
        for (int i = lo[a - 1]; i <= hi[a - 1]; ++i) q_out[o++] = q(a)(i);
    return level;
}

}  // extern "C"
