// ORACLE (test infrastructure only) -- a driver that runs the two-level demo's
// own Laplace_ri_Subdomain and Laplace_ir_Subdomain
// (demos/Domain_Decomposition_CPU_Only_Two_Levels/SPGrid_Library/SPGrid_Laplace_Legacy.h:120-178
// and :232-290), compiled from the reference tree (recipe oracle/Makefile.ref,
// output oracle/_ref/libref_two_level.so), to pin the oracle's restatement of
// the two-level couplings bit for bit.  The domain is built as the two-level
// solver builds its V-cycle flags: the divider at sub/2, then Flaging
// (TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Solver.h:129-145).
// PhysBAM's logging and assertion functions are defined by the companion
// driver ref_vcycle.cpp, which is linked with this one.
#include <cstdint>
#include <iostream>

#include <PhysBAM_Tools/Vectors/VECTOR_3D.h>
#include <SPGrid/Core/SPGrid_Allocator.h>
#include <SPGrid/Core/SPGrid_Set.h>
#include <SPGrid/Tools/SPGrid_Block_Iterator.h>
#include <SPGrid_Fluids/Grids/GRID_TOPOLOGY_HELPER.h>
#include "SPGRID_MULTIGRID_FLAGS.h"
#include "SPGRID_MULTIGRID_DATA.h"
using namespace PhysBAM;
using namespace SPGrid;
#define Packed_OffsetXdim template Packed_OffsetXdim
#define Packed_OffsetYdim template Packed_OffsetYdim
#define Packed_OffsetZdim template Packed_OffsetZdim
#define Packed_Offset template Packed_Offset
#include "SPGrid_Laplace_Legacy.h"
#include "SPGrid_Flag_Helper.h"
#include "SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Divider_Helper.h"
#undef Packed_OffsetXdim
#undef Packed_OffsetYdim
#undef Packed_OffsetZdim
#undef Packed_Offset

namespace {
typedef SPGRID_MULTIGRID_DATA<float> T_STRUCT;
typedef SPGrid_Allocator<T_STRUCT, 3> Alloc;
typedef Alloc::Array<unsigned>::type Flags;
typedef SPGrid_Set<Flags> Set;
}  // namespace

extern "C" {

// Dense x-slowest arrays.  With the flags divided at sub/2: ri_out = b_in
// with Laplace_ri_Subdomain(u) at sub applied; ir_out = 0 with
// Laplace_ir_Subdomain(u) at sub applied.  Returns 0.
int reft_subdomain_couplings(const int size[3], const int sub[3], const uint32_t* flags_in, const float* u_in,
                             const float* b_in, float* ri_out, float* ir_out) {
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
                                                     T_INDEX(sub[0] / 2, sub[1] / 2, sub[2] / 2));
    SPGrid_Computations::Flaging<T_STRUCT, 3>(allocator, set.Get_Blocks(), &T_STRUCT::flags, set);
    Alloc::Array<float>::type u = allocator.Get_Array(&T_STRUCT::ch0), ri = allocator.Get_Array(&T_STRUCT::ch1),
                              ir = allocator.Get_Array(&T_STRUCT::ch2);
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                const std_array<unsigned int, 3> c(i, j, k);
                if (!set.IsPageActive(c)) continue;
                const size_t x = ((size_t)i * size[1] + j) * size[2] + k;
                u(c) = u_in[x];
                ri(c) = b_in[x];
                ir(c) = 0.0f;
            }
    std_array<int, 3> s1(sub[0], sub[1], sub[2]);
    SPGrid_Computations::Laplace_ri_Subdomain<T_STRUCT, float, unsigned, 3>(allocator, set.Get_Blocks(), &T_STRUCT::ch0,
                                                                            &T_STRUCT::ch1, &T_STRUCT::flags, s1);
    SPGrid_Computations::Laplace_ir_Subdomain<T_STRUCT, float, unsigned, 3>(allocator, set.Get_Blocks(), &T_STRUCT::ch0,
                                                                            &T_STRUCT::ch2, &T_STRUCT::flags, s1);
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                const std_array<unsigned int, 3> c(i, j, k);
                const size_t x = ((size_t)i * size[1] + j) * size[2] + k;
                const bool on = set.IsPageActive(c);
                ri_out[x] = on ? ri(c) : b_in[x];
                ir_out[x] = on ? ir(c) : 0.0f;
            }
    return 0;
}

}  // extern "C"
