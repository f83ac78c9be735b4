// ORACLE (test infrastructure only) -- a driver that runs PhysBAM's own
// preconditioned conjugate gradient loop, compiled from the reference tree
// where it lies (recipe: oracle/Makefile.ref, output oracle/_ref/libref_cg.so),
// so the tests can pin the oracle's PCG recurrence (stopping rule, rho / beta /
// alpha sequence, projections) to the reference's code.
//
// Reference code run here (nothing of it is copied):
//   PB/Public_Library/PhysBAM_Tools/Krylov_Solvers/CONJUGATE_GRADIENT.cpp:22-67 (Solve),
//   KRYLOV_SOLVER.cpp, KRYLOV_VECTOR_BASE.cpp and KRYLOV_SYSTEM_BASE.cpp:100-106
//   (Precondition: Apply_Preconditioner, then Project and Project_Nullspace),
//   CPU/SPGrid_Domain_Decomposition_Solver/CG_VECTOR.cpp (the vector updates,
//   SPGrid_Gemini_Arithmetic_Helpers.h SPGrid_Copy / SPGrid_Copy2 / SPGrid_Minus_Equal),
//   SPGrid_Gemini_Arithmetic_Helpers.h SPGrid_Laplace (the operator of
//   CG_SYSTEM::Multiply).
// CPU/SPGrid_Domain_Decomposition_Solver/CG_SYSTEM.cpp cannot be compiled
// here (its header pulls in the whole preconditioner, which needs Eigen and
// MKL), so the system class below restates its members: Multiply calls
// SPGrid_Laplace as CG_SYSTEM.cpp:29-44 does; Inner_Product is the FP64 sum
// of FP32 products over the set's blocks in block order (CG_SYSTEM.cpp:50-73);
// Convergence_Norm the max |v| (:78-96); Project zeroes cells that are
// neither Active nor Interface (:101-119); Set_Boundary_Conditions and
// Project_Nullspace do nothing (:124-133); Apply_Preconditioner calls the
// preconditioner it is given (the oracle's, by function pointer) on dense
// copies.  The system is built as
// CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Solver.h:165-194
// builds it: KRYLOV_SYSTEM_BASE(false,false) with use_preconditioner then set.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <SPGrid/Core/SPGrid_Allocator.h>
#include <SPGrid/Core/SPGrid_Set.h>
#include <SPGrid/Tools/SPGrid_Block_Iterator.h>
#include <PhysBAM_Tools/Krylov_Solvers/CONJUGATE_GRADIENT.h>
#include "SPGRID_MULTIGRID_FLAGS.h"

using namespace PhysBAM;
using namespace SPGrid;
#define Packed_OffsetXdim template Packed_OffsetXdim
#define Packed_OffsetYdim template Packed_OffsetYdim
#define Packed_OffsetZdim template Packed_OffsetZdim
#define Packed_Offset template Packed_Offset
// CG_VECTOR.cpp is compiled in this unit, where it lies, so that the
// spellings above apply to the SPGrid helpers it includes.
#include "SPGrid_Domain_Decomposition_Solver/CG_VECTOR.cpp"
#undef Packed_OffsetXdim
#undef Packed_OffsetYdim
#undef Packed_OffsetZdim
#undef Packed_Offset

// CONJUGATE_GRADIENT's diagnostics report through LOG::Stat and
// Test_System through LOG::filecout; the Krylov bases report unimplemented
// members through Not_Implemented and Function_Is_Not_Defined.
namespace PhysBAM {
namespace LOG {
void Stat_Helper(const std::string&, const std::stringstream&, const int) {}
void filecout(const std::string& buffer, const int) { std::cout << buffer; }
}  // namespace LOG
namespace DEBUG_UTILITIES {
void Function_Is_Not_Defined(const char* function, const char* file, unsigned int line, const std::type_info&) {
    std::fprintf(stderr, "reference: function not defined (%s, %s:%u)\n", function, file, line);
    std::abort();
}
void Not_Implemented(const char* function, const char* file, unsigned int line) {
    std::fprintf(stderr, "reference: not implemented (%s, %s:%u)\n", function, file, line);
    std::abort();
}
}  // namespace DEBUG_UTILITIES
}  // namespace PhysBAM

namespace {
typedef SPGRID_DOMAIN_DECOMPOSITION_DATA<float> T_STRUCT;
typedef SPGrid_Allocator<T_STRUCT, 3> Alloc;
typedef Alloc::Array<unsigned>::type Flags;
typedef Alloc::Array<float>::type Data;
typedef SPGrid_Set<Flags> Set;
typedef CG_VECTOR<T_STRUCT, float, 3> Vec;
// Cells of one SPGrid block of a 16-byte struct: 4 x 8 x 8.
const unsigned kPerBlock = 256;

typedef void (*precondition_fn)(void* ctx, const void* rhs, void* result);

class System : public KRYLOV_SYSTEM_BASE<float> {
public:
    Alloc& flags_alloc;
    const Set& set;
    const int* size;
    precondition_fn pre;
    void* ctx;
    std::vector<double>* history;
    mutable std::vector<float> rd, zd;

    System(Alloc& fa, const Set& s, const int* sz, precondition_fn p, void* c, std::vector<double>* h)
        : KRYLOV_SYSTEM_BASE<float>(false, false), flags_alloc(fa), set(s), size(sz), pre(p), ctx(c), history(h) {}

    void Multiply(const KRYLOV_VECTOR_BASE<float>& v, KRYLOV_VECTOR_BASE<float>& result) const {
        SPGrid_Computations::SPGrid_Laplace<T_STRUCT, float, unsigned, 3>(
            Vec::Allocator(result), set.Get_Blocks(), Vec::Allocator(v), flags_alloc, Vec::Cg_Vector(v).field,
            Vec::Cg_Vector(result).field, &T_STRUCT::flags,
            SPGrid_Solver_Cell_Type_Active | SPGrid_Solver_Cell_Type_Interface);
    }
    double Inner_Product(const KRYLOV_VECTOR_BASE<float>& a, const KRYLOV_VECTOR_BASE<float>& b) const {
        Alloc::Array<const float>::type da = Vec::Allocator(a).Get_Const_Array(Vec::Cg_Vector(a).field);
        Alloc::Array<const float>::type db = Vec::Allocator(b).Get_Const_Array(Vec::Cg_Vector(b).field);
        const std::pair<const unsigned long*, unsigned> blocks = set.Get_Blocks();
        double sum = 0;
        for (unsigned bl = 0; bl < blocks.second; ++bl)
            for (unsigned e = 0; e < kPerBlock; ++e) {
                const unsigned long off = blocks.first[bl] + e * sizeof(float);
                sum += da(off) * db(off);
            }
        return sum;
    }
    float Convergence_Norm(const KRYLOV_VECTOR_BASE<float>& v) const {
        Alloc::Array<const float>::type d = Vec::Allocator(v).Get_Const_Array(Vec::Cg_Vector(v).field);
        const std::pair<const unsigned long*, unsigned> blocks = set.Get_Blocks();
        float m = 0;
        for (unsigned bl = 0; bl < blocks.second; ++bl)
            for (unsigned e = 0; e < kPerBlock; ++e) {
                const float a = std::fabs(d(blocks.first[bl] + e * sizeof(float)));
                m = (a > m) ? a : m;
            }
        if (history) history->push_back((double)m);
        return m;
    }
    void Project(KRYLOV_VECTOR_BASE<float>& v) const {
        Data d = Vec::Allocator(v).Get_Array(Vec::Cg_Vector(v).field);
        Alloc::Array<const unsigned>::type f = flags_alloc.Get_Const_Array(&T_STRUCT::flags);
        const std::pair<const unsigned long*, unsigned> blocks = set.Get_Blocks();
        for (unsigned bl = 0; bl < blocks.second; ++bl)
            for (unsigned e = 0; e < kPerBlock; ++e) {
                const unsigned long off = blocks.first[bl] + e * sizeof(float);
                if (!(f(off) & (SPGrid_Solver_Cell_Type_Active | SPGrid_Solver_Cell_Type_Interface))) d(off) = 0.f;
            }
    }
    void Set_Boundary_Conditions(KRYLOV_VECTOR_BASE<float>&) const {}
    void Project_Nullspace(KRYLOV_VECTOR_BASE<float>&) const {}

protected:
    void Apply_Preconditioner(const KRYLOV_VECTOR_BASE<float>& r, KRYLOV_VECTOR_BASE<float>& z) const {
        const size_t n = (size_t)size[0] * size[1] * size[2];
        rd.assign(n, 0.f);
        zd.assign(n, 0.f);
        to_dense(Vec::Allocator(r), Vec::Cg_Vector(r).field, rd.data());
        pre(ctx, rd.data(), zd.data());
        from_dense(Vec::Allocator(z), Vec::Cg_Vector(z).field, zd.data());
    }

public:
    void to_dense(const Alloc& a, float T_STRUCT::* field, float* out) const {
        Alloc::Array<const float>::type d = a.Get_Const_Array(field);
        for (int i = 0; i < size[0]; ++i)
            for (int j = 0; j < size[1]; ++j)
                for (int k = 0; k < size[2]; ++k) {
                    const std_array<unsigned int, 3> c(i, j, k);
                    out[((size_t)i * size[1] + j) * size[2] + k] = set.IsPageActive(c) ? d(c) : 0.f;
                }
    }
    void from_dense(Alloc& a, float T_STRUCT::* field, const float* in) const {
        Data d = a.Get_Array(field);
        for (int i = 0; i < size[0]; ++i)
            for (int j = 0; j < size[1]; ++j)
                for (int k = 0; k < size[2]; ++k) {
                    const std_array<unsigned int, 3> c(i, j, k);
                    if (set.IsPageActive(c)) d(c) = in[((size_t)i * size[1] + j) * size[2] + k];
                }
    }
};
}  // namespace

extern "C" {

// Solves A x = b with PhysBAM's CONJUGATE_GRADIENT<float>::Solve.  flags_in:
// dense x-slowest level-0 cell flags in the reference's bit values (after
// Flaging); pages holding a non-zero flag are the SPGrid set.  b_in / x_out:
// dense arrays (x starts at 0).  tolerance, min_it, max_it: Solve's own
// arguments (the stop test is max|r| <= tolerance).  pre(ctx, r, z): the
// preconditioner on dense arrays.  history[0 .. history_len): the
// convergence norm seen at each iteration.  Returns the iteration count
// (iterations_used), or -1 if Solve reported no convergence.
int refcg_solve(const int size[3], const uint32_t* flags_in, const float* b_in, float* x_out, float tolerance,
                int min_it, int max_it, precondition_fn pre, void* ctx, double* history, int history_len) {
    std_array<int, 3> sz(size[0], size[1], size[2]);
    // As the demo lays them out (SPGrid_Domain_Decomposition_Solver.h:75-82):
    // the first allocator holds the flags and z, r, k; the second x, b, q, s;
    // one set over the pages that hold a non-zero flag.
    Alloc first(sz), second(sz);
    Set set(first.Get_Array(&T_STRUCT::flags));
    for (int i = 0; i < size[0]; ++i)
        for (int j = 0; j < size[1]; ++j)
            for (int k = 0; k < size[2]; ++k) {
                const uint32_t f = flags_in[((size_t)i * size[1] + j) * size[2] + k];
                if (f) set.Mask(std_array<unsigned int, 3>(i, j, k), f);
            }
    set.Refresh_Block_Offsets();
    std::vector<double> hist;
    System sys(first, set, size, pre, ctx, &hist);
    sys.use_preconditioner = true;
    std::vector<float> zero((size_t)size[0] * size[1] * size[2], 0.f);
    sys.from_dense(second, &T_STRUCT::ch0, zero.data());
    sys.from_dense(second, &T_STRUCT::ch1, b_in);
    Vec x(second, set, &T_STRUCT::ch0), b(second, set, &T_STRUCT::ch1), q(second, set, &T_STRUCT::ch2),
        s(second, set, &T_STRUCT::ch3), z(first, set, &T_STRUCT::ch0), r(first, set, &T_STRUCT::ch1),
        k(first, set, &T_STRUCT::ch2);
    CONJUGATE_GRADIENT<float> cg;
    cg.print_residuals = false;
    cg.print_diagnostics = false;
    int used = -1;
    cg.iterations_used = &used;
    const bool converged = cg.Solve(sys, x, b, q, s, r, k, z, tolerance, min_it, max_it);
    sys.to_dense(second, &T_STRUCT::ch0, x_out);
    for (int i = 0; i < history_len && i < (int)hist.size(); ++i) history[i] = hist[i];
    return converged ? used : -1;
}

}  // extern "C"
