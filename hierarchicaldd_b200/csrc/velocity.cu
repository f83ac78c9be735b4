// Velocity -> divergence right-hand side: the reference Test_Bench's
// "velocity" mode (GPU/Test_Bench_3D/main.cpp:317-324) on a uniform,
// single-level grid, followed by its flag conversion (Convert,
// GPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Convertor.h:213-236).
//
// Per cell (one thread): Divergence_Helper's 3D Run_Index_Range
// (PB/Common_Libraries/SPGrid_Fluids/Projection/Divergence_Helper.cpp:150-240)
// at Interior|Ghost cells: a float result starting at 0 takes, for x, y, z in
// turn, -= scale * u_face(cell) when the cell's face is valid and += scale *
// u_face(cell + e) when the neighbour's is, each step in double and rounded
// to float; scale = (1/dx)^3 * (-dx * dx) in double with 1/dx in float
// (GRID_HIERARCHY_PROJECTION.h:31-42, OLD_SCALING).  The solver flags are
// Dirichlet where the fluid cell is Dirichlet, else Active where it is Active.
// Memory bound: 4 x 4 B read and 8 B written per cell, plus the +x/+y/+z
// neighbours' flags and velocities, which come from the same lines or L2.
#include <cuda_runtime.h>

#include "hdd_common.h"
#include "velocity.h"

namespace hdd {

namespace {

constexpr int kVT = 256;
// Fluid flag bits (FLUIDS_SIMULATION_FLAGS.h:13-25).
constexpr uint32_t kInterior = 0x1u, kDirichlet = 0x2u, kGhost = 0x4u, kActive = 0x8u;

__global__ void __launch_bounds__(kVT) divergence_kernel(int n0, int n1, int n2, const uint32_t* __restrict__ ff,
                                                         const float* __restrict__ u, const float* __restrict__ v,
                                                         const float* __restrict__ w, double scale,
                                                         uint32_t* __restrict__ flags_out,
                                                         float* __restrict__ rhs_out) {
    const size_t n = (size_t)n0 * n1 * n2;
    const size_t x = (size_t)blockIdx.x * kVT + threadIdx.x;
    if (x >= n) return;
    const int k = (int)(x % n2);
    const size_t t = x / n2;
    const int j = (int)(t % n1), i = (int)(t / n1);
    const uint32_t f = ff[x];
    flags_out[x] = (f & kDirichlet) ? F_DIRICHLET : ((f & kActive) ? F_ACTIVE : 0u);
    float result = 0.0f;
    if (f & (kInterior | kGhost)) {
        const float* vel[3] = {u, v, w};
        const size_t stride[3] = {(size_t)n1 * n2, (size_t)n2, 1};
        const bool in[3] = {i + 1 < n0, j + 1 < n1, k + 1 < n2};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const uint32_t valid = 0x10u << a;
            const uint32_t fp = in[a] ? ff[x + stride[a]] : 0u;
            if (f & valid) result = (float)__dsub_rn((double)result, __dmul_rn(scale, (double)vel[a][x]));
            if (fp & valid) result = (float)__dadd_rn((double)result, __dmul_rn(scale, (double)vel[a][x + stride[a]]));
        }
    }
    rhs_out[x] = result;
}

}  // namespace

double divergence_scale(float dx) {
    const float odx = 1.0f / dx;
    return ((double)odx * (double)odx * (double)odx) * ((double)(-1.) * (double)dx * (double)dx);
}

cudaError_t launch_velocity_divergence(const int size[3], const uint32_t* fluid_flags, const float* u, const float* v,
                                       const float* w, float dx, uint32_t* flags_out, float* rhs_out,
                                       cudaStream_t stream) {
    const size_t n = (size_t)size[0] * size[1] * size[2];
    if (n == 0) return cudaSuccess;
    divergence_kernel<<<(unsigned)((n + kVT - 1) / kVT), kVT, 0, stream>>>(
        size[0], size[1], size[2], fluid_flags, u, v, w, divergence_scale(dx), flags_out, rhs_out);
    return cudaGetLastError();
}

}  // namespace hdd
