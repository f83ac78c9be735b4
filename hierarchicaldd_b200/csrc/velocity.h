// Velocity -> divergence right-hand side and flag conversion (velocity.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace hdd {

// scale = (1/dx)^3 * (-dx * dx), 1/dx in float, the rest in double.
double divergence_scale(float dx);

// Device arrays, dense x-slowest over size[0..2] cells: fluid flags and face
// velocities in; the solver's flags and the divergence right-hand side out.
cudaError_t launch_velocity_divergence(const int size[3], const uint32_t* fluid_flags, const float* u, const float* v,
                                       const float* w, float dx, uint32_t* flags_out, float* rhs_out,
                                       cudaStream_t stream);

}  // namespace hdd
