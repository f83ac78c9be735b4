// Allocation-free Laplacian + dot product (noalloc.cu).
#pragma once
#include <cuda_runtime.h>

#include "kernels.h"

namespace hdd {

// Largest number of stored tiles the fixed scratch array covers
// (32768 doubles = 256 KiB of device memory per GPU).
constexpr int kNoAllocMaxTiles = 32768;

// y = Project(A x) on dense device arrays (x-major, z fastest, size[0..2]) and
// *dot = sum(x*y) over the stored tiles, with no device allocation.  The
// first call on a device looks up the scratch array's device address.
void multiply_dot_dense_device_noalloc(const TileGeom& g, const int* tile_xyz, const int size[3], int device,
                                       const float* x, float* y, double* dot, cudaStream_t stream);

}  // namespace hdd
