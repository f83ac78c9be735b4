// Allocation-free Laplacian + dot product on caller-owned device arrays.
//
// Some callers cannot call cudaMalloc at the point where they need the
// operator: a host framework whose caching allocator already owns the device
// memory budget, or a time-critical loop that must not take the implicit
// device synchronisation of an allocation.  This entry point lets them apply
// y = Project(A x) and read sum(x*y) with nothing allocated per call: the
// per-tile partial sums live in one fixed, file-scope device array.
//
// The kernel applies the tiled path's per-cell arithmetic on dense addresses:
// the same FP64 face sums in the same face order, so y is bit-identical to
// the tiled Laplacian on the same data; the dot sums the same FP32 products
// in FP64, per tile and then over tiles, in an order of its own.  Cells
// outside the stored tiles read as zero (as they do in the tiled vectors) and
// are not written.
//
// The scratch array is shared by every call in the process: two calls whose
// kernels overlap on the GPU race on it.  Every slot a call reads is written
// earlier by that same call, so nothing needs clearing between calls.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "dev_util.h"
#include "kernels.h"
#include "noalloc.h"

namespace hdd {
namespace {

constexpr int kNT = 256;
constexpr int kMaxDevices = 64;

// Per-tile FP64 partial sums of x*y, at most kNoAllocMaxTiles tiles.
static __device__ __align__(256) double g_noalloc_partial[kNoAllocMaxTiles];

std::mutex g_addr_mu;
double* g_addr[kMaxDevices] = {nullptr};

__device__ __forceinline__ float dense_value(const float* v, int sx, int sy, int sz, int gx, int gy, int gz) {
    if (gx < 0 || gy < 0 || gz < 0 || gx >= sx || gy >= sy || gz >= sz) return 0.0f;
    return v[((size_t)gx * sy + gy) * sz + gz];
}

__global__ void __launch_bounds__(kNT) laplace_dot_dense_kernel(TileGeom g, const int* __restrict__ tile_xyz, int sx,
                                                                int sy, int sz, const float* __restrict__ xv,
                                                                float* __restrict__ yv, double* partial) {
    const int t = blockIdx.x;
    const int S = g.sub, TC = S * S * S;
    const size_t base = (size_t)t * TC;
    const int ox = tile_xyz[3 * t] * S, oy = tile_xyz[3 * t + 1] * S, oz = tile_xyz[3 * t + 2] * S;
    double acc = 0.0;
    for (int c = threadIdx.x; c < TC; c += kNT) {
        const uint32_t fl = g.flags[base + c];
        const int z = c % S, tmp = c / S, y = tmp % S, x = tmp / S;
        const int gx = ox + x, gy = oy + y, gz = oz + z;
        const float sv = dense_value(xv, sx, sy, sz, gx, gy, gz);
        float out = 0.0f;
        if (fl & (C_ACTIVE | C_INTERFACE)) {
            const double cd = (double)sv;
            double result = 0.0;
#pragma unroll
            for (int face = 0; face < 6; ++face) {
                if (!(fl & (1u << face))) continue;
                // A neighbour across the tile face counts only if its tile is stored.
                const int axis = face >> 1, dir = (face & 1) ? 1 : -1;
                const int lc = axis == 0 ? x : (axis == 1 ? y : z);
                const bool crosses = (dir < 0) ? (lc == 0) : (lc == S - 1);
                float nv = 0.0f;
                if (!crosses || g.nbr[6 * t + face] >= 0)
                    nv = dense_value(xv, sx, sy, sz, gx + (axis == 0 ? dir : 0), gy + (axis == 1 ? dir : 0),
                                     gz + (axis == 2 ? dir : 0));
                result -= ((double)nv - cd);
            }
            out = (float)result;
        }
        if (gx < sx && gy < sy && gz < sz) yv[((size_t)gx * sy + gy) * sz + gz] = out;
        acc += (double)(sv * out);
    }
    // Block reduction.
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = acc;
    __syncthreads();
    if (w == 0) {
        acc = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    }
    if (threadIdx.x == 0) partial[t] = acc;
}

// Device address of the scratch array on the current device (looked up once
// per device; the host symbol itself is not a device address).
double* scratch_address(int device) {
    if (device < 0 || device >= kMaxDevices) throw Error(HDD_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (!g_addr[device]) {
        void* p = nullptr;
        dev::ck(cudaGetSymbolAddress(&p, g_noalloc_partial), "cudaGetSymbolAddress(no-alloc scratch)");
        g_addr[device] = static_cast<double*>(p);
    }
    return g_addr[device];
}

}  // namespace

void multiply_dot_dense_device_noalloc(const TileGeom& g, const int* tile_xyz, const int size[3], int device,
                                       const float* x, float* y, double* dot, cudaStream_t stream) {
    if (g.ntiles > kNoAllocMaxTiles)
        throw Error(HDD_ERR_INVALID_ARGUMENT, "domain has " + std::to_string(g.ntiles) +
                                                  " stored tiles; the allocation-free path holds at most " +
                                                  std::to_string(kNoAllocMaxTiles));
    double* partial = scratch_address(device);
    if (g.ntiles > 0) {
        laplace_dot_dense_kernel<<<g.ntiles, kNT, 0, stream>>>(g, tile_xyz, size[0], size[1], size[2], x, y, partial);
        dev::ck(cudaGetLastError(), "laplace_dot_dense_kernel");
    }
    dev::ck(launch_reduce_sum(partial, g.ntiles, dot, stream), "reduce_sum");
}

}  // namespace hdd
