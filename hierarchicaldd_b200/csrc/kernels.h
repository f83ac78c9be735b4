// Launch interfaces of the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace hdd {

constexpr int kMaxLevels = 8;

// k independent systems on one domain solved side by side: system j's
// vectors start j * vstride elements after system 0's, its per-tile partial
// sums j * pstride after, its scalars at PcgScalars + j.  active[j] == 0
// leaves system j's state untouched (its slot is free); first[j] != 0 starts
// its search direction afresh.  k = 1 with null arrays is a single system.
struct Batch {
    int k = 1;
    size_t vstride = 0;
    int pstride = 0;
    const int* active = nullptr;
    const int* first = nullptr;
};

struct VcycleArgs {
    float* u;                  // tiled level-0 solution (read halos, write interiors)
    const float* b;            // tiled level-0 right-hand side
    const uint8_t* box_flags;  // per-box flag records (all levels)
    const int* box_tile;       // [nbox]
    const int* box_nb;         // [nbox*3] +x/+y/+z neighbour tiles (-1 absent)
    // Optional (null = zero): the level-0 residual at the box's lower-face
    // cells (x, y or z = 0), which the V-cycle never computes there but the
    // first restriction reads (its stencil reaches box cells 0 .. sub-1).
    // The reference's V-cycle reads its residual channel there, and two-level
    // DD leaves Laplace_ir_Subdomain values in it
    // (TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Preconditioner.h:131-137).
    const float* r_halo;
    int nbox;
    int sub;                   // cubic subdomain edge
    int levels;
    size_t box_stride;
    size_t level_off[kMaxLevels];
    int n_vcycles, interior_itr, boundary_itr, bottom_itr;
    int halo_from_u;           // 1: halo planes hold interface values read from u
    int zero_init;             // 1: interior u starts at zero
    int cluster;               // CTAs per subdomain for sub 16 (1 or 2); sub 32 always uses 4
    float inv_diag[8];         // omega / face_count (float division on the host)
    float restrict_w[64];      // (1/8,3/8,3/8,1/8)^3 tensor weights
    float prolong_w[8];        // 4 * (3/4,1/4)^3 tensor weights
    // Systems side by side (blockIdx.y): u and b of system j at + j * slot_stride;
    // a system whose active entry is 0 is skipped.
    int nslots;
    size_t slot_stride;
    const int* active;
};

cudaError_t launch_vcycle(const VcycleArgs& a, cudaStream_t stream);

// The V-cycle's float constants (as in VcycleArgs).
struct VcycleWeights {
    float inv_diag[8];
    float restrict_w[64];
    float prolong_w[8];
};

struct TileGeom;

// Whole-grid V-cycle (kernels_vcycle_global.cu), for domains whose coarse
// levels couple subdomain boxes: level l is a dense x-slowest grid of
// dims[l] cells with compact8 flags f[l]; u, b, r are its vectors (level 0
// staged from and back to the tiled vectors).  Coarse r must be zero where a
// level is not Active (allocated zeroed; never written there).
struct GlobalVcycleArgs {
    int levels;
    int dims[kMaxLevels][3];
    const uint8_t* f[kMaxLevels];
    float* u[kMaxLevels];
    float* b[kMaxLevels];
    float* r[kMaxLevels];
    int n_vcycles, interior_itr, boundary_itr, bottom_itr;
    int halo_from_u, zero_init;   // as in VcycleArgs
    VcycleWeights w;
};
// Runs the V-cycles on the tiled u (read as VcycleArgs says, Active and other
// non-Interface cells written back) and b; r_halo (nullable) gives the
// level-0 residual where none is computed (as VcycleArgs::r_halo).  Returns
// the launches issued; throws hdd::Error on a launch error.
long long launch_vcycle_global(const GlobalVcycleArgs& a, const TileGeom& g, const int* tile_xyz, float* u,
                               const float* b, const float* r_halo, cudaStream_t stream);

// ---------------------------------------------------------------------------
// PCG kernels over tiled vectors
// ---------------------------------------------------------------------------
struct TileGeom {
    int sub;                   // cubic tile edge
    int ntiles;
    const int* nbr;            // [ntiles*6] face-neighbour tiles (-x,+x,-y,+y,-z,+z), -1 absent
    const uint16_t* flags;     // compact16 per tile cell
};

// q = Project(A s) (double accumulation, CG_SYSTEM::Multiply + Project);
// partial[0 .. laplace_partials(g)) = sums of (double)(s*q) (float products)
// over fixed parts of the tiles, to be reduced with launch_reduce_sum.
cudaError_t launch_laplace_dot(const TileGeom& g, const float* s, float* q, double* partial,
                               cudaStream_t stream, const Batch& B = Batch());
int laplace_partials(const TileGeom& g);

// Deterministic final sums of per-tile partials into out[slot] (double);
// batched: system j's n partials at partial + j * pstride into out[j * ostride].
cudaError_t launch_reduce_sum(const double* partial, int n, double* out, cudaStream_t stream,
                              const Batch& B = Batch(), int ostride = 0);
cudaError_t launch_reduce_max(const float* partial, int n, float* out, cudaStream_t stream,
                              const Batch& B = Batch(), int ostride = 0);

// Scalar state of the PCG loop on the device.
struct PcgScalars {
    double rho_d, rho_old_d, sdq_d;   // raw FP64 sums
    double alpha_d, beta_d;           // mixed-precision scalars
    float rho, rho_old, alpha, beta;  // reference FP32 scalars
    float rmax;                       // max|r|
    int iteration;
    int status;                       // 0 ok, 1 non-finite scalar
};

// partial[tile] = sum (double)(a*b) with project(a) applied in place.
cudaError_t launch_project_dot(const TileGeom& g, float* a, const float* b, double* partial,
                               cudaStream_t stream, const Batch& B = Batch());
// s = beta*s + z (first: s = z); beta from scalars (mode 0 float, 1 double).
cudaError_t launch_update_s(const TileGeom& g, float* s, const float* z, const PcgScalars* sc, int first,
                            int mode, cudaStream_t stream, const Batch& B = Batch());
// x += alpha s; r -= alpha q; partial max|r| per tile.  With xd (mode 1) the
// iterate is kept in FP64 (xd += alpha s) and x is its FP32 rounding.
cudaError_t launch_update_xr(const TileGeom& g, float* x, float* r, const float* s, const float* q,
                             const PcgScalars* sc, int mode, float* partial_max, cudaStream_t stream,
                             double* xd = nullptr, const Batch& B = Batch());
// r = Project((float)(b - A x)) for an FP64 iterate x, in FP64; partial max|r|
// (batched: only the systems whose active entry is set).
cudaError_t launch_residual_f64(const TileGeom& g, const float* b, const double* x, float* r, float* partial_max,
                                cudaStream_t stream, const Batch& B = Batch());
// Scalar steps (one thread per system); batched sums at sum + j * sstride.
cudaError_t launch_scalar_rho(PcgScalars* sc, const double* rho_sum, int first, cudaStream_t stream,
                              const Batch& B = Batch(), int sstride = 0);
cudaError_t launch_scalar_alpha(PcgScalars* sc, const double* sdq_sum, cudaStream_t stream, const Batch& B = Batch(),
                                int sstride = 0);
// r = Project(b - A x); partial max|r|.  precise = 1 subtracts A x in FP64
// before rounding r (else A x is rounded to FP32 first, as the reference).
cudaError_t launch_residual(const TileGeom& g, const float* b, const float* x, float* r, float* partial_max,
                            cudaStream_t stream, int precise = 0);
// v = Project(v).
cudaError_t launch_project(const TileGeom& g, float* v, cudaStream_t stream);
// Dense (x-slowest grid of size[0..2]) <-> tiled copies on the device;
// tile_xyz holds the tile coordinates of every stored tile.
cudaError_t launch_dense_to_tiles(const TileGeom& g, const int* tile_xyz, int sx, int sy, int sz, const float* dense,
                                  float* tiled, cudaStream_t stream);
cudaError_t launch_tiles_to_dense(const TileGeom& g, const int* tile_xyz, int sx, int sy, int sz, const float* tiled,
                                  float* dense, cudaStream_t stream);
cudaError_t launch_tiles_to_dense_f64(const TileGeom& g, const int* tile_xyz, int sx, int sy, int sz,
                                      const double* tiled, double* dense, cudaStream_t stream);

// ---------------------------------------------------------------------------
// Interface coupling (Laplace_ri gather and the interface scatter)
// ---------------------------------------------------------------------------
// With s_i = (float)(-sum of z over the cell's listed neighbour slots, in
// FP64, face order -x,+x,-y,+y,-z,+z), at the listed cells c_i:
//   kGatherRi    b0[i] = r[c_i] - s_i        (Laplace_ri / Laplace_ri_Subdomain, then the copy)
//   kGatherIr    b0[i] = -s_i                (Laplace_ir_Subdomain, then the copy)
//   kGatherRiAdd b0[i] = b0[i] + (r[c_i] - s_i)  (Laplace_ri, then Accumulate_To_Eigen_Array)
//   kGatherIrTiled b0[c_i] = -s_i            (Laplace_ir_Subdomain into a tiled vector b0)
// The neighbour lists choose which neighbours count (-1 = none).
// Batched: system j's r and z at + j * B.vstride, its b0 at + j * istride.
enum { kGatherRi = 0, kGatherIr = 1, kGatherRiAdd = 2, kGatherIrTiled = 3 };
cudaError_t launch_interface_gather(const TileGeom& g, const long long* iface_slot, const int* iface_nb_slots,
                                    int n_iface, const float* r, const float* z, float* b0,
                                    cudaStream_t stream, const Batch& B = Batch(), size_t istride = 0,
                                    int mode = kGatherRi);
// z[c_i] = u0[i].
cudaError_t launch_interface_scatter(const long long* iface_slot, int n_iface, const float* u0, float* z,
                                     cudaStream_t stream, const Batch& B = Batch(), size_t istride = 0);

}  // namespace hdd
