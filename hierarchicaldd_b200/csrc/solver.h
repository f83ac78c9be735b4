// Solver object behind the C ABI: host setup, device buffers and the PCG
// orchestration on one stream.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <memory>
#include <string>
#include <vector>

#include "hdd_common.h"
#include "host_setup.h"
#include "kernels.h"
#include "sigma.h"

namespace hdd {

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        release();
        if (count == 0) return;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            throw Error(e == cudaErrorMemoryAllocation ? HDD_ERR_OUT_OF_MEMORY : HDD_ERR_CUDA,
                        std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        n = count;
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        alloc(count);
        if (count) check(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void zero(cudaStream_t s) {
        if (n) check(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
    static void check(cudaError_t e) {
        if (e != cudaSuccess) throw Error(HDD_ERR_CUDA, cudaGetErrorString(e));
    }
};

// Host-side NVTX range named after the reference's LOG::SCOPE phases
// (SPGrid_Domain_Decomposition_Preconditioner.h:119-152 of the GPU demo:
// "Step ONE", "Sigma_V_Cycle", "Step Two"; Solver.h:193 "solve"), for Nsight
// timelines; a no-op unless a profiler is attached.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(HDD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

struct Solver {
    hdd_options opts;
    std::string last_error;
    long long launches = 0;

    bool have_domain = false, initialized = false, solved = false;
    DomainLayout L;
    std::vector<uint32_t> flags_in;
    std::vector<float> rhs_dense;

    cudaStream_t stream = nullptr;
    DevBuf<float> x, b, r, z, s, q;
    DevBuf<double> xd;      // precision form: the FP64 iterate (x is its FP32 rounding)
    DevBuf<uint16_t> tflags;
    DevBuf<int> tile_nbr, box_tile, box_nb, tile_xyz;
    DevBuf<float> dense;   // staging buffer in the caller's dense layout
    DevBuf<uint8_t> box_flags;
    DevBuf<double> partial, sums;
    DevBuf<float> partial_max, scalars_f;
    DevBuf<PcgScalars> scal;
    // Level-0 interface DOFs (sigma level 0 order).
    DevBuf<long long> iface_slot;
    DevBuf<int> iface_nb;
    SigmaGpu sigma;
    InterfaceHost ih;
    int iomode = HDD_IOMODE_NEITHER;  // interface dump / reload at initialize()
    std::string io_dir;
    double setup_ms = 0;
    // max|r| of the recursively updated residual at the start of each PCG
    // iteration of the last solve (entry 0: r = b), for parity checks against
    // the oracle's history.
    std::vector<double> history;
    // Step lengths alpha and beta of every PCG iteration of the last solve.
    std::vector<double> alphas, betas;
    // Host wall time of the setup phases: layout and vector uploads, interface
    // system (assembly or reload, and dump), interface solver (factorisations
    // and solve plans), total.
    double setup_phase_ms[4] = {0, 0, 0, 0};

    // Optional per-phase device timing with CUDA events on the solver stream
    // (categories: 0 V-cycle kernel, 1 Laplacian kernel, 2 PCG vector kernels,
    // 3 interface gather/scatter, 4 sigma V-cycle (includes 6 and 7),
    // 5 dense<->tile copies, 6 supernodal forward, 7 supernodal backward),
    // with each phase's algorithmic bytes.
    static constexpr int kCats = 8;
    bool timing = false;
    double cat_ms[kCats] = {0};
    long long cat_n[kCats] = {0};
    double cat_bytes[kCats] = {0};
    double vcycle_bytes = 0, laplace_bytes = 0;  // algorithmic bytes of one launch
    struct Pending { int cat; cudaEvent_t a, b; double bytes; };
    std::vector<Pending> pending;
    struct Tm {
        Solver* s; int cat; double bytes; cudaEvent_t a = nullptr, b = nullptr;
        Tm(Solver* sv, int c, double by = 0) : s(sv), cat(c), bytes(by) {
            if (!s->timing) return;
            cudaEventCreate(&a); cudaEventCreate(&b);
            cudaEventRecord(a, s->stream);
        }
        ~Tm() {
            if (!a) return;
            cudaEventRecord(b, s->stream);
            s->pending.push_back({cat, a, b, bytes});
        }
    };
    // Phase hook for the sigma solver's supernodal launches.
    struct Hook : PhaseHook {
        Solver* s = nullptr;
        cudaEvent_t a = nullptr;
        void begin(int) override {
            if (!s->timing) return;
            cudaEventCreate(&a);
            cudaEventRecord(a, s->stream);
        }
        void end(int phase, double bytes) override {
            if (!s->timing || !a) return;
            cudaEvent_t b;
            cudaEventCreate(&b);
            cudaEventRecord(b, s->stream);
            s->pending.push_back({phase, a, b, bytes});
            a = nullptr;
        }
    } hook;
    void collect_timing();

    explicit Solver(const hdd_options& o);
    ~Solver();

    void set_domain(const uint32_t* flags, const float* rhs);
    // Same, taking over dense arrays the caller built (no second copy).
    void set_domain(std::vector<uint32_t>&& flags, std::vector<float>&& rhs);
    void set_rhs(const float* rhs);
    void initialize();
    void solve(hdd_result* res);
    void get_solution(float* out);
    void get_solution_f64(double* out);
    void apply_preconditioner_dense(const float* r, float* zout);
    void vcycle_dense(float* u, const float* bb, int nv);
    void multiply_dense(const float* xin, float* yout);
    void sigma_vcycle_host(const float* b0, float* u0);
    // One Arr (kind 0) or concatenated Aii (kind 1) supernodal solve of a sigma level.
    void interface_solve(int kind, int level, const float* bh, float* xh, int* n);
    // Throws HDD_ERR_TIMEOUT when a device-side bounded wait gave up.
    void check_waits();

    // Device pieces.
    TileGeom geom() const;
    VcycleArgs vcycle_args(float* u, const float* bb, int halo_from_u, int zero_init, int nv) const;
    void run_vcycle(float* u, const float* bb, int halo_from_u, int zero_init, int nv);
    void apply_preconditioner(const float* rr, float* zz);   // device tiled vectors
    void count(int n = 1) { launches += n; }
    void sync() { cuda_check(cudaStreamSynchronize(stream), "stream sync"); }
    // Device memory held by this solver (vectors, tables, interface solver).
    size_t device_bytes() const {
        size_t t = 0;
        for (const DevBuf<float>* v : {&x, &b, &r, &z, &s, &q, &dense, &partial_max, &scalars_f}) t += v->n * sizeof(float);
        t += tflags.n * sizeof(uint16_t) + box_flags.n;
        for (const DevBuf<int>* v : {&tile_nbr, &box_tile, &box_nb, &tile_xyz, &iface_nb}) t += v->n * sizeof(int);
        t += (partial.n + sums.n + xd.n) * sizeof(double) + iface_slot.n * sizeof(long long);
        return t + sigma.device_bytes;
    }
};

}  // namespace hdd
