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

// The device state one PCG solve writes, on its own stream: the tiled
// vectors, reduction partials and scalars, the sigma V-cycle's buffers, the
// CUDA graph of one preconditioner application on them, and the last solve's
// record.  A Solver's first context (`w0`) serves the C ABI's single-solve
// calls; a server adds contexts to run several solves of one resident domain
// at once, all reading the domain's factors, matrices and layout tables.
struct Work {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // Systems held side by side (1, 2 or 4): system j's tiled vectors at
    // + j * vstride, its per-tile partial sums at + j * pstride, its scalars at
    // scal + j; active / first / replace are per-system flags on the device.
    int k = 1;
    size_t vstride = 0;
    int pstride = 0;
    DevBuf<int> active, first, replace;
    DevBuf<float> x, b, r, z, s, q;
    DevBuf<float> hr;       // two-level DD: the V-cycle's lower-face residual input
    DevBuf<float> gu[kMaxLevels], gb[kMaxLevels], gr[kMaxLevels];  // whole-grid V-cycle levels
    DevBuf<double> xd;      // precision form: the FP64 iterate (x is its FP32 rounding)
    DevBuf<float> dense;    // staging buffer in the caller's dense layout
    DevBuf<double> partial, sums;
    DevBuf<float> partial_max, scalars_f;
    DevBuf<PcgScalars> scal;
    SigmaScratch sig;
    bool own_sig = false;
    SigmaScratch sig2;      // two-level DD: the second-level interface solver's vectors
    bool own_sig2 = false;
    // CUDA graph of one preconditioner application (on buffers pc_r -> pc_z)
    // and the kernel launches it holds; dropped when a launch parameter
    // changes (re-initialisation, the wait limit).
    bool use_graphs = true;
    cudaGraphExec_t pc_exec = nullptr;
    const float* pc_r = nullptr;
    float* pc_z = nullptr;
    long long pc_launches = 0;
    long long launches = 0;  // kernel launches issued on this context
    bool solved = false;
    // max|r| of the recursively updated residual at the start of each PCG
    // iteration of the last solve (entry 0: r = b), for parity checks against
    // the oracle's history; step lengths alpha and beta of every iteration.
    std::vector<double> history, alphas, betas;

    Work() = default;
    Work(const Work&) = delete;
    Work& operator=(const Work&) = delete;
    ~Work();
    void release_graphs();
    size_t bytes() const {
        size_t t = 0;
        for (const DevBuf<float>* v : {&x, &b, &r, &z, &s, &q, &hr, &dense, &partial_max, &scalars_f})
            t += v->n * sizeof(float);
        for (int l = 0; l < kMaxLevels; ++l) t += (gu[l].n + gb[l].n + gr[l].n) * sizeof(float);
        t += (partial.n + sums.n + xd.n) * sizeof(double) + scal.n * sizeof(PcgScalars);
        t += (active.n + first.n + replace.n) * sizeof(int);
        return t + (own_sig ? sig.bytes : 0) + (own_sig2 ? sig2.bytes : 0);
    }
    // The launch description of all k systems (a plain single system for k = 1).
    Batch batch() const {
        Batch B;
        if (k == 1) return B;
        B.k = k;
        B.vstride = vstride;
        B.pstride = pstride;
        B.active = active.p;
        B.first = first.p;
        return B;
    }
};

// Supplies a batched solve with requests and takes their results: next()
// fills a free system's right-hand side (dense, in the caller's layout) and
// returns false when nothing is waiting; done() hands back a finished
// request's status, result and dense solution.
struct BatchFeeder {
    virtual bool next(const float** rhs, long long* id) = 0;
    virtual void done(long long id, hdd_status st, const hdd_result& res, std::vector<float>&& x) = 0;

protected:
    ~BatchFeeder() = default;
};

struct Solver {
    hdd_options opts;
    std::string last_error;

    bool have_domain = false, initialized = false;
    DomainLayout L;
    std::vector<uint32_t> flags_in;
    std::vector<float> rhs_dense;

    // Read-only device data of the domain, shared by every solve context.
    DevBuf<uint16_t> tflags;
    DevBuf<int> tile_nbr, box_tile, box_nb, tile_xyz;
    DevBuf<uint8_t> box_flags;
    DevBuf<uint8_t> gflags[kMaxLevels];  // whole-grid V-cycle: compact8 flags per level
    // Level-0 interface DOFs (sigma level 0 order).
    DevBuf<long long> iface_slot;
    DevBuf<int> iface_nb;
    SigmaGpu sigma;
    InterfaceHost ih;
    // Two-level DD (opts.multilevel): the second-level interface system (all
    // first-level subdomains' systems as one block-diagonal system), its
    // cells' slots and the neighbour lists of its three gathers.  iface_nb
    // then lists, for the first-level interface cells, the neighbours off the
    // first-level planes (Laplace_ri_Subdomain).
    SigmaGpu sigma2;
    InterfaceHost ih2;
    DevBuf<long long> iface2_slot;
    DevBuf<int> iface2_nb_ir, iface2_nb_ri;
    // The cells where Laplace_ir_Subdomain can leave a nonzero value on a
    // V-cycle box face: Interface cells off the first-level planes with a
    // first-level plane neighbour; their slots and those neighbours.
    DevBuf<long long> face_slot;
    DevBuf<int> face_nb;
    int n_face = 0;
    int iomode = HDD_IOMODE_NEITHER;  // interface dump / reload at initialize()
    std::string io_dir;
    double setup_ms = 0;
    Work w0;                    // the first solve context (owns the solver's stream)
    cudaStream_t& stream = w0.stream;
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
    // Timed phases are recorded on the first context only.
    struct Tm {
        Solver* s; cudaStream_t st; int cat; double bytes; cudaEvent_t a = nullptr, b = nullptr;
        Tm(Solver* sv, const Work& w, int c, double by = 0) : s(sv), st(w.stream), cat(c), bytes(by) {
            if (!s->timing || &w != &s->w0) return;
            cudaEventCreate(&a); cudaEventCreate(&b);
            cudaEventRecord(a, st);
        }
        ~Tm() {
            if (!a) return;
            cudaEventRecord(b, st);
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
    void set_rhs(const float* rhs) { set_rhs(w0, rhs); }
    void initialize();
    void solve(hdd_result* res) { solve(w0, res); }
    void get_solution(float* out) { get_solution(w0, out); }
    void get_solution_f64(double* out);
    // A further solve context of this domain on a stream of its own (device
    // buffers for the vectors and the sigma V-cycle; bytes() tells how much).
    // Contexts run solves concurrently from different host threads; the
    // domain's own setup state is only read.
    std::unique_ptr<Work> make_work(int k = 1);
    // Most systems a batch of this domain can hold (the interface solver's
    // largest fronts bound it).
    int max_batch() const;
    // Continuous batching: solves requests from the feeder on w's k systems
    // side by side until no system is busy and none is waiting.  A request
    // joins in the first iteration in which a system is free; each one's
    // result is bit-identical to its solve alone.
    void solve_batch(Work& w, BatchFeeder& feed);
    void set_rhs(Work& w, const float* rhs);
    void solve(Work& w, hdd_result* res);
    void get_solution(Work& w, float* out);
    void apply_preconditioner_dense(const float* r, float* zout);
    void vcycle_dense(float* u, const float* bb, int nv);
    void multiply_dense(const float* xin, float* yout);
    void sigma_vcycle_host(const float* b0, float* u0);
    // One Arr (kind 0) or concatenated Aii (kind 1) supernodal solve of a sigma level.
    void interface_solve(int kind, int level, const float* bh, float* xh, int* n);
    // The same for nrhs (1, 2 or 4) right-hand sides solved in one launch pair.
    void interface_solve_batch(int kind, int level, int nrhs, const float* bh, float* xh, int* n);
    // Throws HDD_ERR_TIMEOUT when a device-side bounded wait gave up.
    void check_waits() { check_waits(w0); }
    void check_waits(Work& w);

    // Device pieces.
    TileGeom geom() const;
    VcycleArgs vcycle_args(float* u, const float* bb, int halo_from_u, int zero_init, int nv) const;
    void run_vcycle(Work& w, float* u, const float* bb, int halo_from_u, int zero_init, int nv,
                    const float* r_halo = nullptr);
    void apply_preconditioner(Work& w, const float* rr, float* zz);   // device tiled vectors (graph replay)
    void apply_preconditioner_launches(Work& w, const float* rr, float* zz);
    void build_two_level_interfaces();
    void two_level_launches(Work& w, const float* rr, float* zz);
    void subdomain_dd(Work& w, const float* rr, float* zz, bool second);
    int wait_error(Work& w);   // the contexts' bounded-wait error words (0: none)
    void clear_wait_errors(Work& w);
    void release_graphs() { w0.release_graphs(); }
    void alloc_vectors(Work& w);
    static void count(Work& w, int n = 1) { w.launches += n; }
    void sync() { cuda_check(cudaStreamSynchronize(stream), "stream sync"); }
    static void sync(Work& w) { cuda_check(cudaStreamSynchronize(w.stream), "stream sync"); }
    // Device memory held by this solver (tables, interface solver and the
    // first context).
    size_t device_bytes() const {
        size_t t = tflags.n * sizeof(uint16_t) + box_flags.n;
        for (int l = 0; l < kMaxLevels; ++l) t += gflags[l].n;
        for (const DevBuf<int>* v : {&tile_nbr, &box_tile, &box_nb, &tile_xyz, &iface_nb, &iface2_nb_ir, &iface2_nb_ri})
            t += v->n * sizeof(int);
        t += (iface_slot.n + iface2_slot.n + face_slot.n) * sizeof(long long) + face_nb.n * sizeof(int);
        return t + sigma.device_bytes + sigma2.device_bytes + w0.bytes();
    }
    // Device bytes a further context of this domain allocates.
    size_t work_bytes(int k = 1) const;
};

}  // namespace hdd
