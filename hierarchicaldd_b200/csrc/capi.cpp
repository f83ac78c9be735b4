// C ABI (include/hdd.h): status codes instead of exceptions, opaque handles.
#include <cmath>
#include <cstring>
#include <fstream>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "noalloc.h"
#include "solver.h"
#include "velocity.h"

using hdd::Error;
using hdd::Solver;

struct hdd_solver {
    Solver* impl = nullptr;
    std::string err;
};

namespace {
template <class F>
hdd_status guard(hdd_solver* s, F&& f) {
    if (!s || !s->impl) return HDD_ERR_INVALID_ARGUMENT;
    try {
        f(*s->impl);
        s->err.clear();
        return HDD_OK;
    } catch (const Error& e) {
        s->err = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        s->err = "host allocation failed";
        return HDD_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        s->err = e.what();
        return HDD_ERR_INTERNAL;
    }
}

// Makes `device` current for its lifetime and restores the calling thread's
// previous device afterwards (also when an exception leaves the scope).
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int device) {
        hdd::cuda_check(cudaGetDevice(&prev), "cudaGetDevice");
        if (prev != device) hdd::cuda_check(cudaSetDevice(device), "cudaSetDevice");
        else prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// Reads the reference SPGrid directory format (SPGRID_READ_WRITE.h:31-106):
// `size` = d ints, `block_offset` = int count + PhysBAM array (int length +
// uint64 page offsets), `flags`/`data` = per block a PhysBAM array of 256
// 4-byte values.  Pages are 4x8x8 cells with bit-interleaved page addresses.
bool read_file(const std::string& path, std::vector<char>& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return true;
}
uint64_t compact_bits(uint64_t v, uint64_t mask) {
    uint64_t r = 0, bit = 1;
    for (uint64_t m = mask; m; m &= m - 1) {
        const uint64_t low = m & (~m + 1);
        if (v & low) r |= bit;
        bit <<= 1;
    }
    return r;
}
}  // namespace

extern "C" {

void hdd_options_default(hdd_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    for (int a = 0; a < 3; ++a) { o->size[a] = 257; o->sub_size[a] = 64; }
    o->vlevels = 3;
    o->nVcycles = 1;
    o->interior_smoothing = 1;
    o->boundary_smoothing = 3;
    o->sigma_levels = 3;
    o->sigma_smoothing = 3;
    o->sigma_mg = 1;
    o->tol = 1e-6;
    o->relative_tol = 1;
    o->max_iters = 5000;
    o->min_iters = 0;
    o->precision_mode = HDD_PRECISION_REFERENCE;
    o->true_residual_every = 20;
    o->device = 0;
    o->coarse_solve = HDD_COARSE_REFERENCE;
    o->solve_share = 0;
    o->multilevel = 0;
}

hdd_status hdd_create(const hdd_options* opts, hdd_solver** out) {
    if (!opts || !out) return HDD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    hdd_solver* h = new (std::nothrow) hdd_solver();
    if (!h) return HDD_ERR_OUT_OF_MEMORY;
    try {
        h->impl = new Solver(*opts);
    } catch (const Error& e) {
        delete h;
        return e.status;
    } catch (...) {
        delete h;
        return HDD_ERR_INTERNAL;
    }
    *out = h;
    return HDD_OK;
}

hdd_status hdd_set_domain_dense(hdd_solver* s, const uint32_t* flags, const float* rhs) {
    if (!flags || !rhs) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) { v.set_domain(flags, rhs); });
}

namespace {
// Runs the velocity conversion on the solver's device into host flags/rhs.
void velocity_to_domain(Solver& v, const uint32_t* ff, const float* u, const float* vv, const float* w, float dx,
                        uint32_t* flags_out, float* rhs_out) {
    if (!(dx > 0.0f) || !std::isfinite(dx)) throw Error(HDD_ERR_INVALID_ARGUMENT, "dx must be positive and finite");
    hdd::cuda_check(cudaSetDevice(v.opts.device), "cudaSetDevice");
    const size_t N = (size_t)v.opts.size[0] * v.opts.size[1] * v.opts.size[2];
    hdd::DevBuf<uint32_t> dff, dfo;
    hdd::DevBuf<float> du, dv, dw, dr;
    cudaStream_t st = v.stream;
    dff.upload(ff, N, st);
    du.upload(u, N, st);
    dv.upload(vv, N, st);
    dw.upload(w, N, st);
    dfo.alloc(N);
    dr.alloc(N);
    hdd::cuda_check(hdd::launch_velocity_divergence(v.opts.size, dff.p, du.p, dv.p, dw.p, dx, dfo.p, dr.p, st),
                    "velocity divergence");
    v.count(v.w0);
    hdd::cuda_check(cudaMemcpyAsync(flags_out, dfo.p, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "D2H");
    hdd::cuda_check(cudaMemcpyAsync(rhs_out, dr.p, N * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H");
    v.sync();
}
}  // namespace

hdd_status hdd_velocity_divergence_dense(hdd_solver* s, const uint32_t* fluid_flags, const float* u, const float* v,
                                         const float* w, float dx, uint32_t* flags_out, float* rhs_out) {
    if (!fluid_flags || !u || !v || !w || !flags_out || !rhs_out) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& sv) { velocity_to_domain(sv, fluid_flags, u, v, w, dx, flags_out, rhs_out); });
}

hdd_status hdd_set_domain_velocity_dense(hdd_solver* s, const uint32_t* fluid_flags, const float* u, const float* v,
                                         const float* w, float dx) {
    if (!fluid_flags || !u || !v || !w) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& sv) {
        const size_t N = (size_t)sv.opts.size[0] * sv.opts.size[1] * sv.opts.size[2];
        std::vector<uint32_t> f(N);
        std::vector<float> b(N);
        velocity_to_domain(sv, fluid_flags, u, v, w, dx, f.data(), b.data());
        sv.set_domain(std::move(f), std::move(b));
    });
}

hdd_status hdd_set_domain_pages(hdd_solver* s, long long n_pages, const int32_t* page_origin,
                                const uint32_t* flags, const float* rhs) {
    if ((n_pages > 0 && (!page_origin || !flags || !rhs)) || n_pages < 0) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        const size_t N = (size_t)v.opts.size[0] * v.opts.size[1] * v.opts.size[2];
        std::vector<uint32_t> f(N, 0u);
        std::vector<float> b(N, 0.0f);
        hdd::pages_to_dense(v.opts.size, n_pages, page_origin, flags, f.data());
        hdd::pages_to_dense(v.opts.size, n_pages, page_origin, rhs, b.data());
        v.set_domain(std::move(f), std::move(b));
    });
}

hdd_status hdd_set_rhs_pages(hdd_solver* s, long long n_pages, const int32_t* page_origin, const float* rhs) {
    if ((n_pages > 0 && (!page_origin || !rhs)) || n_pages < 0) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        if (!v.initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
        std::vector<float> b((size_t)v.opts.size[0] * v.opts.size[1] * v.opts.size[2], 0.0f);
        hdd::pages_to_dense(v.opts.size, n_pages, page_origin, rhs, b.data());
        v.set_rhs(b.data());
    });
}

hdd_status hdd_get_solution_pages(hdd_solver* s, long long n_pages, const int32_t* page_origin, float* x) {
    if ((n_pages > 0 && (!page_origin || !x)) || n_pages < 0) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        std::vector<float> d((size_t)v.opts.size[0] * v.opts.size[1] * v.opts.size[2]);
        v.get_solution(d.data());
        hdd::dense_to_pages(v.opts.size, n_pages, page_origin, d.data(), x);
    });
}

hdd_status hdd_load_spgrid_dir(hdd_solver* s, const char* dir) {
    if (!dir) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        const std::string d(dir);
        std::vector<char> fs, fo, ff, fd;
        if (!read_file(d + "/size", fs) || !read_file(d + "/block_offset", fo) || !read_file(d + "/flags", ff) ||
            !read_file(d + "/data", fd))
            throw Error(HDD_ERR_IO, "cannot read SPGrid directory " + d);
        if (fs.size() != 12) throw Error(HDD_ERR_UNSUPPORTED, "only 3D SPGrid directories are supported");
        // The writer stores the allocator's padded size (a multiple of the block
        // size), so any size at least options.size is accepted; cells beyond
        // options.size are ignored.
        int32_t size[3];
        std::memcpy(size, fs.data(), 12);
        for (int a = 0; a < 3; ++a)
            if (size[a] < v.opts.size[a])
                throw Error(HDD_ERR_INVALID_ARGUMENT, "SPGrid size is smaller than options.size");
        for (int a = 0; a < 3; ++a) size[a] = v.opts.size[a];
        int32_t count = 0, alen = 0;
        if (fo.size() < 8) throw Error(HDD_ERR_IO, "truncated block_offset");
        std::memcpy(&count, fo.data(), 4);
        std::memcpy(&alen, fo.data() + 4, 4);
        if (count < 0 || alen != count || fo.size() != 8 + (size_t)count * 8) throw Error(HDD_ERR_IO, "bad block_offset");
        const size_t rec = 4 + 256 * 4;
        if (ff.size() != (size_t)count * rec || fd.size() != (size_t)count * rec) throw Error(HDD_ERR_IO, "bad flags/data size");
        const size_t N = (size_t)size[0] * size[1] * size[2];
        std::vector<uint32_t> flags(N, 0u);
        std::vector<float> rhs(N, 0.0f);
        const uint64_t XM = 0x9249249249249000ull | 0x300ull, YM = 0x4924924924924000ull | 0x0e0ull,
                       ZM = 0x2492492492492000ull | 0x01cull;
        for (int bi = 0; bi < count; ++bi) {
            uint64_t off;
            std::memcpy(&off, fo.data() + 8 + 8 * (size_t)bi, 8);
            for (int e = 0; e < 256; ++e) {
                const uint64_t lin = off + (uint64_t)e * 4;  // flags field (4-byte) offsets
                const int x = (int)compact_bits(lin, XM), y = (int)compact_bits(lin, YM), z = (int)compact_bits(lin, ZM);
                uint32_t fv;
                float dv;
                std::memcpy(&fv, ff.data() + (size_t)bi * rec + 4 + 4 * e, 4);
                std::memcpy(&dv, fd.data() + (size_t)bi * rec + 4 + 4 * e, 4);
                if (x < size[0] && y < size[1] && z < size[2]) {
                    const size_t di = ((size_t)x * size[1] + y) * size[2] + z;
                    flags[di] = fv;
                    rhs[di] = dv;
                }
            }
        }
        v.set_domain(std::move(flags), std::move(rhs));
    });
}

hdd_status hdd_initialize_preconditioner(hdd_solver* s) {
    return guard(s, [&](Solver& v) { v.initialize(); });
}

hdd_status hdd_set_rhs_dense(hdd_solver* s, const float* rhs) {
    if (!rhs) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        if (!v.initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
        v.set_rhs(rhs);
    });
}

hdd_status hdd_solve(hdd_solver* s, hdd_result* result) {
    return guard(s, [&](Solver& v) { v.solve(result); });
}

hdd_status hdd_get_solution_dense(hdd_solver* s, float* x) {
    if (!x) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) { v.get_solution(x); });
}

hdd_status hdd_get_solution_dense_f64(hdd_solver* s, double* x) {
    if (!x) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) { v.get_solution_f64(x); });
}

hdd_status hdd_get_residual_history(hdd_solver* s, double* out, int capacity, int* n) {
    if (!n || capacity < 0 || (capacity > 0 && !out)) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        if (!v.w0.solved) throw Error(HDD_ERR_NOT_INITIALIZED, "no solve has run");
        *n = (int)v.w0.history.size();
        for (int i = 0; i < capacity && i < *n; ++i) out[i] = v.w0.history[i];
    });
}

hdd_status hdd_apply_preconditioner_dense(hdd_solver* s, const float* r, float* z) {
    if (!r || !z) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) { v.apply_preconditioner_dense(r, z); });
}

hdd_status hdd_vcycle_dense(hdd_solver* s, float* u, const float* b, int n_vcycles) {
    if (!u || !b || n_vcycles < 0) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) { v.vcycle_dense(u, b, n_vcycles); });
}

hdd_status hdd_get_setup_timing(hdd_solver* s, double* ms) {
    if (!ms) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        if (!v.initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
        for (int k = 0; k < 4; ++k) ms[k] = v.setup_phase_ms[k];
    });
}

hdd_status hdd_set_iomode(hdd_solver* s, int iomode, const char* directory) {
    return guard(s, [&](Solver& v) {
        if (iomode < HDD_IOMODE_NEITHER || iomode > HDD_IOMODE_INPUT)
            throw Error(HDD_ERR_INVALID_ARGUMENT, "iomode must be HDD_IOMODE_NEITHER, _OUTPUT or _INPUT");
        if (iomode != HDD_IOMODE_NEITHER && (!directory || !*directory))
            throw Error(HDD_ERR_INVALID_ARGUMENT, "iomode output/input needs a directory");
        v.iomode = iomode;
        v.io_dir = directory ? directory : "";
    });
}

hdd_status hdd_multiply_dense(hdd_solver* s, const float* x, float* y) {
    if (!x || !y) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) { v.multiply_dense(x, y); });
}

hdd_status hdd_multiply_dot_dense_device_noalloc(hdd_solver* s, const float* x, float* y, double* dot,
                                                 void* stream) {
    if (!x || !y || !dot) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        if (!v.initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
        // The caller's thread may be working on another device: switch for
        // the launch and switch back on every exit path.
        DeviceGuard dg(v.opts.device);
        hdd::multiply_dot_dense_device_noalloc(v.geom(), v.tile_xyz.p, v.L.opt.size, v.opts.device, x, y, dot,
                                               static_cast<cudaStream_t>(stream));
        v.count(v.w0, 2);
    });
}

hdd_status hdd_sigma_vcycle(hdd_solver* s, const float* b0, float* u0) {
    if (!b0 || !u0) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) { v.sigma_vcycle_host(b0, u0); });
}

hdd_status hdd_interface_solve_batch(hdd_solver* s, int kind, int level, int nrhs, const float* b, float* x, int* n) {
    if (!n || (kind != 0 && kind != 1)) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) { v.interface_solve_batch(kind, level, nrhs, b, x, n); });
}

hdd_status hdd_interface_solve(hdd_solver* s, int kind, int level, const float* b, float* x, int* n) {
    if (!n || (kind != 0 && kind != 1)) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) { v.interface_solve(kind, level, b, x, n); });
}

hdd_status hdd_interface_size(hdd_solver* s, int level, int* n) {
    if (!n) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        if (!v.initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
        if (level < 0 || level >= v.ih.M) throw Error(HDD_ERR_INVALID_ARGUMENT, "level out of range");
        *n = v.ih.n_iface[level];
    });
}

hdd_status hdd_interface_map(hdd_solver* s, int* cells) {
    if (!cells) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        if (!v.initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
        for (size_t i = 0; i < v.ih.iface_map.size(); ++i)
            for (int a = 0; a < 3; ++a) cells[3 * i + a] = v.ih.iface_map[i][a];
    });
}

hdd_status hdd_interface_matrix(hdd_solver* s, int kind, int level, int sub, int* rows, int* cols, int* nnz, int* ptr,
                                int* col, double* val) {
    return guard(s, [&](Solver& v) {
        if (!v.initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
        const hdd::InterfaceHost& ih = v.ih;
        if (level < 0 || level >= ih.M) throw Error(HDD_ERR_INVALID_ARGUMENT, "level out of range");
        const hdd::CsrF* m = nullptr;
        if (kind == 0) m = &ih.Arr[level];
        else if (kind == 1 || kind == 2) {
            if (sub < 0 || sub >= ih.n_sub) throw Error(HDD_ERR_INVALID_ARGUMENT, "subdomain out of range");
            m = kind == 1 ? &ih.Aii[level][sub] : &ih.Air[level][sub];
        } else if (kind == 3) {
            if (level >= ih.M - 1) throw Error(HDD_ERR_INVALID_ARGUMENT, "no Prr at the coarsest level");
            m = &ih.Prr[level];
        } else throw Error(HDD_ERR_INVALID_ARGUMENT, "kind must be 0..3");
        if (rows) *rows = m->rows;
        if (cols) *cols = m->cols;
        if (nnz) *nnz = (int)m->col.size();
        if (ptr) std::memcpy(ptr, m->ptr.data(), m->ptr.size() * sizeof(int));
        if (col) std::memcpy(col, m->col.data(), m->col.size() * sizeof(int));
        if (val)
            for (size_t i = 0; i < m->val.size(); ++i) val[i] = m->val[i];
    });
}

hdd_status hdd_set_kernel_timing(hdd_solver* s, int enable) {
    return guard(s, [&](Solver& v) {
        v.collect_timing();
        v.timing = enable != 0;
        for (int c = 0; c < Solver::kCats; ++c) { v.cat_ms[c] = 0; v.cat_n[c] = 0; v.cat_bytes[c] = 0; }
    });
}

hdd_status hdd_get_kernel_timing(hdd_solver* s, double* ms, long long* launches) {
    if (!ms || !launches) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        v.collect_timing();
        for (int c = 0; c < Solver::kCats; ++c) { ms[c] = v.cat_ms[c]; launches[c] = v.cat_n[c]; }
    });
}

hdd_status hdd_get_kernel_bytes(hdd_solver* s, double* bytes) {
    if (!bytes) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        v.collect_timing();
        for (int c = 0; c < Solver::kCats; ++c) bytes[c] = v.cat_bytes[c];
    });
}

hdd_status hdd_set_wait_limit(hdd_solver* s, long long polls) {
    if (polls < 1) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        if (!v.initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
        v.sync();
        v.release_graphs();  // the limit is a launch parameter of the captured solves
        v.sigma.set_wait_limit(polls);
        v.sigma2.set_wait_limit(polls);
    });
}

hdd_status hdd_test_stall_dependency(hdd_solver* s, int on) {
    return guard(s, [&](Solver& v) {
        if (!v.initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
        hdd::cuda_check(cudaSetDevice(v.opts.device), "cudaSetDevice");
        v.sigma.stall_dependency(on != 0, v.stream);
    });
}

hdd_status hdd_get_pcg_coefficients(hdd_solver* s, double* alpha, double* beta, int capacity, int* n) {
    if (!n || capacity < 0 || (capacity > 0 && (!alpha || !beta))) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) {
        if (!v.w0.solved) throw Error(HDD_ERR_NOT_INITIALIZED, "no solve has run");
        *n = (int)v.w0.alphas.size();
        for (int i = 0; i < capacity && i < *n; ++i) { alpha[i] = v.w0.alphas[i]; beta[i] = v.w0.betas[i]; }
    });
}

hdd_status hdd_kernel_launch_count(hdd_solver* s, long long* count) {
    if (!count) return HDD_ERR_INVALID_ARGUMENT;
    return guard(s, [&](Solver& v) { *count = v.w0.launches; });
}

const char* hdd_status_string(hdd_status st) {
    switch (st) {
        case HDD_OK: return "ok";
        case HDD_ERR_INVALID_ARGUMENT: return "invalid argument";
        case HDD_ERR_CUDA: return "CUDA error";
        case HDD_ERR_OUT_OF_MEMORY: return "out of memory";
        case HDD_ERR_NOT_INITIALIZED: return "not initialized";
        case HDD_ERR_UNSUPPORTED: return "unsupported input";
        case HDD_ERR_NOT_CONVERGED: return "not converged";
        case HDD_ERR_BREAKDOWN: return "PCG breakdown";
        case HDD_ERR_TIMEOUT: return "device wait timed out";
        case HDD_ERR_IO: return "I/O error";
        case HDD_ERR_BUSY: return "busy";
        case HDD_ERR_NOT_FOUND: return "not found";
        case HDD_ERR_INTERNAL: return "internal error";
    }
    return "unknown status";
}

const char* hdd_last_error(const hdd_solver* s) { return s ? s->err.c_str() : "null handle"; }

void hdd_destroy(hdd_solver* s) {
    if (!s) return;
    delete s->impl;
    delete s;
}

}  // extern "C"
