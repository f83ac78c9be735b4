// Solver orchestration: host setup, device residency and the PCG loop.
//
// PCG follows PB/Public_Library/PhysBAM_Tools/Krylov_Solvers/CONJUGATE_GRADIENT.cpp:22-67
// with KRYLOV_SYSTEM_BASE::Precondition (Apply_Preconditioner then Project) and
// the preconditioner of
// CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Preconditioner.h:88-128:
//   pass 1: z_i = V-cycles(r) with interface values 0          (vcycle kernel)
//   b_G    = r_G - A_Gi z_i                                      (interface gather, Laplace_ri)
//   u_G    = sigma V-cycle(b_G)                                  (sigma.cu)
//   pass 2: z_G = u_G, z_i = V-cycles(r) with z_G as boundary     (scatter + vcycle kernel)
// All vectors stay resident in HBM in the tile layout; scalars live on the
// device and only max|r| (and a status word) return to the host per iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cerrno>
#include <cstring>

#include <sys/stat.h>

#include "solver.h"

namespace hdd {

static Options to_options(const hdd_options& o) {
    Options p;
    // Two-level DD runs its V-cycles on boxes of sub_size/2
    // (TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Solver.h:129-145).
    for (int a = 0; a < 3; ++a) { p.size[a] = o.size[a]; p.sub[a] = o.multilevel ? o.sub_size[a] / 2 : o.sub_size[a]; }
    p.vlevels = o.vlevels;
    p.nvcycles = o.nVcycles;
    p.interior = o.interior_smoothing;
    p.boundary = o.boundary_smoothing;
    p.sigma_levels = o.sigma_levels;
    p.sigma_smoothing = o.sigma_smoothing;
    p.sigma_mg = o.sigma_mg;
    return p;
}

Solver::Solver(const hdd_options& o) : opts(o) {
    hook.s = this;
    for (int a = 0; a < 3; ++a)
        if (o.size[a] < 3 || o.sub_size[a] < 1) throw Error(HDD_ERR_INVALID_ARGUMENT, "invalid size or sub_size");
    if (o.sub_size[0] != o.sub_size[1] || o.sub_size[0] != o.sub_size[2])
        throw Error(HDD_ERR_UNSUPPORTED, "sub_size must be equal on all axes");
    if (o.vlevels < 1 || o.vlevels > kMaxLevels) throw Error(HDD_ERR_INVALID_ARGUMENT, "vlevels out of range");
    if (o.solve_share < 0 || o.solve_share > 64) throw Error(HDD_ERR_INVALID_ARGUMENT, "solve_share out of range");
    if (o.coarse_solve != HDD_COARSE_REFERENCE && o.coarse_solve != HDD_COARSE_EXACT)
        throw Error(HDD_ERR_INVALID_ARGUMENT, "coarse_solve must be HDD_COARSE_REFERENCE or HDD_COARSE_EXACT");
    if (o.multilevel != 0 && o.multilevel != 1) throw Error(HDD_ERR_INVALID_ARGUMENT, "multilevel must be 0 or 1");
    if (o.multilevel && o.sub_size[0] % 2 != 0)
        throw Error(HDD_ERR_INVALID_ARGUMENT, "two-level DD needs an even sub_size");  // the demo's PHYSBAM_ASSERT
    if (o.multilevel && o.sub_size[0] != 16 && o.sub_size[0] != 32 && o.sub_size[0] != 64)
        throw Error(HDD_ERR_UNSUPPORTED, "two-level DD runs its V-cycles on boxes of sub_size/2: sub_size must be "
                                         "16, 32 or 64 (got " + std::to_string(o.sub_size[0]) + ")");
    if (o.sigma_levels < 1 || o.nVcycles < 0 || o.sigma_mg < 0 || o.interior_smoothing < 0 ||
        o.boundary_smoothing < 0 || o.sigma_smoothing < 0)
        throw Error(HDD_ERR_INVALID_ARGUMENT, "negative iteration counts");
    int ndev = 0;
    cuda_check(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (o.device < 0 || o.device >= ndev) throw Error(HDD_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    cuda_check(cudaSetDevice(o.device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&w0.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    w0.own_stream = true;
}

Solver::~Solver() {
    if (stream) {
        cudaStreamSynchronize(stream);
        release_graphs();
        sigma.release();
        sigma2.release();
    }
}

Work::~Work() {
    if (!stream) return;
    cudaStreamSynchronize(stream);
    release_graphs();
    if (own_sig) SigmaGpu::free_scratch(sig);
    if (own_sig2) SigmaGpu::free_scratch(sig2);
    if (own_stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

void Work::release_graphs() {
    if (pc_exec) cudaGraphExecDestroy(pc_exec);
    pc_exec = nullptr;
    pc_r = nullptr;
    pc_z = nullptr;
    pc_launches = 0;
}

void Solver::collect_timing() {
    if (pending.empty()) return;
    cuda_check(cudaStreamSynchronize(stream), "timing sync");
    for (auto& p : pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        cat_ms[p.cat] += ms;
        cat_n[p.cat] += 1;
        cat_bytes[p.cat] += p.bytes;
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    pending.clear();
}

void Solver::set_domain(const uint32_t* flags, const float* rhs) {
    const size_t n = (size_t)opts.size[0] * opts.size[1] * opts.size[2];
    flags_in.assign(flags, flags + n);
    rhs_dense.assign(rhs, rhs + n);
    have_domain = true;
    initialized = false;
    w0.solved = false;
}

void Solver::set_domain(std::vector<uint32_t>&& flags, std::vector<float>&& rhs) {
    const size_t n = (size_t)opts.size[0] * opts.size[1] * opts.size[2];
    if (flags.size() != n || rhs.size() != n) throw Error(HDD_ERR_INTERNAL, "dense domain arrays of the wrong size");
    flags_in = std::move(flags);
    rhs_dense = std::move(rhs);
    have_domain = true;
    initialized = false;
    w0.solved = false;
}

TileGeom Solver::geom() const {
    TileGeom g;
    g.sub = L.opt.sub[0];
    g.ntiles = (int)L.tiles.size();
    g.nbr = tile_nbr.p;
    g.flags = tflags.p;
    return g;
}

void Solver::initialize() {
    if (!have_domain) throw Error(HDD_ERR_NOT_INITIALIZED, "no domain set");
    release_graphs();
    NvtxRange range("Initialize_Preconditioner");
    cuda_check(cudaSetDevice(opts.device), "cudaSetDevice");
    const auto t0 = std::chrono::steady_clock::now();
    build_layout(to_options(opts), flags_in.data(), L);
    const int S = L.opt.sub[0];
    const size_t nt = L.tiles.size(), tc = (size_t)L.tile_cells, N = nt * tc;
    // Tile neighbour table (-x,+x,-y,+y,-z,+z).
    std::vector<int> nbr(nt * 6, -1);
    for (size_t t = 0; t < nt; ++t) {
        const auto& c = L.tiles[t];
        const int d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
        for (int q = 0; q < 6; ++q) {
            const int a = c[0] + d[q][0], b = c[1] + d[q][1], e = c[2] + d[q][2];
            if (a < 0 || b < 0 || e < 0 || a >= L.nt[0] || b >= L.nt[1] || e >= L.nt[2]) continue;
            nbr[6 * t + q] = L.tile_of[((size_t)a * L.nt[1] + b) * L.nt[2] + e];
        }
    }
    tile_nbr.upload(nbr.data(), nbr.size(), stream);
    {
        std::vector<int> txyz(3 * nt);
        for (size_t t = 0; t < nt; ++t)
            for (int a = 0; a < 3; ++a) txyz[3 * t + a] = L.tiles[t][a];
        tile_xyz.upload(txyz.data(), txyz.size(), stream);
    }
    tflags.upload(L.tile_flags.data(), L.tile_flags.size(), stream);
    {
        // Algorithmic HBM bytes of one launch: the Laplacian reads s (4 B)
        // and the flags (2 B) and writes q (4 B) once per stored tile cell,
        // the storage unit of the tiled vectors (10 B); the V-cycle reads u,
        // b and the level-0 flags and writes u once per box cell (13 B).
        const double sub3 = (double)L.opt.sub[0] * L.opt.sub[0] * L.opt.sub[0];
        laplace_bytes = 10.0 * sub3 * (double)L.tiles.size();
        vcycle_bytes = 13.0 * sub3 * (double)L.boxes.size();
    }
    std::vector<int> btile(L.boxes.size()), bnb(3 * L.boxes.size());
    for (size_t i = 0; i < L.boxes.size(); ++i) {
        btile[i] = L.boxes[i].tile;
        for (int q = 0; q < 3; ++q) bnb[3 * i + q] = L.boxes[i].nb_tile[q];
    }
    box_tile.upload(btile.data(), btile.size(), stream);
    box_nb.upload(bnb.data(), bnb.size(), stream);
    box_flags.upload(L.box_flags.data(), L.box_flags.size(), stream);
    for (int l = 0; l < kMaxLevels; ++l) {
        if (L.global_vcycle && l < L.opt.vlevels) gflags[l].upload(L.g_flags[l].data(), L.g_flags[l].size(), stream);
        else gflags[l].release();
    }
    alloc_vectors(w0);
    (void)S;
    (void)N;

    // Interface system (host assembly + factorisations) and its device solver.
    auto since_ms = [&](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
    };
    setup_phase_ms[0] = since_ms(t0);
    const auto t_iface = std::chrono::steady_clock::now();
    if (std::getenv("HDD_VERBOSE"))
        std::fprintf(stderr, "[hdd setup] layout %.2f s (%zu tiles, %zu boxes)\n",
                     std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(), L.tiles.size(),
                     L.boxes.size());
    if (opts.multilevel) {
        if (iomode != HDD_IOMODE_NEITHER)
            throw Error(HDD_ERR_UNSUPPORTED, "interface dump and reload are not implemented for two-level DD");
        build_two_level_interfaces();
    } else if (iomode == HDD_IOMODE_INPUT) {
        read_interface_dir(io_dir, ih);
        check_interface(L, opts.sigma_levels, ih);
    } else {
        build_interface(L, opts.sigma_levels, ih);
    }
    if (iomode == HDD_IOMODE_OUTPUT) {
        if (::mkdir(io_dir.c_str(), 0777) != 0 && errno != EEXIST)
            throw Error(HDD_ERR_IO, "cannot create " + io_dir + ": " + std::strerror(errno));
        write_interface_dir(ih, io_dir);
    }
    if (std::getenv("HDD_VERBOSE"))
        std::fprintf(stderr, "[hdd setup] interface assembly done at %.2f s\n",
                     std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    // Level-0 interface DOFs: cell slots and their Active face neighbours.
    const int n_if = ih.n_iface.empty() ? 0 : ih.n_iface[0];
    setup_phase_ms[1] = since_ms(t_iface);
    const auto t_sigma = std::chrono::steady_clock::now();
    // A domain inside one subdomain has no interface: the preconditioner is
    // then the two subdomain V-cycle passes alone, and the coarser interface
    // levels (which only feed level 0) are not built.
    if (n_if > 0) sigma.setup(ih, opts.sigma_smoothing, stream, opts.coarse_solve == HDD_COARSE_EXACT);
    else sigma.release();
    setup_phase_ms[2] = since_ms(t_sigma);
    // Interface cells' slots and, per cell, the slots of the face neighbours
    // that one gather reads (-1 for the others).  A neighbour counts when the
    // cell's face bit is set and keep(neighbour flags, neighbour on a
    // first-level plane) holds.  Single level: Laplace_ri's Active neighbours
    // (SPGrid_Laplace_Legacy.h:70-117).
    const int* n = L.opt.size;
    const int* s1 = opts.sub_size;
    auto on_plane1 = [&](int a, int b, int c) { return a % s1[0] == 0 || b % s1[1] == 0 || c % s1[2] == 0; };
    auto tables = [&](const InterfaceHost& h, std::vector<long long>& slot, std::vector<int>& nbs, auto keep) {
        const int m = h.n_iface.empty() ? 0 : h.n_iface[0];
        const int d6[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
        slot.assign(m, 0);
        nbs.assign(6 * (size_t)m, -1);
        for (int i = 0; i < m; ++i) {
            const auto& c = h.iface_map[i];
            slot[i] = L.tile_slot(c[0], c[1], c[2]);
            const uint32_t f = L.flags0[L.dense_index(c[0], c[1], c[2])];
            if (slot[i] < 0 || !(f & F_INTERFACE)) throw Error(HDD_ERR_INTERNAL, "interface DOF outside the tile layout");
            for (int qf = 0; qf < 6; ++qf) {
                if (!(f & (F_FACE_MX << qf))) continue;
                const int a = c[0] + d6[qf][0], bb = c[1] + d6[qf][1], e = c[2] + d6[qf][2];
                if (a < 0 || bb < 0 || e < 0 || a >= n[0] || bb >= n[1] || e >= n[2]) continue;
                if (!keep(L.flags0[L.dense_index(a, bb, e)], on_plane1(a, bb, e))) continue;
                const long long sl = L.tile_slot(a, bb, e);
                if (sl < 0) throw Error(HDD_ERR_INTERNAL, "interface neighbour outside the tile layout");
                if (sl > INT32_MAX) throw Error(HDD_ERR_UNSUPPORTED, "domain too large for 32-bit neighbour slots");
                nbs[6 * (size_t)i + qf] = (int)sl;
            }
        }
    };
    std::vector<long long> slot;
    std::vector<int> nbs;
    if (!opts.multilevel) {
        tables(ih, slot, nbs, [](uint32_t f, bool) { return (f & F_ACTIVE) != 0; });
    } else {
        // First level: Laplace_ri_Subdomain, the Active|Interface neighbours
        // off the first-level planes (TWO/SPGrid_Library/SPGrid_Laplace_Legacy.h:120-178).
        tables(ih, slot, nbs, [](uint32_t f, bool p1) { return (f & (F_ACTIVE | F_INTERFACE)) && !p1; });
        // Second level: Laplace_ir_Subdomain's neighbours on the first-level
        // planes (:232-290) and Laplace_ri's Active neighbours (:70-117).
        std::vector<long long> slot2, slot2b;
        std::vector<int> nb_ir, nb_ri;
        tables(ih2, slot2, nb_ir, [](uint32_t f, bool p1) { return (f & (F_ACTIVE | F_INTERFACE)) && p1; });
        tables(ih2, slot2b, nb_ri, [](uint32_t f, bool) { return (f & F_ACTIVE) != 0; });
        // Laplace_ir_Subdomain's box-face cells (the V-cycle's face residual):
        // Interface cells off the first-level planes with an open face to an
        // Active|Interface cell on them.
        std::vector<long long> fslot;
        std::vector<int> fnb;
        const int d6[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
        for (int i = 0; i < n[0]; ++i)
            for (int j = 0; j < n[1]; ++j)
                for (int k = 0; k < n[2]; ++k) {
                    const uint32_t f = L.flags0[L.dense_index(i, j, k)];
                    if (!(f & F_INTERFACE) || on_plane1(i, j, k)) continue;
                    int nb6[6] = {-1, -1, -1, -1, -1, -1};
                    bool any = false;
                    for (int qf = 0; qf < 6; ++qf) {
                        if (!(f & (F_FACE_MX << qf))) continue;
                        const int a = i + d6[qf][0], bb = j + d6[qf][1], e = k + d6[qf][2];
                        if (a < 0 || bb < 0 || e < 0 || a >= n[0] || bb >= n[1] || e >= n[2]) continue;
                        if (!(L.flags0[L.dense_index(a, bb, e)] & (F_ACTIVE | F_INTERFACE)) || !on_plane1(a, bb, e))
                            continue;
                        const long long sl = L.tile_slot(a, bb, e);
                        if (sl < 0 || sl > INT32_MAX) throw Error(HDD_ERR_INTERNAL, "face neighbour outside the tile layout");
                        nb6[qf] = (int)sl;
                        any = true;
                    }
                    if (!any) continue;
                    const long long sc = L.tile_slot(i, j, k);
                    if (sc < 0) throw Error(HDD_ERR_INTERNAL, "face cell outside the tile layout");
                    fslot.push_back(sc);
                    fnb.insert(fnb.end(), nb6, nb6 + 6);
                }
        n_face = (int)fslot.size();
        face_slot.upload(fslot.data(), fslot.size(), stream);
        face_nb.upload(fnb.data(), fnb.size(), stream);
        iface2_slot.upload(slot2.data(), slot2.size(), stream);
        iface2_nb_ir.upload(nb_ir.data(), nb_ir.size(), stream);
        iface2_nb_ri.upload(nb_ri.data(), nb_ri.size(), stream);
        const int n2 = ih2.n_iface.empty() ? 0 : ih2.n_iface[0];
        if (n2 > 0) sigma2.setup(ih2, opts.sigma_smoothing, stream, opts.coarse_solve == HDD_COARSE_EXACT);
        else sigma2.release();
        w0.sig2 = sigma2.primary();
        w0.sig2.set_grid_div(std::max(1, opts.solve_share));
        w0.own_sig2 = false;
    }
    iface_slot.upload(slot.data(), slot.size(), stream);
    iface_nb.upload(nbs.data(), nbs.size(), stream);
    w0.sig = sigma.primary();
    w0.sig.set_grid_div(std::max(1, opts.solve_share));
    w0.own_sig = false;
    set_rhs(rhs_dense.data());
    sync();
    initialized = true;
    setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    setup_phase_ms[3] = setup_ms;
}

void Solver::alloc_vectors(Work& w) {
    const size_t nt = L.tiles.size(), N = std::max<size_t>(nt * (size_t)L.tile_cells, 1);
    const size_t P = std::max<size_t>({nt, (size_t)laplace_partials(geom()), (size_t)1});
    const size_t k = (size_t)w.k;
    w.vstride = N;
    w.pstride = (int)P;
    w.dense.alloc(std::max<size_t>(L.cell_count(), 1));
    for (DevBuf<float>* v : {&w.x, &w.b, &w.r, &w.z, &w.s, &w.q}) { v->alloc(N * k); v->zero(w.stream); }
    if (opts.precision_mode == HDD_PRECISION_MIXED) w.xd.alloc(N * k);
    else w.xd.release();
    if (opts.multilevel) w.hr.alloc(N * k);
    else w.hr.release();
    for (int l = 0; l < kMaxLevels; ++l) {
        const bool on = L.global_vcycle && l < L.opt.vlevels;
        const size_t c = on ? (size_t)L.g_dims[l][0] * L.g_dims[l][1] * L.g_dims[l][2] : 0;
        for (DevBuf<float>* v : {&w.gu[l], &w.gb[l], &w.gr[l]}) {
            if (on) { v->alloc(c); v->zero(w.stream); }
            else v->release();
        }
    }
    w.partial.alloc(P * k);
    w.partial_max.alloc(P * k);
    w.sums.alloc(8 * k);
    w.scalars_f.alloc(8 * k);
    w.scal.alloc(k);
    if (w.k > 1) {
        for (DevBuf<int>* v : {&w.active, &w.first, &w.replace}) { v->alloc(k); v->zero(w.stream); }
    }
}

int Solver::max_batch() const {
    if (!initialized || opts.multilevel || L.global_vcycle) return 1;
    return sigma.lv.empty() ? 4 : sigma.max_rhs();
}

std::unique_ptr<Work> Solver::make_work(int k) {
    if (!initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
    if (k != 1 && k != 2 && k != 4) throw Error(HDD_ERR_INVALID_ARGUMENT, "systems per context: 1, 2 or 4");
    if (k > max_batch()) throw Error(HDD_ERR_UNSUPPORTED, "the interface solver's fronts leave no room for that batch");
    std::unique_ptr<Work> w(new Work());
    w->k = k;
    cuda_check(cudaSetDevice(opts.device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    w->own_stream = true;
    alloc_vectors(*w);
    if (!sigma.lv.empty()) {
        sigma.alloc_scratch(w->sig, w->stream, k);
        w->sig.set_grid_div(std::max(1, opts.solve_share));
        w->own_sig = true;
    }
    if (!sigma2.lv.empty()) {
        sigma2.alloc_scratch(w->sig2, w->stream, k);
        w->sig2.set_grid_div(std::max(1, opts.solve_share));
        w->own_sig2 = true;
    }
    sync(*w);
    return w;
}

size_t Solver::work_bytes(int k) const {
    const size_t nt = L.tiles.size(), N = nt * (size_t)L.tile_cells;
    const size_t P = std::max<size_t>({nt, (size_t)laplace_partials(geom()), (size_t)1});
    size_t t = std::max<size_t>(L.cell_count(), 1) * 4 + (opts.multilevel ? 7 : 6) * std::max<size_t>(N, 1) * 4 * k;
    if (opts.precision_mode == HDD_PRECISION_MIXED) t += std::max<size_t>(N, 1) * 8 * k;
    t += (P * 12 + 128 + sizeof(PcgScalars) + 12) * k;
    if (L.global_vcycle)
        for (int l = 0; l < L.opt.vlevels; ++l) t += 12 * (size_t)L.g_dims[l][0] * L.g_dims[l][1] * L.g_dims[l][2];
    return t + sigma.scratch_bytes(k) + (sigma2.lv.empty() ? 0 : sigma2.scratch_bytes(k));
}

void Solver::set_rhs(Work& w, const float* rhs) {
    // H2D of the dense right-hand side, then a device gather into the tiles.
    if (&w == &w0 && rhs != rhs_dense.data()) rhs_dense.clear();
    Tm tm(this, w, 5);
    cuda_check(cudaMemcpyAsync(w.dense.p, rhs, L.cell_count() * sizeof(float), cudaMemcpyHostToDevice, w.stream),
               "H2D rhs");
    cuda_check(launch_dense_to_tiles(geom(), tile_xyz.p, L.opt.size[0], L.opt.size[1], L.opt.size[2], w.dense.p,
                                     w.b.p, w.stream), "dense_to_tiles");
    count(w);
    sync(w);
}

VcycleArgs Solver::vcycle_args(float* u, const float* bb, int halo_from_u, int zero_init, int nv) const {
    VcycleArgs a;
    std::memset(&a, 0, sizeof(a));
    a.u = u;
    a.b = bb;
    a.box_flags = box_flags.p;
    a.box_tile = box_tile.p;
    a.box_nb = box_nb.p;
    a.nbox = (int)L.boxes.size();
    a.sub = L.opt.sub[0];
    a.levels = L.opt.vlevels;
    a.box_stride = L.box_stride;
    for (int l = 0; l < L.opt.vlevels; ++l) a.level_off[l] = L.level_off[l];
    a.n_vcycles = nv;
    a.interior_itr = L.opt.interior;
    a.boundary_itr = L.opt.boundary;
    a.bottom_itr = 200;  // CPU/SPGrid_Library/SPGrid_V_Cycle_Helper.h:179
    a.halo_from_u = halo_from_u;
    a.zero_init = zero_init;
    a.cluster = 1;
    a.nslots = 1;
    a.slot_stride = 0;
    a.active = nullptr;
    if (const char* e = std::getenv("HDD_VCYCLE_CLUSTER")) a.cluster = std::atoi(e);
    // Correction weights omega/face_count with omega = (float)(2/3)
    // (SPGrid_Correction_Legacy.h:35,76), divided in float on the host.
    const float omega = (float)(2. / 3.);
    a.inv_diag[0] = 0.0f;
    for (int k = 1; k < 8; ++k) a.inv_diag[k] = omega / (float)k;
    // Restriction tensor weights (SPGrid_Restriction_Legacy.h:49-57).
    const float s1[4] = {(float)(1. / 8.), (float)(3. / 8.), (float)(3. / 8.), (float)(1. / 8.)};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 4; ++k) a.restrict_w[(i * 4 + j) * 4 + k] = s1[i] * s1[j] * s1[k];
    // Prolongation tensor weights (SPGrid_Prolongation_Legacy.h:48-53).
    const float p1[2] = {(float)(3. / 4.f), (float)(1. / 4.f)};
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int k = 0; k < 2; ++k) a.prolong_w[(i * 2 + j) * 2 + k] = p1[i] * p1[j] * p1[k] * 4.0f;
    return a;
}

void Solver::run_vcycle(Work& w, float* u, const float* bb, int halo_from_u, int zero_init, int nv,
                        const float* r_halo) {
    VcycleArgs a = vcycle_args(u, bb, halo_from_u, zero_init, nv);
    a.r_halo = r_halo;
    if (L.global_vcycle) {
        // Coarse levels couple the boxes: the whole-grid V-cycle (one system).
        if (w.k > 1) throw Error(HDD_ERR_INTERNAL, "whole-grid V-cycle with a batched context");
        GlobalVcycleArgs ga;
        std::memset(&ga, 0, sizeof(ga));
        ga.levels = L.opt.vlevels;
        for (int l = 0; l < ga.levels; ++l) {
            for (int q = 0; q < 3; ++q) ga.dims[l][q] = L.g_dims[l][q];
            ga.f[l] = gflags[l].p;
            ga.u[l] = w.gu[l].p;
            ga.b[l] = w.gb[l].p;
            ga.r[l] = w.gr[l].p;
        }
        ga.n_vcycles = nv;
        ga.interior_itr = a.interior_itr;
        ga.boundary_itr = a.boundary_itr;
        ga.bottom_itr = a.bottom_itr;
        ga.halo_from_u = halo_from_u;
        ga.zero_init = zero_init;
        std::memcpy(ga.w.inv_diag, a.inv_diag, sizeof(a.inv_diag));
        std::memcpy(ga.w.restrict_w, a.restrict_w, sizeof(a.restrict_w));
        std::memcpy(ga.w.prolong_w, a.prolong_w, sizeof(a.prolong_w));
        Tm tm(this, w, 0, vcycle_bytes);
        w.launches += launch_vcycle_global(ga, geom(), tile_xyz.p, u, bb, r_halo, w.stream);
        return;
    }
    if (w.k > 1) {
        a.nslots = w.k;
        a.slot_stride = w.vstride;
        a.active = w.active.p;
    }
    Tm tm(this, w, 0, vcycle_bytes);
    cuda_check(launch_vcycle(a, w.stream), "vcycle kernel");
    count(w);
}

void Solver::apply_preconditioner(Work& w, const float* rr, float* zz) {
    // One application is a fixed sequence of launches on fixed buffers (for a
    // 32^3-subdomain domain whose coarsest interface level runs the 200
    // smoothing steps, well over a thousand): it is captured once as a CUDA
    // graph and replayed, so the host issues one launch per application.
    // Per-phase timing needs events between the launches and runs them
    // directly; a failed capture falls back to direct launches for good.
    if (w.use_graphs && !timing) {
        if (w.pc_exec && w.pc_r == rr && w.pc_z == zz) {
            cuda_check(cudaGraphLaunch(w.pc_exec, w.stream), "cudaGraphLaunch");
            w.launches += w.pc_launches;
            return;
        }
        w.release_graphs();
        cudaGraph_t graph = nullptr;
        const long long before = w.launches;
        if (cudaStreamBeginCapture(w.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            bool ok = true;
            try {
                apply_preconditioner_launches(w, rr, zz);
            } catch (const Error&) {
                ok = false;
            }
            const cudaError_t e = cudaStreamEndCapture(w.stream, &graph);
            if (ok && e == cudaSuccess && graph &&
                cudaGraphInstantiate(&w.pc_exec, graph, 0) == cudaSuccess) {
                cudaGraphDestroy(graph);
                w.pc_r = rr;
                w.pc_z = zz;
                w.pc_launches = w.launches - before;
                w.launches = before;
                cuda_check(cudaGraphLaunch(w.pc_exec, w.stream), "cudaGraphLaunch");
                w.launches += w.pc_launches;
                return;
            }
            if (graph) cudaGraphDestroy(graph);
            w.pc_exec = nullptr;
            cudaGetLastError();  // clear a capture error; run the launches directly from now on
        }
        w.launches = before;
        w.use_graphs = false;
    }
    apply_preconditioner_launches(w, rr, zz);
}

void Solver::apply_preconditioner_launches(Work& w, const float* rr, float* zz) {
    if (opts.multilevel) {
        two_level_launches(w, rr, zz);
        return;
    }
    NvtxRange range("Apply_Preconditioner");
    const TileGeom g = geom();
    {
        NvtxRange step("Step ONE");
        run_vcycle(w, zz, rr, 0, 1, opts.nVcycles);
    }
    const int n_if = ih.n_iface.empty() ? 0 : ih.n_iface[0];
    {
        Tm tm(this, w, 3);
        const size_t is = w.sig.lv.empty() ? 0 : w.sig.lv[0].si;
        cuda_check(launch_interface_gather(g, iface_slot.p, iface_nb.p, n_if, rr, zz, w.sig.b0(), w.stream, w.batch(),
                                           is),
                   "gather");
        count(w);
    }
    if (n_if > 0) {
        // u_G = 0 then sigma_mg V-cycles (Preconditioner.h:105,110-117).
        NvtxRange sigma_range("Sigma_V_Cycle");
        Tm tm(this, w, 4);
        cuda_check(cudaMemsetAsync(w.sig.u0(), 0, sizeof(float) * w.sig.lv[0].si * w.k, w.stream), "memset u0");
        for (int i = 0; i < opts.sigma_mg; ++i) sigma.vcycle(w.sig, w.stream, w.launches, &w == &w0 ? &hook : nullptr);
    }
    {
        Tm tm(this, w, 3);
        const size_t is = w.sig.lv.empty() ? 0 : w.sig.lv[0].si;
        cuda_check(launch_interface_scatter(iface_slot.p, n_if, w.sig.u0(), zz, w.stream, w.batch(), is), "scatter");
        count(w);
    }
    NvtxRange step("Step Two");
    run_vcycle(w, zz, rr, 1, 1, opts.nVcycles);
}

void Solver::build_two_level_interfaces() {
    // Two-level DD (demos/Domain_Decomposition_CPU_Only_Two_Levels, "TWO/"):
    // the first-level interface system is assembled on boxes of sub_size from
    // the caller's flags (TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Subdomain_Splitter.h:53-160).
    // The second-level systems, one per first-level subdomain (:168-193),
    // are stacked into one block-diagonal system (build_second_level).
    DomainLayout Lf;
    Lf.opt = L.opt;
    for (int a = 0; a < 3; ++a) Lf.opt.sub[a] = opts.sub_size[a];
    Lf.flags_in = flags_in;
    build_interface(Lf, opts.sigma_levels, ih);
    build_second_level(Lf, opts.sub_size, opts.sigma_levels, ih2);
}

// Subdomain_DD (TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Preconditioner.h:127-181;
// its residual prints dropped): a DD solve inside every first-level
// subdomain, the first-level interface values in zz as its boundary data.
// On entry zz holds only first-level interface values (zero the first time).
//
// The reference computes Laplace_ir_Subdomain into its tmp channel and runs
// the first V-cycles on that channel without clearing it; its restriction
// reads the channel at the boxes' face cells, where the V-cycle computes no
// residual, so at the second-level interface cells it restricts those
// values.  They are zero on the first call (zz is zero) and are passed to the
// V-cycle as its face residual (hr) on the second, for the same result.
// (Every Active|Interface cell off the first-level planes gets a value; only
// those on box faces are read, and only those next to a first-level plane
// are nonzero: face_slot.)
void Solver::subdomain_dd(Work& w, const float* rr, float* zz, bool second) {
    const TileGeom g = geom();
    const int n2 = ih2.n_iface.empty() ? 0 : ih2.n_iface[0];
    const int n1 = ih.n_iface.empty() ? 0 : ih.n_iface[0];
    {
        // b2 = Laplace_ir_Subdomain(zz) at the second-level interface cells.
        Tm tm(this, w, 3);
        cuda_check(launch_interface_gather(g, iface2_slot.p, iface2_nb_ir.p, n2, rr, zz, w.sig2.b0(), w.stream,
                                           Batch(), 0, kGatherIr), "gather ir");
        count(w);
        if (second && n_face > 0) {
            cuda_check(cudaMemsetAsync(w.hr.p, 0, sizeof(float) * w.vstride, w.stream), "memset hr");
            cuda_check(launch_interface_gather(g, face_slot.p, face_nb.p, n_face, rr, zz, w.hr.p, w.stream, Batch(), 0,
                                               kGatherIrTiled), "gather ir faces");
            count(w);
        }
    }
    run_vcycle(w, zz, rr, 1, 1, opts.nVcycles, second && n_face > 0 ? w.hr.p : nullptr);
    if (n2 > 0) {
        {
            // b2 += rr - A_ri zz (Laplace_ri, then Accumulate_To_Eigen_Array).
            Tm tm(this, w, 3);
            cuda_check(launch_interface_gather(g, iface2_slot.p, iface2_nb_ri.p, n2, rr, zz, w.sig2.b0(), w.stream,
                                               Batch(), 0, kGatherRiAdd), "gather ri");
            count(w);
        }
        NvtxRange sigma_range("Sigma_V_Cycle (second level)");
        Tm tm(this, w, 4);
        cuda_check(cudaMemsetAsync(w.sig2.u0(), 0, sizeof(float) * w.sig2.lv[0].si, w.stream), "memset u2");
        for (int i = 0; i < opts.sigma_mg; ++i) sigma2.vcycle(w.sig2, w.stream, w.launches, &w == &w0 ? &hook : nullptr);
    }
    {
        // zz = 0, then the first- and second-level interface values.
        Tm tm(this, w, 3);
        cuda_check(cudaMemsetAsync(zz, 0, sizeof(float) * w.vstride, w.stream), "memset z");
        cuda_check(launch_interface_scatter(iface_slot.p, n1, w.sig.u0(), zz, w.stream), "scatter u1");
        cuda_check(launch_interface_scatter(iface2_slot.p, n2, w.sig2.u0(), zz, w.stream), "scatter u2");
        count(w, 2);
    }
    run_vcycle(w, zz, rr, 1, 1, opts.nVcycles);
}

// Apply_Preconditioner with multilevel
// (TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Preconditioner.h:182-230):
// Subdomain_DD in place of each V-cycle pass, the first-level interface
// right-hand side from Laplace_ri_Subdomain.
void Solver::two_level_launches(Work& w, const float* rr, float* zz) {
    NvtxRange range("Apply_Preconditioner (two-level)");
    const TileGeom g = geom();
    const int n1 = ih.n_iface.empty() ? 0 : ih.n_iface[0];
    cuda_check(cudaMemsetAsync(zz, 0, sizeof(float) * w.vstride, w.stream), "memset z");
    if (n1 > 0) cuda_check(cudaMemsetAsync(w.sig.u0(), 0, sizeof(float) * w.sig.lv[0].si, w.stream), "memset u1");
    subdomain_dd(w, rr, zz, false);
    if (n1 > 0) {
        {
            Tm tm(this, w, 3);
            cuda_check(launch_interface_gather(g, iface_slot.p, iface_nb.p, n1, rr, zz, w.sig.b0(), w.stream),
                       "gather ri_subdomain");
            count(w);
        }
        NvtxRange sigma_range("Sigma_V_Cycle");
        Tm tm(this, w, 4);
        cuda_check(cudaMemsetAsync(w.sig.u0(), 0, sizeof(float) * w.sig.lv[0].si, w.stream), "memset u1");
        for (int i = 0; i < opts.sigma_mg; ++i) sigma.vcycle(w.sig, w.stream, w.launches, &w == &w0 ? &hook : nullptr);
    }
    {
        Tm tm(this, w, 3);
        cuda_check(cudaMemsetAsync(zz, 0, sizeof(float) * w.vstride, w.stream), "memset z");
        cuda_check(launch_interface_scatter(iface_slot.p, n1, w.sig.u0(), zz, w.stream), "scatter u1");
        count(w);
    }
    subdomain_dd(w, rr, zz, true);
}

int Solver::wait_error(Work& w) {
    int e[2] = {0, 0};
    if (w.sig.err) cuda_check(cudaMemcpyAsync(&e[0], w.sig.err, sizeof(int), cudaMemcpyDeviceToHost, w.stream), "D2H");
    if (w.sig2.err) cuda_check(cudaMemcpyAsync(&e[1], w.sig2.err, sizeof(int), cudaMemcpyDeviceToHost, w.stream), "D2H");
    sync(w);
    return e[0] | e[1];
}

void Solver::clear_wait_errors(Work& w) {
    SigmaGpu::clear_error(w.sig, w.stream);
    if (w.sig2.err) SigmaGpu::clear_error(w.sig2, w.stream);
}

void Solver::solve(Work& w, hdd_result* res) {
    if (!initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
    NvtxRange range("solve");
    cuda_check(cudaSetDevice(opts.device), "cudaSetDevice");
    const TileGeom g = geom();
    const int nt = g.ntiles;
    const int mode = opts.precision_mode == HDD_PRECISION_MIXED ? 1 : 0;
    PcgScalars init;
    std::memset(&init, 0, sizeof(init));
    init.rho_old = 3.402823466e+38f;
    init.rho_old_d = 3.402823466e+38;
    cuda_check(cudaMemcpyAsync(w.scal.p, &init, sizeof(init), cudaMemcpyHostToDevice, w.stream), "init scalars");
    w.x.zero(w.stream);
    w.xd.zero(w.stream);
    double* xdp = mode == 1 ? w.xd.p : nullptr;
    clear_wait_errors(w);
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    cuda_check(cudaEventRecord(e0, w.stream), "event record");
    // r = Project(b - A x) with x = 0 (restart branch, CONJUGATE_GRADIENT.cpp:36).
    cuda_check(launch_residual(g, w.b.p, w.x.p, w.r.p, w.partial_max.p, w.stream), "residual"); count(w);
    cuda_check(launch_reduce_max(w.partial_max.p, nt, w.scalars_f.p, w.stream), "reduce"); count(w);
    float rmax = 0;
    PcgScalars hs;
    cuda_check(cudaMemcpyAsync(&rmax, w.scalars_f.p, sizeof(float), cudaMemcpyDeviceToHost, w.stream), "D2H");
    sync(w);
    const double b_inf = rmax;
    w.history.assign(1, (double)rmax);
    w.alphas.clear();
    w.betas.clear();
    const float threshold = opts.relative_tol ? (float)(opts.tol * b_inf) : (float)opts.tol;
    const float small_number = 1.1920929e-07f;
    int it = 0;
    bool converged = false, breakdown = false;
    // The precision form stops on its FP64 true residual: when the recursively
    // updated (FP32) residual reaches the tolerance, r is recomputed from the
    // FP64 iterate (residual replacement) and the loop goes on if the true
    // residual is still above it.  An FP32 recursive residual drifts from the
    // true one by about the FP32 rounding of the updates.
    // When that recomputed residual is still above the tolerance, it differs
    // from the recursive one by far more than the recursive one itself, and
    // the search directions built on the recursive residual no longer fit:
    // PCG restarts from x (s = z, the restart branch of
    // PB/Public_Library/PhysBAM_Tools/Krylov_Solvers/CONJUGATE_GRADIENT.cpp:30-36,47).
    bool replaced = false;  // r was recomputed from x in this iteration
    bool restart = false;   // the next iteration starts a new search direction
    for (;; ++it) {
        if (rmax <= threshold && (it >= opts.min_iters || rmax < small_number)) {
            if (mode != 1 || replaced) { converged = true; break; }
            cuda_check(launch_residual_f64(g, w.b.p, xdp, w.r.p, w.partial_max.p, w.stream), "true residual"); count(w);
            cuda_check(launch_reduce_max(w.partial_max.p, nt, w.scalars_f.p, w.stream), "reduce"); count(w);
            cuda_check(cudaMemcpyAsync(&rmax, w.scalars_f.p, sizeof(float), cudaMemcpyDeviceToHost, w.stream), "D2H");
            sync(w);
            w.history.back() = (double)rmax;
            replaced = true;
            if (rmax <= threshold) { converged = true; break; }
            restart = true;
        }
        if (it >= opts.max_iters) break;
        replaced = false;
        const int first = (it == 0 || restart) ? 1 : 0;
        restart = false;
        apply_preconditioner(w, w.r.p, w.z.p);
        {
            Tm tm(this, w, 2);
            cuda_check(launch_project_dot(g, w.z.p, w.r.p, w.partial.p, w.stream), "project_dot"); count(w);
            cuda_check(launch_reduce_sum(w.partial.p, nt, w.sums.p + 0, w.stream), "reduce"); count(w);
            cuda_check(launch_scalar_rho(w.scal.p, w.sums.p + 0, first, w.stream), "rho"); count(w);
            cuda_check(launch_update_s(g, w.s.p, w.z.p, w.scal.p, first, mode, w.stream), "update_s"); count(w);
        }
        {
            Tm tm(this, w, 1, laplace_bytes);
            cuda_check(launch_laplace_dot(g, w.s.p, w.q.p, w.partial.p, w.stream), "laplace"); count(w);
        }
        {
            Tm tm(this, w, 2);
            cuda_check(launch_reduce_sum(w.partial.p, laplace_partials(g), w.sums.p + 1, w.stream), "reduce"); count(w);
            cuda_check(launch_scalar_alpha(w.scal.p, w.sums.p + 1, w.stream), "alpha"); count(w);
            cuda_check(launch_update_xr(g, w.x.p, w.r.p, w.s.p, w.q.p, w.scal.p, mode, w.partial_max.p, w.stream, xdp), "update_xr");
            count(w);
        }
        if (mode == 1 && opts.true_residual_every > 0 && (it + 1) % opts.true_residual_every == 0) {
            cuda_check(launch_residual_f64(g, w.b.p, xdp, w.r.p, w.partial_max.p, w.stream), "true residual"); count(w);
            replaced = true;
        }
        cuda_check(launch_reduce_max(w.partial_max.p, nt, w.scalars_f.p, w.stream), "reduce"); count(w);
        cuda_check(cudaMemcpyAsync(&rmax, w.scalars_f.p, sizeof(float), cudaMemcpyDeviceToHost, w.stream), "D2H");
        cuda_check(cudaMemcpyAsync(&hs, w.scal.p, sizeof(hs), cudaMemcpyDeviceToHost, w.stream), "D2H");
        int herr = 0, herr2 = 0;
        if (w.sig.err)
            cuda_check(cudaMemcpyAsync(&herr, w.sig.err, sizeof(int), cudaMemcpyDeviceToHost, w.stream), "D2H");
        if (w.sig2.err)
            cuda_check(cudaMemcpyAsync(&herr2, w.sig2.err, sizeof(int), cudaMemcpyDeviceToHost, w.stream), "D2H");
        sync(w);
        herr |= herr2;
        w.history.push_back((double)rmax);
        w.alphas.push_back(mode == 1 ? hs.alpha_d : (double)hs.alpha);
        w.betas.push_back(first ? 0.0 : (mode == 1 ? hs.beta_d : (double)hs.beta));
        // A bounded wait that gave up leaves this iteration's preconditioner
        // invalid: stop here (check_waits below reports HDD_ERR_TIMEOUT).
        if (herr != 0) { ++it; break; }
        if (hs.status != 0 || !std::isfinite(rmax)) { breakdown = true; ++it; break; }
    }
    cuda_check(cudaEventRecord(e1, w.stream), "event record");
    cuda_check(cudaEventSynchronize(e1), "event sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // True residual of the returned iterate (reported, not used for stopping):
    // the FP64 iterate in the precision form, else x.
    if (xdp) cuda_check(launch_residual_f64(g, w.b.p, xdp, w.q.p, w.partial_max.p, w.stream), "true residual");
    else cuda_check(launch_residual(g, w.b.p, w.x.p, w.q.p, w.partial_max.p, w.stream), "true residual");
    count(w);
    cuda_check(launch_reduce_max(w.partial_max.p, nt, w.scalars_f.p + 1, w.stream), "reduce"); count(w);
    cuda_check(launch_project_dot(g, w.q.p, w.q.p, w.partial.p, w.stream), "dot"); count(w);
    cuda_check(launch_reduce_sum(w.partial.p, nt, w.sums.p + 2, w.stream), "reduce"); count(w);
    cuda_check(launch_project_dot(g, w.b.p, w.b.p, w.partial.p, w.stream), "dot"); count(w);
    cuda_check(launch_reduce_sum(w.partial.p, nt, w.sums.p + 3, w.stream), "reduce"); count(w);
    float tmax = 0;
    double d2[2] = {0, 0};
    cuda_check(cudaMemcpyAsync(&tmax, w.scalars_f.p + 1, sizeof(float), cudaMemcpyDeviceToHost, w.stream), "D2H");
    cuda_check(cudaMemcpyAsync(d2, w.sums.p + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, w.stream), "D2H");
    sync(w);
    w.solved = true;
    check_waits(w);
    if (res) {
        res->iterations = it;
        res->converged = converged ? 1 : 0;
        res->final_norm = rmax;
        res->b_inf = b_inf;
        res->true_residual_inf = b_inf > 0 ? tmax / b_inf : tmax;
        res->true_residual_l2 = d2[1] > 0 ? std::sqrt(d2[0] / d2[1]) : std::sqrt(d2[0]);
        res->solve_ms = ms;
        res->setup_ms = setup_ms;
    }
    if (breakdown) throw Error(HDD_ERR_BREAKDOWN, "PCG breakdown: non-finite scalar");
    if (!converged) throw Error(HDD_ERR_NOT_CONVERGED, "PCG did not converge within max_iters");
}

void Solver::solve_batch(Work& w, BatchFeeder& feed) {
    if (!initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
    NvtxRange range("solve_batch");
    cuda_check(cudaSetDevice(opts.device), "cudaSetDevice");
    const TileGeom g = geom();
    const int nt = g.ntiles, K = w.k;
    const int mode = opts.precision_mode == HDD_PRECISION_MIXED ? 1 : 0;
    const int np = laplace_partials(g);
    const size_t N = w.vstride;
    const float small_number = 1.1920929e-07f;
    // Per-system state, the host side of what Solver::solve keeps in locals.
    struct Sys {
        bool busy = false, replaced = false, restart = false;
        long long id = -1;
        int it = 0;
        double b_inf = 0;
        float threshold = 0, rmax = 0;
        std::chrono::steady_clock::time_point t0;
    };
    std::vector<Sys> sys(K);
    std::vector<int> h_active(K, 0), h_first(K, 0), h_rep(K, 0);
    std::vector<float> h_rmax(K, 0.0f);
    std::vector<PcgScalars> h_scal(K);
    PcgScalars init;
    std::memset(&init, 0, sizeof(init));
    init.rho_old = 3.402823466e+38f;
    init.rho_old_d = 3.402823466e+38;
    auto xs = [&](int j) { return w.x.p + j * N; };
    auto rs = [&](int j) { return w.r.p + j * N; };
    auto bs = [&](int j) { return w.b.p + j * N; };
    auto qs = [&](int j) { return w.q.p + j * N; };
    auto xds = [&](int j) { return mode == 1 ? w.xd.p + j * N : nullptr; };
    auto pms = [&](int j) { return w.partial_max.p + (size_t)j * w.pstride; };
    auto pds = [&](int j) { return w.partial.p + (size_t)j * w.pstride; };
    auto read_max = [&](int j, float* slot_out) {
        float v = 0;
        cuda_check(launch_reduce_max(pms(j), nt, slot_out, w.stream), "reduce");
        count(w);
        cuda_check(cudaMemcpyAsync(&v, slot_out, sizeof(float), cudaMemcpyDeviceToHost, w.stream), "D2H");
        sync(w);
        return v;
    };
    // Ends system j: the true residual of its iterate (reported), its
    // solution in the caller's layout, the feeder told.
    auto finish = [&](int j, hdd_status st) {
        Sys& S = sys[j];
        float* sf = w.scalars_f.p + 8 * j;
        if (mode == 1) cuda_check(launch_residual_f64(g, bs(j), xds(j), qs(j), pms(j), w.stream), "true residual");
        else cuda_check(launch_residual(g, bs(j), xs(j), qs(j), pms(j), w.stream), "true residual");
        count(w);
        cuda_check(launch_reduce_max(pms(j), nt, sf + 1, w.stream), "reduce"); count(w);
        cuda_check(launch_project_dot(g, qs(j), qs(j), pds(j), w.stream), "dot"); count(w);
        cuda_check(launch_reduce_sum(pds(j), nt, w.sums.p + 8 * j + 2, w.stream), "reduce"); count(w);
        cuda_check(launch_project_dot(g, bs(j), bs(j), pds(j), w.stream), "dot"); count(w);
        cuda_check(launch_reduce_sum(pds(j), nt, w.sums.p + 8 * j + 3, w.stream), "reduce"); count(w);
        float tmax = 0;
        double d2[2] = {0, 0};
        cuda_check(cudaMemcpyAsync(&tmax, sf + 1, sizeof(float), cudaMemcpyDeviceToHost, w.stream), "D2H");
        cuda_check(cudaMemcpyAsync(d2, w.sums.p + 8 * j + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, w.stream),
                   "D2H");
        cuda_check(cudaMemsetAsync(w.dense.p, 0, L.cell_count() * sizeof(float), w.stream), "memset");
        cuda_check(launch_tiles_to_dense(g, tile_xyz.p, L.opt.size[0], L.opt.size[1], L.opt.size[2], xs(j), w.dense.p,
                                         w.stream),
                   "tiles_to_dense");
        count(w);
        std::vector<float> x(L.cell_count());
        cuda_check(cudaMemcpyAsync(x.data(), w.dense.p, x.size() * sizeof(float), cudaMemcpyDeviceToHost, w.stream),
                   "D2H x");
        sync(w);
        hdd_result res{};
        res.iterations = S.it;
        res.converged = st == HDD_OK ? 1 : 0;
        res.final_norm = S.rmax;
        res.b_inf = S.b_inf;
        res.true_residual_inf = S.b_inf > 0 ? tmax / S.b_inf : tmax;
        res.true_residual_l2 = d2[1] > 0 ? std::sqrt(d2[0] / d2[1]) : std::sqrt(d2[0]);
        res.solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - S.t0).count();
        res.setup_ms = setup_ms;
        const long long id = S.id;
        S = Sys();
        h_active[j] = 0;
        feed.done(id, st, res, std::move(x));
    };
    // The stop test of Solver::solve for system j (its rmax just read):
    // true when the system is finished (converged, or its true residual
    // check asked for a restart and it goes on).
    auto stop_test = [&](int j) -> bool {
        Sys& S = sys[j];
        if (S.rmax <= S.threshold && (S.it >= opts.min_iters || S.rmax < small_number)) {
            if (mode != 1 || S.replaced) { finish(j, HDD_OK); return true; }
            float* sf = w.scalars_f.p + 8 * j;
            cuda_check(launch_residual_f64(g, bs(j), xds(j), rs(j), pms(j), w.stream), "true residual"); count(w);
            S.rmax = read_max(j, sf);
            S.replaced = true;
            if (S.rmax <= S.threshold) { finish(j, HDD_OK); return true; }
            S.restart = true;
        }
        if (S.it >= opts.max_iters) { finish(j, HDD_ERR_NOT_CONVERGED); return true; }
        return false;
    };
    // Starts a request on free system j: b from its right-hand side, x = 0,
    // r = Project(b) (the restart branch of CONJUGATE_GRADIENT.cpp:36).
    auto start = [&](int j, const float* rhs, long long id) {
        Sys& S = sys[j];
        S = Sys();
        S.busy = true;
        S.id = id;
        S.t0 = std::chrono::steady_clock::now();
        cuda_check(cudaMemcpyAsync(w.dense.p, rhs, L.cell_count() * sizeof(float), cudaMemcpyHostToDevice, w.stream),
                   "H2D rhs");
        cuda_check(launch_dense_to_tiles(g, tile_xyz.p, L.opt.size[0], L.opt.size[1], L.opt.size[2], w.dense.p, bs(j),
                                         w.stream),
                   "dense_to_tiles");
        count(w);
        cuda_check(cudaMemcpyAsync(w.scal.p + j, &init, sizeof(init), cudaMemcpyHostToDevice, w.stream), "scalars");
        cuda_check(cudaMemsetAsync(xs(j), 0, N * sizeof(float), w.stream), "memset x");
        if (mode == 1) cuda_check(cudaMemsetAsync(xds(j), 0, N * sizeof(double), w.stream), "memset xd");
        cuda_check(launch_residual(g, bs(j), xs(j), rs(j), pms(j), w.stream), "residual"); count(w);
        S.rmax = read_max(j, w.scalars_f.p + 8 * j);
        S.b_inf = S.rmax;
        S.threshold = opts.relative_tol ? (float)(opts.tol * S.b_inf) : (float)opts.tol;
        h_active[j] = 1;
        if (stop_test(j)) return;
    };
    clear_wait_errors(w);
    // A failure of a device call ends every request the batch holds with its
    // status, then propagates.
    auto fail_all = [&](hdd_status st) {
        for (int j = 0; j < K; ++j) {
            if (!sys[j].busy) continue;
            const long long id = sys[j].id;
            sys[j] = Sys();
            feed.done(id, st, hdd_result{}, std::vector<float>());
        }
    };
    try {
    for (;;) {
        // Free systems take waiting requests.
        for (int j = 0; j < K; ++j) {
            while (!sys[j].busy) {
                const float* rhs = nullptr;
                long long id = -1;
                if (!feed.next(&rhs, &id)) break;
                start(j, rhs, id);
            }
        }
        bool any = false;
        for (int j = 0; j < K; ++j) any |= sys[j].busy;
        if (!any) break;
        for (int j = 0; j < K; ++j) {
            h_first[j] = sys[j].busy && (sys[j].it == 0 || sys[j].restart) ? 1 : 0;
            if (sys[j].busy) { sys[j].replaced = false; sys[j].restart = false; }
        }
        // One system runs as a plain solve (first passed by value below).
        if (K > 1) {
            cuda_check(cudaMemcpyAsync(w.active.p, h_active.data(), K * sizeof(int), cudaMemcpyHostToDevice,
                                       w.stream),
                       "H2D active");
            cuda_check(cudaMemcpyAsync(w.first.p, h_first.data(), K * sizeof(int), cudaMemcpyHostToDevice, w.stream),
                       "H2D first");
        }
        const Batch B = w.batch();
        const int first1 = K == 1 ? h_first[0] : 0;
        apply_preconditioner(w, w.r.p, w.z.p);
        cuda_check(launch_project_dot(g, w.z.p, w.r.p, w.partial.p, w.stream, B), "project_dot"); count(w);
        cuda_check(launch_reduce_sum(w.partial.p, nt, w.sums.p + 0, w.stream, B, 8), "reduce"); count(w);
        cuda_check(launch_scalar_rho(w.scal.p, w.sums.p + 0, first1, w.stream, B, 8), "rho"); count(w);
        cuda_check(launch_update_s(g, w.s.p, w.z.p, w.scal.p, first1, mode, w.stream, B), "update_s"); count(w);
        cuda_check(launch_laplace_dot(g, w.s.p, w.q.p, w.partial.p, w.stream, B), "laplace"); count(w);
        cuda_check(launch_reduce_sum(w.partial.p, np, w.sums.p + 1, w.stream, B, 8), "reduce"); count(w);
        cuda_check(launch_scalar_alpha(w.scal.p, w.sums.p + 1, w.stream, B, 8), "alpha"); count(w);
        cuda_check(launch_update_xr(g, w.x.p, w.r.p, w.s.p, w.q.p, w.scal.p, mode, w.partial_max.p, w.stream,
                                    mode == 1 ? w.xd.p : nullptr, B),
                   "update_xr");
        count(w);
        bool rep = false;
        for (int j = 0; j < K; ++j) {
            h_rep[j] = sys[j].busy && mode == 1 && opts.true_residual_every > 0 &&
                       (sys[j].it + 1) % opts.true_residual_every == 0;
            rep |= h_rep[j] != 0;
        }
        if (rep) {
            Batch R = B;
            if (K > 1) {
                cuda_check(cudaMemcpyAsync(w.replace.p, h_rep.data(), K * sizeof(int), cudaMemcpyHostToDevice,
                                           w.stream),
                           "H2D replace");
                R.active = w.replace.p;
            }
            cuda_check(launch_residual_f64(g, w.b.p, w.xd.p, w.r.p, w.partial_max.p, w.stream, R), "true residual");
            count(w);
        }
        cuda_check(launch_reduce_max(w.partial_max.p, nt, w.scalars_f.p, w.stream, B, 8), "reduce"); count(w);
        for (int j = 0; j < K; ++j) {
            if (!sys[j].busy) continue;
            cuda_check(cudaMemcpyAsync(&h_rmax[j], w.scalars_f.p + 8 * j, sizeof(float), cudaMemcpyDeviceToHost,
                                       w.stream),
                       "D2H");
        }
        cuda_check(cudaMemcpyAsync(h_scal.data(), w.scal.p, K * sizeof(PcgScalars), cudaMemcpyDeviceToHost, w.stream),
                   "D2H");
        int herr = 0, herr2 = 0;
        if (w.sig.err)
            cuda_check(cudaMemcpyAsync(&herr, w.sig.err, sizeof(int), cudaMemcpyDeviceToHost, w.stream), "D2H");
        if (w.sig2.err)
            cuda_check(cudaMemcpyAsync(&herr2, w.sig2.err, sizeof(int), cudaMemcpyDeviceToHost, w.stream), "D2H");
        sync(w);
        herr |= herr2;
        for (int j = 0; j < K; ++j) {
            Sys& S = sys[j];
            if (!S.busy) continue;
            ++S.it;
            S.rmax = h_rmax[j];
            if (h_rep[j]) S.replaced = true;
            // A bounded wait that gave up leaves this iteration's
            // preconditioner invalid for every system of the batch.
            if (herr != 0) { finish(j, HDD_ERR_TIMEOUT); continue; }
            if (h_scal[j].status != 0 || !std::isfinite(S.rmax)) { finish(j, HDD_ERR_BREAKDOWN); continue; }
            stop_test(j);
        }
        if (herr != 0) clear_wait_errors(w);
    }
    } catch (const Error& e) {
        cudaStreamSynchronize(w.stream);
        fail_all(e.status);
        throw;
    } catch (...) {
        cudaStreamSynchronize(w.stream);
        fail_all(HDD_ERR_INTERNAL);
        throw;
    }
}

void Solver::get_solution(Work& w, float* out) {
    if (!w.solved) throw Error(HDD_ERR_NOT_INITIALIZED, "no solution available");
    Tm tm(this, w, 5);
    cuda_check(cudaMemsetAsync(w.dense.p, 0, L.cell_count() * sizeof(float), w.stream), "memset");
    cuda_check(launch_tiles_to_dense(geom(), tile_xyz.p, L.opt.size[0], L.opt.size[1], L.opt.size[2], w.x.p,
                                     w.dense.p, w.stream), "tiles_to_dense");
    count(w);
    cuda_check(cudaMemcpyAsync(out, w.dense.p, L.cell_count() * sizeof(float), cudaMemcpyDeviceToHost, w.stream),
               "D2H x");
    sync(w);
}

void Solver::get_solution_f64(double* out) {
    if (!w0.solved) throw Error(HDD_ERR_NOT_INITIALIZED, "no solution available");
    const size_t n = L.cell_count();
    DevBuf<double> tmp_dense;
    const double* src = w0.xd.p;
    if (!src) {
        // Reference precision: the FP32 iterate, widened.
        std::vector<float> xf(n);
        get_solution(xf.data());
        for (size_t i = 0; i < n; ++i) out[i] = xf[i];
        return;
    }
    tmp_dense.alloc(std::max<size_t>(n, 1));
    cuda_check(cudaMemsetAsync(tmp_dense.p, 0, n * sizeof(double), stream), "memset");
    cuda_check(launch_tiles_to_dense_f64(geom(), tile_xyz.p, L.opt.size[0], L.opt.size[1], L.opt.size[2], src,
                                         tmp_dense.p, stream), "tiles_to_dense_f64");
    count(w0);
    cuda_check(cudaMemcpyAsync(out, tmp_dense.p, n * sizeof(double), cudaMemcpyDeviceToHost, stream), "D2H x");
    sync();
}

void Solver::apply_preconditioner_dense(const float* rin, float* zout) {
    if (!initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
    std::vector<float> t(L.tiled_count());
    dense_to_tiles(L, rin, t.data());
    cuda_check(cudaMemcpyAsync(w0.r.p, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice, stream), "H2D");
    w0.z.zero(stream);
    clear_wait_errors(w0);
    apply_preconditioner(w0, w0.r.p, w0.z.p);
    cuda_check(launch_project(geom(), w0.z.p, stream), "project"); count(w0);
    cuda_check(cudaMemcpyAsync(t.data(), w0.z.p, t.size() * sizeof(float), cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    check_waits();
    tiles_to_dense(L, t.data(), zout);
}

void Solver::vcycle_dense(float* u, const float* bb, int nv) {
    if (!initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
    std::vector<float> t(L.tiled_count());
    dense_to_tiles(L, u, t.data());
    cuda_check(cudaMemcpyAsync(w0.z.p, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice, stream), "H2D");
    std::vector<float> tb(L.tiled_count());
    dense_to_tiles(L, bb, tb.data());
    cuda_check(cudaMemcpyAsync(w0.q.p, tb.data(), tb.size() * sizeof(float), cudaMemcpyHostToDevice, stream), "H2D");
    run_vcycle(w0, w0.z.p, w0.q.p, 1, 0, nv);
    cuda_check(cudaMemcpyAsync(t.data(), w0.z.p, t.size() * sizeof(float), cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    // Cells outside stored tiles keep the caller's values.
    std::vector<float> dense(L.cell_count());
    tiles_to_dense(L, t.data(), dense.data());
    const int* n = L.opt.size;
    for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
            for (int k = 0; k < n[2]; ++k)
                if (L.tile_slot(i, j, k) >= 0) u[L.dense_index(i, j, k)] = dense[L.dense_index(i, j, k)];
}

void Solver::multiply_dense(const float* xin, float* yout) {
    if (!initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
    std::vector<float> t(L.tiled_count());
    dense_to_tiles(L, xin, t.data());
    cuda_check(cudaMemcpyAsync(w0.s.p, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice, stream), "H2D");
    cuda_check(launch_laplace_dot(geom(), w0.s.p, w0.q.p, w0.partial.p, stream), "laplace"); count(w0);
    cuda_check(cudaMemcpyAsync(t.data(), w0.q.p, t.size() * sizeof(float), cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    tiles_to_dense(L, t.data(), yout);
}

void Solver::sigma_vcycle_host(const float* b0, float* u0) {
    if (!initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
    const int n_if = ih.n_iface.empty() ? 0 : ih.n_iface[0];
    if (n_if == 0) return;
    cuda_check(cudaMemcpyAsync(sigma.b0(), b0, n_if * sizeof(float), cudaMemcpyHostToDevice, stream), "H2D");
    cuda_check(cudaMemsetAsync(sigma.u0(), 0, n_if * sizeof(float), stream), "memset");
    sigma.clear_error(stream);
    sigma.vcycle(stream, w0.launches);
    cuda_check(cudaMemcpyAsync(u0, sigma.u0(), n_if * sizeof(float), cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    check_waits();
}

void Solver::interface_solve(int kind, int level, const float* bh, float* xh, int* n) {
    if (!initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
    if (level < 0 || level >= (int)sigma.lv.size()) throw Error(HDD_ERR_INVALID_ARGUMENT, "level out of range");
    SigmaLevel& Lv = sigma.lv[level];
    const SolvePlan& plan = kind == 0 ? Lv.arr_solve : Lv.aii;
    const int rows = kind == 0 ? Lv.n_iface : Lv.n_int;
    *n = rows;
    if (!bh || !xh) return;
    if (plan.nsn == 0 && rows > 0)
        throw Error(HDD_ERR_UNSUPPORTED, "no separate solve plan at this level (coarsest level solved as a whole)");
    if (rows == 0) return;
    float* db = kind == 0 ? Lv.tmp : Lv.vb;
    float* dx = kind == 0 ? Lv.u : Lv.vx;
    cuda_check(cudaSetDevice(opts.device), "cudaSetDevice");
    cuda_check(cudaMemcpyAsync(db, bh, rows * sizeof(float), cudaMemcpyHostToDevice, stream), "H2D");
    cuda_check(cudaMemsetAsync(dx, 0, rows * sizeof(float), stream), "memset");
    sigma.clear_error(stream);
    plan.solve(db, dx, stream, w0.launches, &hook);
    cuda_check(cudaMemcpyAsync(xh, dx, rows * sizeof(float), cudaMemcpyDeviceToHost, stream), "D2H");
    sync();
    check_waits();
}

void Solver::interface_solve_batch(int kind, int level, int nrhs, const float* bh, float* xh, int* n) {
    if (!initialized) throw Error(HDD_ERR_NOT_INITIALIZED, "initialize_preconditioner not called");
    if (level < 0 || level >= (int)sigma.lv.size()) throw Error(HDD_ERR_INVALID_ARGUMENT, "level out of range");
    if (nrhs != 1 && nrhs != 2 && nrhs != 4) throw Error(HDD_ERR_INVALID_ARGUMENT, "nrhs must be 1, 2 or 4");
    const SigmaLevel& Lv = sigma.lv[level];
    const SolvePlan& plan = kind == 0 ? Lv.arr_solve : Lv.aii;
    const int rows = kind == 0 ? Lv.n_iface : Lv.n_int;
    *n = rows;
    if (!bh || !xh) return;
    if (plan.nsn == 0 && rows > 0)
        throw Error(HDD_ERR_UNSUPPORTED, "no separate solve plan at this level (coarsest level solved as a whole)");
    if (rows == 0) return;
    if (nrhs > plan.kmax) throw Error(HDD_ERR_UNSUPPORTED, "this plan's fronts leave no shared memory for that many right-hand sides");
    cuda_check(cudaSetDevice(opts.device), "cudaSetDevice");
    DevBuf<float> db, dx;
    db.upload(bh, (size_t)rows * nrhs, stream);
    dx.alloc((size_t)rows * nrhs);
    dx.zero(stream);
    PlanScratch sc;
    size_t bytes = 0;
    plan.alloc_scratch(sc, nullptr, stream, bytes, nrhs);
    try {
        plan.solve(sc, db.p, dx.p, stream, w0.launches, nullptr, nrhs, rows, rows);
        cuda_check(cudaMemcpyAsync(xh, dx.p, (size_t)rows * nrhs * sizeof(float), cudaMemcpyDeviceToHost, stream),
                   "D2H");
        sync();
    } catch (...) {
        cudaStreamSynchronize(stream);
        SolvePlan::free_scratch(sc);
        throw;
    }
    int herr = 0;
    cuda_check(cudaMemcpy(&herr, sc.err, sizeof(int), cudaMemcpyDeviceToHost), "D2H");
    SolvePlan::free_scratch(sc);
    if (herr) throw Error(HDD_ERR_TIMEOUT, "a bounded device wait in the batched solve gave up");
}

void Solver::check_waits(Work& w) {
    if (wait_error(w))
        throw Error(HDD_ERR_TIMEOUT, "a bounded device wait in the sigma solve gave up; results are invalid");
}

}  // namespace hdd
