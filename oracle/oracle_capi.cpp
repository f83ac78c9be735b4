// ORACLE (test infrastructure only) -- solver object and C entry points used by
// tests/ (through ctypes), __graft_entry__.smoke() and bench.py's cpu_baseline.
//
// Restates the CPU dd_pcg driver:
//   CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Solver.h:121-197
//   CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Preconditioner.h:88-128
//   CPU/SPGrid_Domain_Decomposition_Solver/CG_SYSTEM.cpp:28-119
//   PB/Public_Library/PhysBAM_Tools/Krylov_Solvers/CONJUGATE_GRADIENT.cpp:22-67
//   PB/Public_Library/PhysBAM_Tools/Krylov_Solvers/KRYLOV_SYSTEM_BASE.cpp:100-106
// Vectors are dense x-slowest/z-fastest arrays over the level-0 grid.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>

#include "oracle_core.h"
#include "oracle_interface.h"

namespace oracle {

struct SolverBase {
    virtual ~SolverBase() {}
    Dims d0;
    int sub[3];
    int vlevels, nvcycles, interior, boundary, sigma_levels, sigma_smoothing, sigma_mg;
    int multilevel = 0;  // two-level DD (the Two_Levels demo's -multilevel yes)
    std::vector<uint32_t> flags_in;
    virtual int num_levels() const = 0;
    virtual const Dims& level_dims(int l) const = 0;
    virtual const uint32_t* level_flags(int l) const = 0;
};

template <class T>
struct Solver : SolverBase {
    std::vector<MGLevel<T>> lv;
    InterfaceSystem<T> sys;
    SigmaSolver<T> sigma;
    std::vector<T> k_tmp;  // preconditioner tmp channel (CG_SYSTEM's preconditioner_tmp_field)
    // Two-level DD: one interface system per first-level subdomain box, on
    // the box split at sub/2 (iface_map in global cells).
    std::vector<std::unique_ptr<InterfaceSystem<T>>> sys2;
    std::vector<std::unique_ptr<SigmaSolver<T>>> sigma2;

    int num_levels() const override { return (int)lv.size(); }
    const Dims& level_dims(int l) const override { return lv[l].d; }
    const uint32_t* level_flags(int l) const override { return lv[l].flags.data(); }

    void setup() {
        // SPGrid_Domain_Decomposition_Solver.h:121-155.
        const bool verbose = std::getenv("HDDO_VERBOSE") != nullptr;
        auto t0 = std::chrono::steady_clock::now();
        auto stamp = [&](const char* what) {
            if (!verbose) return;
            const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::fprintf(stderr, "[oracle setup] %s at %.2f s\n", what, s);
        };
        build_interface_system<T>(d0, flags_in.data(), sub, sigma_levels, sys);
        stamp("interface system");
        // Two-level: the V-cycles run on boxes of sub/2, whose planes (both
        // levels) are Interface (TWO/SPGrid_Domain_Decomposition_Solver/
        // SPGrid_Domain_Decomposition_Solver.h:124-158).
        int vsub[3] = {sub[0], sub[1], sub[2]};
        if (multilevel) {
            for (int a = 0; a < 3; ++a) {
                if (sub[a] % 2) throw std::runtime_error("two-level DD needs an even sub_size");
                vsub[a] = sub[a] / 2;
            }
            setup_second_level();
            stamp("second-level interface systems");
        }
        lv.resize(vlevels);
        lv[0].d = d0;
        lv[0].flags = flags_in;
        divide_domain(d0, lv[0].flags.data(), vsub);
        flag_faces(d0, lv[0].flags.data());
        for (int l = 0; l + 1 < vlevels; ++l) {
            for (int a = 0; a < 3; ++a) lv[l + 1].d.n[a] = lv[l].d.n[a] / 2 + 1;
            lv[l + 1].flags.assign(lv[l + 1].d.count(), 0u);
            downsample_topology(lv[l].d, lv[l].flags.data(), lv[l + 1].d, lv[l + 1].flags.data());
        }
        for (int l = 0; l < vlevels; ++l) {
            flag_faces(lv[l].d, lv[l].flags.data());
            flag_boundary(lv[l].d, lv[l].flags.data());
            if (l > 0) {
                lv[l].u.assign(lv[l].d.count(), T(0));
                lv[l].r.assign(lv[l].d.count(), T(0));
                lv[l].b.assign(lv[l].d.count(), T(0));
            }
        }
        stamp("topology");
        sigma.initialize(sys, sigma_smoothing);
        stamp("factorisations");
        k_tmp.assign(d0.count(), T(0));
    }

    // TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Subdomain_Splitter.h:168-193:
    // each first-level subdomain box [lo, lo + sub] gets the caller's flags
    // with its Active cells on first-level planes made Dirichlet
    // (Domain_Divider with clear_flag, TWO/.../SPGrid_Domain_Divider_Helper.h:61-72),
    // split again at sub/2 into its own interface system.  The box is built
    // as a local grid whose origin is a multiple of sub, so plane tests on
    // local indices equal those on global ones.
    void setup_second_level() {
        int ns[3], sub2[3];
        number_of_subdomains(d0.n, sub, ns);
        for (int a = 0; a < 3; ++a) sub2[a] = sub[a] / 2;
        sys2.clear();
        sigma2.clear();
        for (int si = 0; si < ns[0]; ++si)
            for (int sj = 0; sj < ns[1]; ++sj)
                for (int sk = 0; sk < ns[2]; ++sk) {
                    const int lo[3] = {si * sub[0], sj * sub[1], sk * sub[2]};
                    Dims ld;
                    for (int a = 0; a < 3; ++a) ld.n[a] = std::min(sub[a] + 1, d0.n[a] - lo[a]);
                    std::vector<uint32_t> lf(ld.count(), 0u);
                    for (int i = 0; i < ld.n[0]; ++i)
                        for (int j = 0; j < ld.n[1]; ++j)
                            for (int k = 0; k < ld.n[2]; ++k) {
                                uint32_t f = flags_in[d0.at(lo[0] + i, lo[1] + j, lo[2] + k)];
                                if ((f & ACTIVE) && (i % sub[0] == 0 || j % sub[1] == 0 || k % sub[2] == 0))
                                    f = DIRICHLET;
                                lf[ld.at(i, j, k)] = f;
                            }
                    std::unique_ptr<InterfaceSystem<T>> sy(new InterfaceSystem<T>());
                    build_interface_system<T>(ld, lf.data(), sub2, sigma_levels, *sy);
                    if (sy->n_iface.empty() || sy->n_iface[0] == 0) continue;
                    for (auto& c : sy->iface_map)
                        for (int a = 0; a < 3; ++a) c[a] += lo[a];
                    std::unique_ptr<SigmaSolver<T>> sg(new SigmaSolver<T>());
                    sg->initialize(*sy, sigma_smoothing);
                    sys2.push_back(std::move(sy));
                    sigma2.push_back(std::move(sg));
                }
    }

    // b[i] = v at the map's Interface cells (EIGEN_INTERFACE::Copy_To_Eigen_Array),
    // or b[i] += v (TWO/Interface_Solver/EIGEN_INTERFACE.cpp:33-50, Accumulate_To_Eigen_Array).
    void to_interface(const std::vector<std::array<int, 3>>& map, std::vector<T>& b, const T* v, bool acc) const {
        const uint32_t* f = lv[0].flags.data();
        for (size_t i = 0; i < map.size(); ++i) {
            const size_t x = d0.at(map[i][0], map[i][1], map[i][2]);
            if (!(f[x] & INTERFACE)) continue;
            if (acc) b[i] += v[x];
            else b[i] = v[x];
        }
    }
    void from_interface(const std::vector<std::array<int, 3>>& map, const std::vector<T>& u, T* v) const {
        const uint32_t* f = lv[0].flags.data();
        for (size_t i = 0; i < map.size(); ++i) {
            const size_t x = d0.at(map[i][0], map[i][1], map[i][2]);
            if (f[x] & INTERFACE) v[x] = u[i];
        }
    }

    // TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Preconditioner.h:127-181
    // (Subdomain_DD; residual prints dropped): a DD solve inside every
    // first-level subdomain with the first-level interface values in result
    // as its boundary data.
    void subdomain_dd(T* result, const T* rhs, T* tmp) {
        const size_t n = d0.count();
        const uint32_t* f = lv[0].flags.data();
        for (auto& sg : sigma2) std::fill(sg->b[0].begin(), sg->b[0].end(), T(0));
        std::fill(tmp, tmp + n, T(0));
        laplace_ir_subdomain<T>(d0, f, result, tmp, sub);
        for (size_t s = 0; s < sys2.size(); ++s) to_interface(sys2[s]->iface_map, sigma2[s]->b[0], tmp, false);
        for (int i = 0; i < nvcycles; ++i) v_cycle<T>(lv, result, tmp, rhs, interior, boundary);
        std::copy(rhs, rhs + n, tmp);
        laplace_ri<T>(d0, f, result, tmp);
        for (size_t s = 0; s < sys2.size(); ++s) {
            to_interface(sys2[s]->iface_map, sigma2[s]->b[0], tmp, true);
            std::fill(sigma2[s]->u[0].begin(), sigma2[s]->u[0].end(), T(0));
            for (int i = 0; i < sigma_mg; ++i) sigma2[s]->v_cycle();
        }
        std::fill(result, result + n, T(0));
        std::fill(tmp, tmp + n, T(0));
        from_interface(sys.iface_map, sigma.u[0], result);
        for (size_t s = 0; s < sys2.size(); ++s) from_interface(sys2[s]->iface_map, sigma2[s]->u[0], result);
        for (int i = 0; i < nvcycles; ++i) v_cycle<T>(lv, result, tmp, rhs, interior, boundary);
    }

    // TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Preconditioner.h:182-230
    // with multilevel: the subdomain V-cycles replaced by Subdomain_DD, and the
    // first-level interface right-hand side from Laplace_ri_Subdomain.
    void apply_two_level(T* result, const T* rhs, T* tmp) {
        const size_t n = d0.count();
        const uint32_t* f = lv[0].flags.data();
        std::fill(sigma.u[0].begin(), sigma.u[0].end(), T(0));
        std::fill(result, result + n, T(0));
        std::fill(tmp, tmp + n, T(0));
        subdomain_dd(result, rhs, tmp);
        std::copy(rhs, rhs + n, tmp);
        laplace_ri_subdomain<T>(d0, f, result, tmp, sub);
        std::fill(sigma.b[0].begin(), sigma.b[0].end(), T(0));
        to_interface(sys.iface_map, sigma.b[0], tmp, false);
        std::fill(sigma.u[0].begin(), sigma.u[0].end(), T(0));
        for (int i = 0; i < sigma_mg; ++i) sigma.v_cycle();
        std::fill(result, result + n, T(0));
        std::fill(tmp, tmp + n, T(0));
        from_interface(sys.iface_map, sigma.u[0], result);
        subdomain_dd(result, rhs, tmp);
    }

    void project(T* v) const {
        const uint32_t* f = lv[0].flags.data();
        for (size_t x = 0; x < d0.count(); ++x)
            if (!(f[x] & (ACTIVE | INTERFACE))) v[x] = T(0);
    }

    // SPGrid_Domain_Decomposition_Preconditioner.h:88-128 (debug residual prints dropped).
    void apply_preconditioner(T* result, const T* rhs, T* tmp) {
        if (multilevel) { apply_two_level(result, rhs, tmp); return; }
        const size_t n = d0.count();
        const uint32_t* f = lv[0].flags.data();
        std::fill(result, result + n, T(0));
        std::fill(tmp, tmp + n, T(0));
        for (int i = 0; i < nvcycles; ++i) v_cycle<T>(lv, result, tmp, rhs, interior, boundary);
        std::copy(rhs, rhs + n, tmp);
        laplace_ri<T>(d0, f, result, tmp);
        std::vector<T>& b0 = sigma.b[0];
        std::fill(b0.begin(), b0.end(), T(0));
        for (size_t i = 0; i < sys.iface_map.size(); ++i) {
            auto& c = sys.iface_map[i];
            size_t x = d0.at(c[0], c[1], c[2]);
            if (f[x] & INTERFACE) b0[i] = tmp[x];
        }
        std::fill(sigma.u[0].begin(), sigma.u[0].end(), T(0));
        for (int i = 0; i < sigma_mg; ++i) sigma.v_cycle();
        std::fill(result, result + n, T(0));
        std::fill(tmp, tmp + n, T(0));
        for (size_t i = 0; i < sys.iface_map.size(); ++i) {
            auto& c = sys.iface_map[i];
            size_t x = d0.at(c[0], c[1], c[2]);
            if (f[x] & INTERFACE) result[x] = sigma.u[0][i];
        }
        for (int i = 0; i < nvcycles; ++i) v_cycle<T>(lv, result, tmp, rhs, interior, boundary);
    }

    double dot(const T* a, const T* b) const {
        double s = 0;
        for (size_t x = 0; x < d0.count(); ++x) s += (double)(a[x] * b[x]);
        return s;
    }
    T max_abs(const T* a) const {
        T m = 0;
        for (size_t x = 0; x < d0.count(); ++x) m = (std::fabs(a[x]) > m) ? std::fabs(a[x]) : m;
        return m;
    }

    // CONJUGATE_GRADIENT.cpp:22-67 with KRYLOV_SYSTEM_BASE::Precondition.  The
    // stop test is max|r| <= tol (relative=0, the reference's test) or
    // max|r| <= tol * max|b| over Active|Interface cells (relative=1).
    // times (optional, history_len entries): wall seconds from the start of
    // the solve to the end of each PCG iteration.
    int solve(const T* b_in, T* x, double tol, bool relative, int min_it, int max_it, double* norms,
              double* history, int history_len, double* times = nullptr) {
        const auto t_start = std::chrono::steady_clock::now();
        const size_t n = d0.count();
        std::vector<T> b(b_in, b_in + n), q(n, T(0)), s(n, T(0)), r(n, T(0)), z(n, T(0));
        project(b.data());
        std::fill(x, x + n, T(0));
        const T small_number = std::numeric_limits<T>::epsilon();
        const double bnorm = (double)max_abs(b.data());
        const T threshold = relative ? (T)(tol * bnorm) : (T)tol;
        T rho_old = (T)FLT_MAX, convergence_norm = 0;
        int it;
        for (it = 0;; ++it) {
            if (it == 0) {
                r = b;
                laplace_ai<T>(d0, lv[0].flags.data(), x, q.data());
                for (size_t i = 0; i < n; ++i) r[i] -= q[i];
                project(r.data());
            }
            convergence_norm = max_abs(r.data());
            if (history && it < history_len) history[it] = (double)convergence_norm;
            if (convergence_norm <= threshold && (it >= min_it || convergence_norm < small_number)) break;
            if (it == max_it) break;
            apply_preconditioner(z.data(), r.data(), k_tmp.data());
            project(z.data());
            T rho = (T)dot(z.data(), r.data());
            if (it == 0) s = z;
            else {
                T beta = rho / rho_old;
                for (size_t i = 0; i < n; ++i) s[i] = s[i] * beta + z[i];
            }
            laplace_ai<T>(d0, lv[0].flags.data(), s.data(), q.data());
            project(q.data());
            T sdq = (T)dot(s.data(), q.data());
            T alpha = sdq ? rho / sdq : (T)FLT_MAX;
            for (size_t i = 0; i < n; ++i) x[i] = s[i] * alpha + x[i];
            for (size_t i = 0; i < n; ++i) r[i] = q[i] * (-alpha) + r[i];
            rho_old = rho;
            if (times && it < history_len)
                times[it] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
        }
        if (norms) {
            norms[0] = (double)convergence_norm;
            norms[1] = bnorm;
            // True residual of the returned x.
            std::vector<T> ax(n, T(0));
            laplace_ai<T>(d0, lv[0].flags.data(), x, ax.data());
            double tmax = 0, t2 = 0, b2 = 0;
            const uint32_t* f = lv[0].flags.data();
            for (size_t i = 0; i < n; ++i)
                if (f[i] & (ACTIVE | INTERFACE)) {
                    double rr = (double)b[i] - (double)ax[i];
                    tmax = std::max(tmax, std::fabs(rr));
                    t2 += rr * rr;
                    b2 += (double)b[i] * (double)b[i];
                }
            norms[2] = tmax;
            norms[3] = std::sqrt(t2);
            norms[4] = std::sqrt(b2);
        }
        return it;
    }
};

}  // namespace oracle

using namespace oracle;

namespace {
struct Handle {
    std::unique_ptr<SolverBase> s;
    bool dbl = false;
    std::string err;
};
template <class T>
Solver<T>& S(Handle* h) { return *static_cast<Solver<T>*>(h->s.get()); }
}  // namespace

#define DISPATCH(h, expr) ((h)->dbl ? ([&](Solver<double>& s) { return expr; })(S<double>(h)) \
                                     : ([&](Solver<float>& s) { return expr; })(S<float>(h)))

extern "C" {

void* hddo_create_ml(const int size[3], const int sub[3], const uint32_t* flags, int vlevels, int nvcycles,
                     int interior, int boundary, int sigma_levels, int sigma_smoothing, int sigma_mg,
                     int use_double, int multilevel, char* err, int errlen) {
    Handle* h = new Handle();
    h->dbl = use_double != 0;
    try {
        SolverBase* base;
        if (h->dbl) base = new Solver<double>(); else base = new Solver<float>();
        h->s.reset(base);
        for (int a = 0; a < 3; ++a) { base->d0.n[a] = size[a]; base->sub[a] = sub[a]; }
        base->vlevels = vlevels;
        base->nvcycles = nvcycles;
        base->interior = interior;
        base->boundary = boundary;
        base->sigma_levels = sigma_levels;
        base->sigma_smoothing = sigma_smoothing;
        base->sigma_mg = sigma_mg;
        base->multilevel = multilevel;
        base->flags_in.assign(flags, flags + base->d0.count());
        if (h->dbl) S<double>(h).setup(); else S<float>(h).setup();
    } catch (const std::exception& e) {
        if (err && errlen > 0) snprintf(err, errlen, "%s", e.what());
        delete h;
        return nullptr;
    }
    return h;
}

void* hddo_create(const int size[3], const int sub[3], const uint32_t* flags, int vlevels, int nvcycles,
                  int interior, int boundary, int sigma_levels, int sigma_smoothing, int sigma_mg,
                  int use_double, char* err, int errlen) {
    return hddo_create_ml(size, sub, flags, vlevels, nvcycles, interior, boundary, sigma_levels, sigma_smoothing,
                          sigma_mg, use_double, 0, err, errlen);
}

// Second-level interface systems of a two-level solver: their count, and
// each one's level-0 interface size.
int hddo_num_second_level(void* hp) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, (int)s.sys2.size());
}
int hddo_second_level_interface(void* hp, int i) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, s.sys2[i]->n_iface[0]);
}
// Second-level system i: interface DOF count of a level, level-0 interface
// cells (global), and its matrices as hddo_matrix_shape / hddo_matrix_get.
int hddo_sl_num_interface(void* hp, int i, int level) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, level < (int)s.sys2[i]->n_iface.size() ? s.sys2[i]->n_iface[level] : -1);
}
void hddo_sl_interface_map(void* hp, int i, int* out) {
    Handle* h = static_cast<Handle*>(hp);
    DISPATCH(h, ([&] { const auto& m = s.sys2[i]->iface_map;
                       for (size_t r = 0; r < m.size(); ++r)
                           for (int a = 0; a < 3; ++a) out[3 * r + a] = m[r][a];
                       return 0; })());
}
int hddo_sl_num_subdomains(void* hp, int i) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, s.sys2[i]->n_sub);
}
int hddo_sl_matrix_shape(void* hp, int i, int kind, int level, int sub, int* rows, int* cols, int* nnz) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, ([&] {
        const auto& y = *s.sys2[i];
        const auto* m = kind == 0 ? &y.Arr[level] : kind == 1 ? &y.Aii[level][sub]
                      : kind == 2 ? &y.Air[level][sub] : &y.Prr[level];
        *rows = m->rows; *cols = m->cols; *nnz = (int)m->col.size();
        return 0; })());
}
int hddo_sl_matrix_get(void* hp, int i, int kind, int level, int sub, int* ptr, int* col, double* val) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, ([&] {
        const auto& y = *s.sys2[i];
        const auto* m = kind == 0 ? &y.Arr[level] : kind == 1 ? &y.Aii[level][sub]
                      : kind == 2 ? &y.Air[level][sub] : &y.Prr[level];
        std::copy(m->ptr.begin(), m->ptr.end(), ptr);
        std::copy(m->col.begin(), m->col.end(), col);
        for (size_t r = 0; r < m->val.size(); ++r) val[r] = (double)m->val[r];
        return 0; })());
}

// The Test_Bench "velocity" mode on a uniform (single-level) grid:
//   PB/Common_Libraries/SPGrid_Fluids/Projection/Divergence_Helper.cpp:150-240 (3D
//   Run_Index_Range): at Interior|Ghost cells, result (T) starts at 0 and takes
//   -= scale * u_face(cell) when the cell's face is valid, += scale *
//   u_face(cell + e) when the neighbour's is, for x, y, z in turn, each in double
//   and rounded to T;
//   GRID_HIERARCHY_PROJECTION.h:31-42 (OLD_SCALING): scale = (1/dx)^3 * (-dx * dx)
//   with one_over_dX = 1/dX in T;
//   GPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Convertor.h:213-236: the
//   solver's flags are Dirichlet where the fluid cell is Dirichlet, else
//   Active where it is Active, else exterior.
// Fluid flag bits (FLUIDS_SIMULATION_FLAGS.h:13-25): Interior 0x1, Dirichlet
// 0x2, Ghost 0x4, Active 0x8, face X/Y/Z valid 0x10/0x20/0x40.  Arrays are
// dense x-slowest over size[0..2] cells; a neighbour outside the grid counts
// as invalid.
void hddo_velocity_divergence(const int size[3], const uint32_t* fflags, const float* u, const float* v,
                              const float* w, float dx, uint32_t* flags_out, float* rhs_out) {
    const Dims d{{size[0], size[1], size[2]}};
    const float odx = 1.0f / dx;
    const double scale = ((double)odx * (double)odx * (double)odx) * ((double)(-1.) * (double)dx * (double)dx);
    const float* vel[3] = {u, v, w};
    const uint32_t valid[3] = {0x10u, 0x20u, 0x40u};
    for (int i = 0; i < d.n[0]; ++i)
        for (int j = 0; j < d.n[1]; ++j)
            for (int k = 0; k < d.n[2]; ++k) {
                const size_t x = d.at(i, j, k);
                const uint32_t f = fflags[x];
                flags_out[x] = (f & 0x2u) ? DIRICHLET : ((f & 0x8u) ? ACTIVE : 0u);
                float result = 0;
                if (f & (0x1u | 0x4u)) {
                    for (int a = 0; a < 3; ++a) {
                        const int ni = i + (a == 0), nj = j + (a == 1), nk = k + (a == 2);
                        const bool in = ni < d.n[0] && nj < d.n[1] && nk < d.n[2];
                        const uint32_t fp = in ? fflags[d.at(ni, nj, nk)] : 0u;
                        const double cur = (double)vel[a][x];
                        const double plus = in ? (double)vel[a][d.at(ni, nj, nk)] : 0.0;
                        if (f & valid[a]) result = (float)((double)result - scale * cur);
                        if (fp & valid[a]) result = (float)((double)result + scale * plus);
                    }
                }
                rhs_out[x] = result;
            }
}

void hddo_destroy(void* hp) { delete static_cast<Handle*>(hp); }

int hddo_num_levels(void* hp) { return static_cast<Handle*>(hp)->s->num_levels(); }
void hddo_level_dims(void* hp, int l, int* out) {
    const Dims& d = static_cast<Handle*>(hp)->s->level_dims(l);
    for (int a = 0; a < 3; ++a) out[a] = d.n[a];
}
void hddo_level_flags(void* hp, int l, uint32_t* out) {
    SolverBase* s = static_cast<Handle*>(hp)->s.get();
    const Dims& d = s->level_dims(l);
    std::memcpy(out, s->level_flags(l), d.count() * sizeof(uint32_t));
}

int hddo_num_subdomains(void* hp) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, s.sys.n_sub);
}
int hddo_num_interface(void* hp, int level) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, s.sys.n_iface[level]);
}
void hddo_interface_map(void* hp, int* out) {
    Handle* h = static_cast<Handle*>(hp);
    DISPATCH(h, ([&] { for (size_t i = 0; i < s.sys.iface_map.size(); ++i)
                           for (int a = 0; a < 3; ++a) out[3 * i + a] = s.sys.iface_map[i][a];
                       return 0; })());
}

// kind: 0 = Arr[level], 1 = Aii[level][sub], 2 = Air[level][sub], 3 = Prr[level]
int hddo_matrix_shape(void* hp, int kind, int level, int sub, int* rows, int* cols, int* nnz) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, ([&] {
        const auto* m = kind == 0 ? &s.sys.Arr[level] : kind == 1 ? &s.sys.Aii[level][sub]
                      : kind == 2 ? &s.sys.Air[level][sub] : &s.sys.Prr[level];
        *rows = m->rows; *cols = m->cols; *nnz = (int)m->col.size();
        return 0; })());
}
int hddo_matrix_get(void* hp, int kind, int level, int sub, int* ptr, int* col, double* val) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, ([&] {
        const auto* m = kind == 0 ? &s.sys.Arr[level] : kind == 1 ? &s.sys.Aii[level][sub]
                      : kind == 2 ? &s.sys.Air[level][sub] : &s.sys.Prr[level];
        std::copy(m->ptr.begin(), m->ptr.end(), ptr);
        std::copy(m->col.begin(), m->col.end(), col);
        for (size_t i = 0; i < m->val.size(); ++i) val[i] = (double)m->val[i];
        return 0; })());
}

void hddo_vcycle(void* hp, void* u, void* r, const void* b) {
    Handle* h = static_cast<Handle*>(hp);
    DISPATCH(h, ([&] {
        using T = typename std::remove_reference<decltype(s.lv[0].u[0])>::type;
        v_cycle<T>(s.lv, (T*)u, (T*)r, (const T*)b, s.interior, s.boundary);
        return 0; })());
}

void hddo_apply_preconditioner(void* hp, const void* rhs, void* result) {
    Handle* h = static_cast<Handle*>(hp);
    DISPATCH(h, ([&] {
        using T = typename std::remove_reference<decltype(s.lv[0].u[0])>::type;
        s.apply_preconditioner((T*)result, (const T*)rhs, s.k_tmp.data());
        s.project((T*)result);
        return 0; })());
}

// lu (in/out) after Laplace_ri(u) on the level-0 flags (the interface
// right-hand side step of Apply_Preconditioner).
void hddo_laplace_ri(void* hp, const void* u, void* lu) {
    Handle* h = static_cast<Handle*>(hp);
    DISPATCH(h, ([&] {
        using T = typename std::remove_reference<decltype(s.lv[0].u[0])>::type;
        laplace_ri<T>(s.d0, s.lv[0].flags.data(), (const T*)u, (T*)lu);
        return 0; })());
}

// lu (in/out) after Laplace_ri_Subdomain (which 0) or Laplace_ir_Subdomain
// (which 1) of u at the solver's sub_size, on the level-0 flags (two-level
// DD's couplings).
void hddo_laplace_subdomain(void* hp, int which, const void* u, void* lu) {
    Handle* h = static_cast<Handle*>(hp);
    DISPATCH(h, ([&] {
        using T = typename std::remove_reference<decltype(s.lv[0].u[0])>::type;
        if (which == 0) laplace_ri_subdomain<T>(s.d0, s.lv[0].flags.data(), (const T*)u, (T*)lu, s.sub);
        else laplace_ir_subdomain<T>(s.d0, s.lv[0].flags.data(), (const T*)u, (T*)lu, s.sub);
        return 0; })());
}

// y = project(A x) with the CG system's Laplacian.
void hddo_multiply(void* hp, const void* x, void* y) {
    Handle* h = static_cast<Handle*>(hp);
    DISPATCH(h, ([&] {
        using T = typename std::remove_reference<decltype(s.lv[0].u[0])>::type;
        laplace_ai<T>(s.d0, s.lv[0].flags.data(), (const T*)x, (T*)y);
        s.project((T*)y);
        return 0; })());
}

// One sigma V-cycle from u = 0 for the level-0 interface right-hand side b0.
void hddo_sigma_vcycle(void* hp, const void* b0, void* u0) {
    Handle* h = static_cast<Handle*>(hp);
    DISPATCH(h, ([&] {
        using T = typename std::remove_reference<decltype(s.lv[0].u[0])>::type;
        const T* bb = (const T*)b0;
        std::copy(bb, bb + s.sigma.b[0].size(), s.sigma.b[0].begin());
        std::fill(s.sigma.u[0].begin(), s.sigma.u[0].end(), T(0));
        s.sigma.v_cycle();
        std::copy(s.sigma.u[0].begin(), s.sigma.u[0].end(), (T*)u0);
        return 0; })());
}

// One sigma smoothing step at the given level, in place on u.
void hddo_sigma_smooth(void* hp, int level, void* u, const void* b) {
    Handle* h = static_cast<Handle*>(hp);
    DISPATCH(h, ([&] {
        using T = typename std::remove_reference<decltype(s.lv[0].u[0])>::type;
        int n = s.sys.n_iface[level];
        std::vector<T> uu((T*)u, (T*)u + n), tmp(n), bb((const T*)b, (const T*)b + n);
        s.sigma.smooth(level, uu, tmp, bb);
        std::copy(uu.begin(), uu.end(), (T*)u);
        return 0; })());
}

int hddo_solve(void* hp, const void* b, void* x, double tol, int relative, int min_it, int max_it,
               double* norms, double* history, int history_len) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, ([&] {
        using T = typename std::remove_reference<decltype(s.lv[0].u[0])>::type;
        return s.solve((const T*)b, (T*)x, tol, relative != 0, min_it, max_it, norms, history, history_len);
    })());
}

// hddo_solve with the wall time at the end of every PCG iteration (seconds
// from the start of the solve) in times[0 .. history_len).
int hddo_solve_timed(void* hp, const void* b, void* x, double tol, int relative, int min_it, int max_it,
                     double* norms, double* history, int history_len, double* times) {
    Handle* h = static_cast<Handle*>(hp);
    return DISPATCH(h, ([&] {
        using T = typename std::remove_reference<decltype(s.lv[0].u[0])>::type;
        return s.solve((const T*)b, (T*)x, tol, relative != 0, min_it, max_it, norms, history, history_len, times);
    })());
}

}  // extern "C"
