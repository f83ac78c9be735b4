// Test shim: the product's host-side setup code (layout, interface assembly,
// supernodal Cholesky) compiled without CUDA device code, so the CPU test suite
// can check it against the oracle.  Built by tests/test_cpu_host.py with g++.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <random>
#include <string>
#include <vector>

#include "host_setup.h"
#include "sigma.h"

using namespace hdd;

namespace {
struct Shim {
    DomainLayout L;
    InterfaceHost ih;
    std::string err;
};
const CsrF* pick(Shim* s, int kind, int level, int sub) {
    if (level < 0 || level >= s->ih.M) return nullptr;
    switch (kind) {
        case 0: return &s->ih.Arr[level];
        case 1: return (sub >= 0 && sub < s->ih.n_sub) ? &s->ih.Aii[level][sub] : nullptr;
        case 2: return (sub >= 0 && sub < s->ih.n_sub) ? &s->ih.Air[level][sub] : nullptr;
        case 3: return level < (int)s->ih.Prr.size() ? &s->ih.Prr[level] : nullptr;
        default: return nullptr;
    }
}
}  // namespace

extern "C" {

// Layout and interface system of a dense flag array; NULL on error (message in err).
void* shim_build(const int size[3], const int sub[3], int vlevels, int sigma_levels, const uint32_t* flags,
                 char* err, int errlen) {
    Shim* s = new Shim();
    try {
        Options o;
        for (int a = 0; a < 3; ++a) { o.size[a] = size[a]; o.sub[a] = sub[a]; }
        o.vlevels = vlevels;
        o.nvcycles = 1;
        o.interior = o.boundary = 1;
        o.sigma_levels = sigma_levels;
        o.sigma_smoothing = 3;
        o.sigma_mg = 1;
        build_layout(o, flags, s->L);
        build_interface(s->L, sigma_levels, s->ih);
        return s;
    } catch (const std::exception& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        delete s;
        return nullptr;
    }
}

// The product's two-level second-level interface system: every first-level
// subdomain's system (first-level planes made Dirichlet, boxes of sub/2),
// stacked block-diagonally.  NULL on error.
void* shim_build_second_level(const int size[3], const int sub[3], int sigma_levels, const uint32_t* flags,
                              char* err, int errlen) {
    Shim* s = new Shim();
    try {
        for (int a = 0; a < 3; ++a) { s->L.opt.size[a] = size[a]; s->L.opt.sub[a] = sub[a]; }
        s->L.opt.sigma_levels = sigma_levels;
        s->L.flags_in.assign(flags, flags + (size_t)size[0] * size[1] * size[2]);
        build_second_level(s->L, sub, sigma_levels, s->ih);
        return s;
    } catch (const std::exception& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        delete s;
        return nullptr;
    }
}

// 1 when the layout runs the whole-grid V-cycle (coarse levels couple boxes).
int shim_global_vcycle(void* h) { return static_cast<Shim*>(h)->L.global_vcycle ? 1 : 0; }

// Interface DOF count of a level.
int shim_num_interface(void* h, int level) {
    const InterfaceHost& ih = static_cast<Shim*>(h)->ih;
    return level >= 0 && level < (int)ih.n_iface.size() ? ih.n_iface[level] : -1;
}

void shim_free(void* h) { delete static_cast<Shim*>(h); }

// Factors a matrix of ncomp disconnected path graphs of csize vertices each
// (diagonal 2.5, off-diagonal -1, interleaved so that every component's
// vertices are spread through the numbering) and returns the relative
// residual of one solve; -1 on an exception.  Interface systems of sparse
// domains fall apart into many such pieces.
double shim_factor_components(int ncomp, int csize) {
    try {
        const int n = ncomp * csize;
        CsrF A;
        A.rows = A.cols = n;
        A.ptr.assign(1, 0);
        auto id = [&](int c, int k) { return k * ncomp + c; };  // component c, position k
        std::vector<int> comp_of(n), pos_of(n);
        for (int c = 0; c < ncomp; ++c)
            for (int k = 0; k < csize; ++k) { comp_of[id(c, k)] = c; pos_of[id(c, k)] = k; }
        for (int r = 0; r < n; ++r) {
            const int c = comp_of[r], k = pos_of[r];
            std::vector<std::pair<int, float>> e = {{r, 2.5f}};
            if (k > 0) e.push_back({id(c, k - 1), -1.0f});
            if (k + 1 < csize) e.push_back({id(c, k + 1), -1.0f});
            std::sort(e.begin(), e.end());
            for (auto& t : e) { A.col.push_back(t.first); A.val.push_back(t.second); }
            A.ptr.push_back((int)A.col.size());
        }
        SnFactor F;
        F.analyze(A, nullptr);
        F.factor(A, 1e-5);
        std::vector<double> b(n), x(n);
        for (int i = 0; i < n; ++i) b[i] = std::sin(0.37 * i);
        x = b;
        F.solve(x.data());
        double rn = 0, bn = 0;
        for (int r = 0; r < n; ++r) {
            double ax = 1e-5 * x[r];
            for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) ax += (double)A.val[p] * x[A.col[p]];
            rn += (ax - b[r]) * (ax - b[r]);
            bn += b[r] * b[r];
        }
        return std::sqrt(rn / bn);
    } catch (const std::exception&) {
        return -1.0;
    }
}

// FNV-1a digest of everything the GPU plans are built from: the interface
// matrices of every level and subdomain, and the solve blocks and L_RJ of the
// level-0 Arr factorisation and of every level-0 Aii factorisation.  Used to
// check that the host setup gives the same bits for any number of threads.
unsigned long long shim_setup_digest(void* h) {
    Shim* s = static_cast<Shim*>(h);
    unsigned long long d = 1469598103934665603ull;
    auto mix = [&](const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) d = (d ^ b[i]) * 1099511628211ull;
    };
    auto csr = [&](const CsrF& A) {
        mix(A.ptr.data(), A.ptr.size() * sizeof(int));
        mix(A.col.data(), A.col.size() * sizeof(int));
        mix(A.val.data(), A.val.size() * sizeof(float));
    };
    auto factor = [&](const CsrF& A, const std::vector<std::array<int, 3>>* xyz) {
        if (A.rows == 0) return;
        SnFactor F;
        F.analyze(A, xyz);
        F.factor(A, 1e-5);
        F.build_solve_blocks();
        mix(F.perm.data(), F.perm.size() * sizeof(int));
        for (const auto& v : F.Fw) mix(v.data(), v.size() * sizeof(double));
        for (const auto& v : F.Lrj) mix(v.data(), v.size() * sizeof(double));
    };
    const InterfaceHost& ih = s->ih;
    for (int l = 0; l < ih.M; ++l) {
        csr(ih.Arr[l]);
        if (l < (int)ih.Prr.size()) csr(ih.Prr[l]);
        for (int sd = 0; sd < ih.n_sub; ++sd) { csr(ih.Aii[l][sd]); csr(ih.Air[l][sd]); }
    }
    factor(ih.Arr[0], &ih.iface_xyz[0]);
    for (int sd = 0; sd < ih.n_sub; ++sd) factor(ih.Aii[0][sd], &ih.aii_xyz[0][sd]);
    return d;
}

// SPGrid page scatter / gather (hdd_set_domain_pages); 0 or the hdd_status.
int shim_pages_to_dense(const int size[3], long long n, const int32_t* origin, const uint32_t* flags,
                        const float* vals, uint32_t* dflags, float* dvals, char* err, int errlen) {
    try {
        pages_to_dense(size, n, origin, flags, dflags);
        pages_to_dense(size, n, origin, vals, dvals);
        return 0;
    } catch (const Error& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        return (int)e.status;
    }
}

int shim_dense_to_pages(const int size[3], long long n, const int32_t* origin, const float* dense, float* vals) {
    try {
        dense_to_pages(size, n, origin, dense, vals);
        return 0;
    } catch (const Error& e) {
        return (int)e.status;
    }
}

// Interface dump / reload (the reference's -iomode): 0 on success, else the
// hdd_status with its message in err.
int shim_write_interface(void* h, const char* dir, char* err, int errlen) {
    try {
        write_interface_dir(static_cast<Shim*>(h)->ih, dir);
        return 0;
    } catch (const Error& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        return (int)e.status;
    }
}

// A handle holding only a reloaded interface system (NULL on error).
void* shim_read_interface(const char* dir, char* err, int errlen) {
    Shim* s = new Shim();
    try {
        read_interface_dir(dir, s->ih);
        return s;
    } catch (const Error& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        delete s;
        return nullptr;
    }
}

// Checks the interface system of `sys` against the layout of `dom`.
int shim_check_interface(void* dom, void* sys, int sigma_levels, char* err, int errlen) {
    try {
        check_interface(static_cast<Shim*>(dom)->L, sigma_levels, static_cast<Shim*>(sys)->ih);
        return 0;
    } catch (const Error& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        return (int)e.status;
    }
}

// Interface DOF positions of level l: n entries (3 ints each) into out when
// out != NULL; sub < 0 selects the interface, else that subdomain's interior.
long long shim_positions(void* h, int l, int sub, int* out) {
    const InterfaceHost& ih = static_cast<Shim*>(h)->ih;
    if (l < 0 || l >= (int)ih.iface_xyz.size()) return -1;
    const std::vector<std::array<int, 3>>& p =
        sub < 0 ? ih.iface_xyz[l] : (sub < (int)ih.aii_xyz[l].size() ? ih.aii_xyz[l][sub] : ih.iface_xyz[l]);
    if (out)
        for (size_t i = 0; i < p.size(); ++i)
            for (int a = 0; a < 3; ++a) out[3 * i + a] = p[i][a];
    return (long long)p.size();
}

// Level-0 interface map: n cells into out (3 ints each) when out != NULL.
long long shim_interface_map(void* h, int* out) {
    const InterfaceHost& ih = static_cast<Shim*>(h)->ih;
    if (out)
        for (size_t i = 0; i < ih.iface_map.size(); ++i)
            for (int a = 0; a < 3; ++a) out[3 * i + a] = ih.iface_map[i][a];
    return (long long)ih.iface_map.size();
}

int shim_num_subdomains(void* h) { return static_cast<Shim*>(h)->ih.n_sub; }

// kind: 0 Arr, 1 Aii, 2 Air, 3 Prr.  shape = {rows, cols, nnz}; returns 0 on success.
int shim_matrix_shape(void* h, int kind, int level, int sub, int* shape) {
    const CsrF* m = pick(static_cast<Shim*>(h), kind, level, sub);
    if (!m) return 1;
    shape[0] = m->rows;
    shape[1] = m->cols;
    shape[2] = (int)m->col.size();
    return 0;
}

int shim_matrix_get(void* h, int kind, int level, int sub, int* ptr, int* col, double* val) {
    const CsrF* m = pick(static_cast<Shim*>(h), kind, level, sub);
    if (!m) return 1;
    for (size_t i = 0; i < m->ptr.size(); ++i) ptr[i] = m->ptr[i];
    for (size_t i = 0; i < m->col.size(); ++i) { col[i] = m->col[i]; val[i] = m->val[i]; }
    return 0;
}

// Factor (A + 1e-5 I) of one matrix with the supernodal Cholesky (geometric
// ordering when positions exist), solve for a random right-hand side on the
// host and return ||(A + 1e-5 I) x - b|| / ||b||; also checks that the explicit
// solve blocks reproduce the same solution (returned in *blocks_diff).
double shim_factor_check(void* h, int kind, int level, int sub, double* blocks_diff) {
    Shim* s = static_cast<Shim*>(h);
    const CsrF* m = pick(s, kind, level, sub);
    if (!m || (kind != 0 && kind != 1) || m->rows == 0) return -1.0;
    const std::vector<std::array<int, 3>>* xyz = nullptr;
    if (kind == 0 && level < (int)s->ih.iface_xyz.size() && (int)s->ih.iface_xyz[level].size() == m->rows)
        xyz = &s->ih.iface_xyz[level];
    if (kind == 1 && (int)s->ih.aii_xyz[level][sub].size() == m->rows) xyz = &s->ih.aii_xyz[level][sub];
    const double eps = 1e-5;
    SnFactor F;
    F.analyze(*m, xyz);
    F.factor(*m, eps);
    F.build_solve_blocks();
    const int n = m->rows;
    std::mt19937 rng(7);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<double> b(n), x(n);
    for (int i = 0; i < n; ++i) b[i] = U(rng);
    x = b;
    F.solve(x.data());
    double rn = 0, bn = 0;
    for (int r = 0; r < n; ++r) {
        double ax = eps * x[r];
        for (int p = m->ptr[r]; p < m->ptr[r + 1]; ++p) ax += (double)m->val[p] * x[m->col[p]];
        rn += (ax - b[r]) * (ax - b[r]);
        bn += b[r] * b[r];
    }
    // Same solve through the explicit blocks Fw = [Linv; -W] the GPU uses:
    // forward [y; v] = Fw f + [0; f_R], backward x_J = Fw^T [y; x_R].
    std::vector<double> f(n), y(n, 0.0), xn(n, 0.0);
    for (int i = 0; i < n; ++i) f[i] = b[F.perm[i]];
    const int ns = (int)F.col0.size();
    std::vector<std::vector<double>> upd(ns);
    std::vector<std::vector<int>> kids(ns);
    for (int j = 0; j < ns; ++j)
        if (F.parent[j] >= 0) kids[F.parent[j]].push_back(j);
    std::vector<int> pos(n, -1);
    for (int j = 0; j < ns; ++j) {
        const int nj = F.ncol[j], nr = (int)F.rows[j].size(), mm = nj + nr;
        std::vector<double> v(mm, 0.0);
        for (int a = 0; a < nj; ++a) { v[a] = f[F.col0[j] + a]; pos[F.col0[j] + a] = a; }
        for (int k = 0; k < nr; ++k) pos[F.rows[j][k]] = nj + k;
        for (int c : kids[j])
            for (size_t k = 0; k < F.rows[c].size(); ++k) v[pos[F.rows[c][k]]] += upd[c][k];
        const BlockVec& W = F.Fw[j];
        for (int r = 0; r < mm; ++r) {
            double acc = 0;
            for (int c = 0; c < nj; ++c) acc += W[(size_t)c * mm + r] * v[c];
            if (r < nj) y[F.col0[j] + r] = acc;
            else upd[j].push_back(v[r] + acc);
        }
    }
    for (int j = ns - 1; j >= 0; --j) {
        const int nj = F.ncol[j], nr = (int)F.rows[j].size(), mm = nj + nr;
        const BlockVec& W = F.Fw[j];
        for (int a = 0; a < nj; ++a) {
            double acc = 0;
            for (int r = 0; r < mm; ++r) {
                const double g = r < nj ? y[F.col0[j] + r] : xn[F.rows[j][r - nj]];
                acc += W[(size_t)a * mm + r] * g;
            }
            xn[F.col0[j] + a] = acc;
        }
    }
    double d = 0, xm = 0;
    for (int i = 0; i < n; ++i) {
        d = std::max(d, std::fabs(xn[i] - x[F.perm[i]]));
        xm = std::max(xm, std::fabs(x[F.perm[i]]));
    }
    *blocks_diff = xm > 0 ? d / xm : d;
    return std::sqrt(rn / bn);
}

// The supernodal solve plan of one interface solve (kind 0: Arr of level l;
// 1: Aii of all subdomains, concatenated), built as the sigma solver builds
// it and solved on the host front by front with the device kernels'
// arithmetic (PlanHost::emulate): x = plan solve of b.  Returns 0, or 1 on an
// exception.
int shim_plan_emulate(void* h, int kind, int level, const float* b, float* x) {
    Shim* s = static_cast<Shim*>(h);
    try {
        if (level < 0 || level >= s->ih.M || (kind != 0 && kind != 1)) return 1;
        std::vector<SnFactor> fs;
        PlanHost plan;
        interface_solve_plan(s->ih, kind, level, fs, plan);
        plan.emulate(b, x);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// Same plan: relative max-norm difference between its host solve (FP32
// coefficients) and the factorisations' own FP64 solve, for a random
// right-hand side; -1 on error.  *n gets the number of unknowns.
double shim_plan_check(void* h, int kind, int level, int* n) {
    Shim* s = static_cast<Shim*>(h);
    try {
        if (level < 0 || level >= s->ih.M || (kind != 0 && kind != 1)) return -1.0;
        std::vector<SnFactor> fs;
        PlanHost plan;
        interface_solve_plan(s->ih, kind, level, fs, plan);
        *n = plan.n;
        std::mt19937 rng(11);
        std::uniform_real_distribution<float> U(-1.0f, 1.0f);
        std::vector<float> b(plan.n), x(plan.n, 0.0f);
        for (float& v : b) v = U(rng);
        plan.emulate(b.data(), x.data());
        std::vector<double> ref(b.begin(), b.end());
        int off = 0;  // unknowns are concatenated in factor order (empty factors add none)
        for (const SnFactor& F : fs) {
            F.solve(ref.data() + off);
            off += F.n;
        }
        double dmax = 0, rmax = 0;
        for (int i = 0; i < plan.n; ++i) {
            dmax = std::max(dmax, std::fabs((double)x[i] - ref[i]));
            rmax = std::max(rmax, std::fabs(ref[i]));
        }
        return rmax > 0 ? dmax / rmax : dmax;
    } catch (const std::exception&) {
        return -1.0;
    }
}
}
