// ORACLE (test infrastructure only) -- flag construction and V-cycle stencils.
// See oracle_core.h for the scope and parity status of this restatement.
#include "oracle_core.h"

#include <algorithm>

namespace oracle {

static inline int popcount6(uint32_t f) { return __builtin_popcount((f >> 20) & 0x3fu); }

void flag_faces(const Dims& d, uint32_t* f) {
    const uint32_t nb_mask = ACTIVE | INTERFACE | DIRICHLET;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d.n[0]; ++i)
        for (int j = 0; j < d.n[1]; ++j)
            for (int k = 0; k < d.n[2]; ++k) {
                uint32_t& fl = f[d.at(i, j, k)];
                if (!(fl & (ACTIVE | INTERFACE))) continue;
                for (int face = 0; face < 6; ++face) {
                    uint32_t nf = flag_at(d, f, i + FACE_D[face][0], j + FACE_D[face][1],
                                          k + FACE_D[face][2]);
                    if (nf & nb_mask) fl |= (FACE_MX << face);
                }
            }
}

void flag_boundary(const Dims& d, uint32_t* f) {
    // Offsets with 1 <= |dx|+|dy|+|dz| <= 3.
    std::vector<std::array<int, 3>> offs;
    for (int a = -3; a <= 3; ++a)
        for (int b = -3; b <= 3; ++b)
            for (int c = -3; c <= 3; ++c) {
                int m = std::abs(a) + std::abs(b) + std::abs(c);
                if (m >= 1 && m <= 3) offs.push_back({a, b, c});
            }
    std::vector<uint8_t> mark(d.count(), 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d.n[0]; ++i)
        for (int j = 0; j < d.n[1]; ++j)
            for (int k = 0; k < d.n[2]; ++k) {
                uint32_t fl = f[d.at(i, j, k)];
                if (!(fl & ACTIVE)) continue;
                for (auto& o : offs) {
                    uint32_t nf = flag_at(d, f, i + o[0], j + o[1], k + o[2]);
                    if (nf == 0u || (nf & (INTERFACE | DIRICHLET))) { mark[d.at(i, j, k)] = 1; break; }
                }
            }
    for (size_t x = 0; x < d.count(); ++x)
        if (mark[x]) f[x] |= BOUNDARY;
}

void number_of_subdomains(const int size[3], const int sub[3], int out[3]) {
    for (int a = 0; a < 3; ++a) {
        out[a] = (size[a] - 1) / sub[a];
        if ((size[a] - 1) % sub[a]) ++out[a];
    }
}

void divide_domain(const Dims& d, uint32_t* f, const int sub[3]) {
    int ns[3];
    number_of_subdomains(d.n, sub, ns);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d.n[0]; ++i)
        for (int j = 0; j < d.n[1]; ++j)
            for (int k = 0; k < d.n[2]; ++k) {
                uint32_t& fl = f[d.at(i, j, k)];
                if (!(fl & ACTIVE)) continue;
                if (i % sub[0] == 0 || j % sub[1] == 0 || k % sub[2] == 0) {
                    fl -= ACTIVE;
                    fl |= INTERFACE;
                } else {
                    int id = ((i / sub[0]) * ns[1] + (j / sub[1])) * ns[2] + (k / sub[2]);
                    fl |= (uint32_t)(id + 1);
                }
            }
}

// SPGrid_Mask<4,2,3> (PB/Common_Libraries/SPGrid/Core/SPGrid_Mask.h): 4 x 8 x 8-cell
// pages whose coordinates are bit-interleaved above the 4 KB page, cells of a
// page x-slowest.  The address of page (a, b, c), as a sort key.
// Page bit k of x sits at address bit 12 + 3k, of z at 13 + 3k, of y at 14 + 3k.
static uint64_t page_address(int a, int b, int c) {
    const uint64_t v[3] = {(uint64_t)a, (uint64_t)b, (uint64_t)c};
    const int lane[3] = {0, 2, 1};
    uint64_t key = 0;
    for (int bit = 0; bit < 17; ++bit)
        for (int axis = 0; axis < 3; ++axis)
            if (v[axis] >> bit & 1u) key |= 1ull << (12 + 3 * bit + lane[axis]);
    return key;
}

void downsample_topology(const Dims& fd, const uint32_t* ff, const Dims& cd, uint32_t* cf) {
    // SPGrid_V_Cycle_Topology.h:35-67 (Topology_Downsample): the fine cells are
    // visited page by page in address order, x-slowest inside a page; coarse
    // cell (f+1)/2.  An unset coarse cell (no Dirichlet, Active or Interface
    // bit) becomes Active on an Active child, Dirichlet on a Dirichlet child,
    // and stays unset on an Interface child; a set one becomes Dirichlet on a
    // Dirichlet or Interface child.
    std::fill(cf, cf + cd.count(), 0u);
    const int np[3] = {(fd.n[0] + 3) / 4, (fd.n[1] + 7) / 8, (fd.n[2] + 7) / 8};
    std::vector<std::pair<uint64_t, long long>> pages;
    for (int a = 0; a < np[0]; ++a)
        for (int b = 0; b < np[1]; ++b)
            for (int c = 0; c < np[2]; ++c) pages.push_back({page_address(a, b, c), ((long long)a * np[1] + b) * np[2] + c});
    std::sort(pages.begin(), pages.end());
    for (const auto& pg : pages) {
        const int a = (int)(pg.second / ((long long)np[1] * np[2])), b = (int)(pg.second / np[2] % np[1]),
                  c = (int)(pg.second % np[2]);
        for (int i = 4 * a; i < 4 * a + 4 && i < fd.n[0]; ++i)
            for (int j = 8 * b; j < 8 * b + 8 && j < fd.n[1]; ++j)
                for (int k = 8 * c; k < 8 * c + 8 && k < fd.n[2]; ++k) {
                    const uint32_t fl = ff[fd.at(i, j, k)];
                    uint32_t& o = cf[cd.at((i + 1) / 2, (j + 1) / 2, (k + 1) / 2)];
                    if (!(o & (DIRICHLET | ACTIVE | INTERFACE))) {
                        if (fl & ACTIVE) o |= ACTIVE;
                        else if (fl & (DIRICHLET | INTERFACE)) o |= (fl & DIRICHLET);
                        continue;
                    }
                    if (fl & (DIRICHLET | INTERFACE)) o = DIRICHLET;
                }
    }
}

template <class T>
void residual(const Dims& d, const uint32_t* f, const T* u, T* r, const T* b) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d.n[0]; ++i)
        for (int j = 0; j < d.n[1]; ++j)
            for (int k = 0; k < d.n[2]; ++k) {
                size_t x = d.at(i, j, k);
                uint32_t fl = f[x];
                if (!(fl & ACTIVE)) continue;
                T c = u[x], result = 0;
                for (int face = 0; face < 6; ++face)
                    if (fl & (FACE_MX << face)) {
                        T nb = val_at(d, u, i + FACE_D[face][0], j + FACE_D[face][1], k + FACE_D[face][2]);
                        result -= (nb - c);
                    }
                r[x] = b[x] - result;
            }
}

template <class T>
void correction(const Dims& d, const uint32_t* f, T* u, const T* r, bool write_interior,
                bool write_boundary) {
    const T omega = (T)(2. / 3.);
#pragma omp parallel for schedule(static)
    for (long x = 0; x < (long)d.count(); ++x) {
        uint32_t fl = f[x];
        uint32_t t = fl & (ACTIVE | BOUNDARY);
        if (t == ACTIVE) { if (!write_interior) continue; }
        else if (t == (ACTIVE | BOUNDARY)) { if (!write_boundary) continue; }
        else continue;
        int fc = popcount6(fl);
        if (fc == 0) abort();  // PHYSBAM_ASSERT(face_count > 0)
        u[x] += (omega / (T)fc) * r[x];
    }
}

template <class T>
void restriction(const Dims& cd, const uint32_t* cf, T* cb, const Dims& fd, const T* fr) {
    const float s1[4] = {(float)(1. / 8.), (float)(3. / 8.), (float)(3. / 8.), (float)(1. / 8.)};
    float sc[4][4][4];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 4; ++k) sc[i][j][k] = s1[i] * s1[j] * s1[k];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < cd.n[0]; ++i)
        for (int j = 0; j < cd.n[1]; ++j)
            for (int k = 0; k < cd.n[2]; ++k) {
                size_t x = cd.at(i, j, k);
                if (!(cf[x] & ACTIVE)) continue;
                T acc = 0;
                for (int i2 = 0; i2 < 4; ++i2)
                    for (int j2 = 0; j2 < 4; ++j2)
                        for (int k2 = 0; k2 < 4; ++k2)
                            acc += sc[i2][j2][k2] *
                                   val_at(fd, fr, 2 * i - 2 + i2, 2 * j - 2 + j2, 2 * k - 2 + k2);
                cb[x] = acc;
            }
}

template <class T>
void prolongation(const Dims& fd, const uint32_t* ff, T* fu, const Dims& cd, const T* cu) {
    const float s1[2] = {(float)(3. / 4.f), (float)(1. / 4.f)};
    float sc[2][2][2];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int k = 0; k < 2; ++k) sc[i][j][k] = s1[i] * s1[j] * s1[k] * 4.0f;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < fd.n[0]; ++i)
        for (int j = 0; j < fd.n[1]; ++j)
            for (int k = 0; k < fd.n[2]; ++k) {
                size_t x = fd.at(i, j, k);
                if (!(ff[x] & ACTIVE)) continue;
                int c[3] = {(i + 1) / 2, (j + 1) / 2, (k + 1) / 2};
                int p[3] = {1 - (i - (2 * c[0] - 1)), 1 - (j - (2 * c[1] - 1)), 1 - (k - (2 * c[2] - 1))};
                T acc = fu[x];
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b)
                        for (int e = 0; e < 2; ++e)
                            acc += sc[a ^ p[0]][b ^ p[1]][e ^ p[2]] *
                                   val_at(cd, cu, c[0] + a - p[0], c[1] + b - p[1], c[2] + e - p[2]);
                fu[x] = acc;
            }
}

template <class T>
static void smooth(const Dims& d, const uint32_t* f, T* u, T* r, const T* b, bool wi, bool wb) {
    residual(d, f, u, r, b);
    correction(d, f, u, r, wi, wb);
}

template <class T>
void v_cycle(std::vector<MGLevel<T>>& lv, T* u0, T* r0, const T* b0, int interior_itr,
             int boundary_itr) {
    const int L = (int)lv.size();
    auto U = [&](int l) { return l == 0 ? u0 : lv[l].u.data(); };
    auto R = [&](int l) { return l == 0 ? r0 : lv[l].r.data(); };
    auto B = [&](int l) { return l == 0 ? const_cast<T*>(b0) : lv[l].b.data(); };
    for (int l = 0; l < L - 1; ++l) {
        const Dims& d = lv[l].d;
        const uint32_t* f = lv[l].flags.data();
        for (int i = 0; i < boundary_itr; ++i) smooth(d, f, U(l), R(l), B(l), false, true);
        for (int i = 0; i < interior_itr; ++i) smooth(d, f, U(l), R(l), B(l), true, false);
        for (int i = 0; i < boundary_itr; ++i) smooth(d, f, U(l), R(l), B(l), false, true);
        residual(d, f, U(l), R(l), B(l));
        std::fill(lv[l + 1].u.begin(), lv[l + 1].u.end(), T(0));
        restriction(lv[l + 1].d, lv[l + 1].flags.data(), B(l + 1), d, R(l));
    }
    {
        const Dims& d = lv[L - 1].d;
        const uint32_t* f = lv[L - 1].flags.data();
        residual(d, f, U(L - 1), R(L - 1), B(L - 1));
        for (int i = 0; i < 200; ++i) smooth(d, f, U(L - 1), R(L - 1), B(L - 1), true, true);
        residual(d, f, U(L - 1), R(L - 1), B(L - 1));
    }
    for (int l = L - 2; l >= 0; --l) {
        const Dims& d = lv[l].d;
        const uint32_t* f = lv[l].flags.data();
        prolongation(d, f, U(l), lv[l + 1].d, U(l + 1));
        for (int i = 0; i < boundary_itr; ++i) smooth(d, f, U(l), R(l), B(l), false, true);
        for (int i = 0; i < interior_itr; ++i) smooth(d, f, U(l), R(l), B(l), true, false);
        for (int i = 0; i < boundary_itr; ++i) smooth(d, f, U(l), R(l), B(l), false, true);
    }
}

template <class T>
void laplace_ai(const Dims& d, const uint32_t* f, const T* u, T* lu) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d.n[0]; ++i)
        for (int j = 0; j < d.n[1]; ++j)
            for (int k = 0; k < d.n[2]; ++k) {
                size_t x = d.at(i, j, k);
                uint32_t fl = f[x];
                if (!(fl & (ACTIVE | INTERFACE))) continue;
                double c = (double)u[x], result = 0.;
                for (int face = 0; face < 6; ++face)
                    if (fl & (FACE_MX << face)) {
                        double nb = (double)val_at(d, u, i + FACE_D[face][0], j + FACE_D[face][1],
                                                   k + FACE_D[face][2]);
                        result -= (nb - c);
                    }
                lu[x] = (T)result;
            }
}

template <class T>
void laplace_ri(const Dims& d, const uint32_t* f, const T* u, T* lu) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d.n[0]; ++i)
        for (int j = 0; j < d.n[1]; ++j)
            for (int k = 0; k < d.n[2]; ++k) {
                size_t x = d.at(i, j, k);
                uint32_t fl = f[x];
                if (!(fl & INTERFACE)) continue;
                double result = 0.;
                for (int face = 0; face < 6; ++face)
                    if (fl & (FACE_MX << face)) {
                        int a = i + FACE_D[face][0], b = j + FACE_D[face][1], c = k + FACE_D[face][2];
                        if (flag_at(d, f, a, b, c) & ACTIVE) result -= (double)u[d.at(a, b, c)];
                    }
                lu[x] -= (T)result;
            }
}

static inline bool on_plane(int i, int j, int k, const int sub[3]) {
    return i % sub[0] == 0 || j % sub[1] == 0 || k % sub[2] == 0;
}

template <class T>
void laplace_ri_subdomain(const Dims& d, const uint32_t* f, const T* u, T* lu, const int sub[3]) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d.n[0]; ++i)
        for (int j = 0; j < d.n[1]; ++j)
            for (int k = 0; k < d.n[2]; ++k) {
                size_t x = d.at(i, j, k);
                uint32_t fl = f[x];
                if (!(fl & (ACTIVE | INTERFACE)) || !on_plane(i, j, k, sub)) continue;
                double result = 0.;
                for (int face = 0; face < 6; ++face)
                    if (fl & (FACE_MX << face)) {
                        int a = i + FACE_D[face][0], b = j + FACE_D[face][1], c = k + FACE_D[face][2];
                        if (!(flag_at(d, f, a, b, c) & (ACTIVE | INTERFACE)) || on_plane(a, b, c, sub)) continue;
                        result -= (double)u[d.at(a, b, c)];
                    }
                lu[x] -= (T)result;
            }
}

template <class T>
void laplace_ir_subdomain(const Dims& d, const uint32_t* f, const T* u, T* lu, const int sub[3]) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d.n[0]; ++i)
        for (int j = 0; j < d.n[1]; ++j)
            for (int k = 0; k < d.n[2]; ++k) {
                size_t x = d.at(i, j, k);
                uint32_t fl = f[x];
                if (!(fl & (ACTIVE | INTERFACE)) || on_plane(i, j, k, sub)) continue;
                double result = 0.;
                for (int face = 0; face < 6; ++face)
                    if (fl & (FACE_MX << face)) {
                        int a = i + FACE_D[face][0], b = j + FACE_D[face][1], c = k + FACE_D[face][2];
                        if (!(flag_at(d, f, a, b, c) & (ACTIVE | INTERFACE)) || !on_plane(a, b, c, sub)) continue;
                        result -= (double)u[d.at(a, b, c)];
                    }
                lu[x] = -(T)result;
            }
}

#define ORACLE_INST(T)                                                                          \
    template void residual<T>(const Dims&, const uint32_t*, const T*, T*, const T*);            \
    template void correction<T>(const Dims&, const uint32_t*, T*, const T*, bool, bool);        \
    template void restriction<T>(const Dims&, const uint32_t*, T*, const Dims&, const T*);      \
    template void prolongation<T>(const Dims&, const uint32_t*, T*, const Dims&, const T*);     \
    template void v_cycle<T>(std::vector<MGLevel<T>>&, T*, T*, const T*, int, int);             \
    template void laplace_ai<T>(const Dims&, const uint32_t*, const T*, T*);                    \
    template void laplace_ri<T>(const Dims&, const uint32_t*, const T*, T*);                    \
    template void laplace_ri_subdomain<T>(const Dims&, const uint32_t*, const T*, T*, const int*); \
    template void laplace_ir_subdomain<T>(const Dims&, const uint32_t*, const T*, T*, const int*);
ORACLE_INST(float)
ORACLE_INST(double)

}  // namespace oracle
