// ORACLE (test infrastructure only) -- interface system and sigma V-cycle.
// See oracle_interface.h for what is restated and what stands in for the
// reference's third-party solvers.
#include "oracle_interface.h"

#include <cstdlib>
#include <chrono>
#include <string>
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <functional>
#include <unordered_set>

namespace oracle {

// --------------------------------------------------------------------------
// Csr helpers
// --------------------------------------------------------------------------
template <class T>
void Csr<T>::spmv(const T* x, T* y) const {
    for (int r = 0; r < rows; ++r) {
        T acc = 0;
        for (int p = ptr[r]; p < ptr[r + 1]; ++p) acc += val[p] * x[col[p]];
        y[r] = acc;
    }
}
template <class T>
void Csr<T>::spmv_t_add(const T* x, T* y) const {
    for (int r = 0; r < rows; ++r) {
        T xr = x[r];
        for (int p = ptr[r]; p < ptr[r + 1]; ++p) y[col[p]] += val[p] * xr;
    }
}

template <class T>
static Csr<T> csr_from_map(int rows, int cols, const std::unordered_map<uint64_t, T>& m) {
    // CPU/Interface_Solver/INTERFACE_MATRIX_GENERATOR.h:660-730 (Convert_To_Eigen):
    // explicit zeros are dropped, duplicates were already summed per key.
    std::vector<std::pair<uint64_t, T>> e;
    e.reserve(m.size());
    for (auto& kv : m)
        if (kv.second != T(0)) e.push_back(kv);
    std::sort(e.begin(), e.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    Csr<T> c;
    c.rows = rows;
    c.cols = cols;
    c.ptr.assign(rows + 1, 0);
    for (auto& kv : e) c.ptr[(int)(kv.first >> 32) + 1]++;
    for (int r = 0; r < rows; ++r) c.ptr[r + 1] += c.ptr[r];
    c.col.resize(e.size());
    c.val.resize(e.size());
    for (size_t i = 0; i < e.size(); ++i) {
        c.col[i] = (int)(uint32_t)e[i].first;
        c.val[i] = e[i].second;
    }
    return c;
}

// --------------------------------------------------------------------------
// Sparse Cholesky (stands in for MKL PARDISO phases 11/22/33)
// --------------------------------------------------------------------------

// Nested dissection by breadth-first level structures: the middle level of a
// pseudo-peripheral BFS is the separator; the two sides are ordered first.
static void nd_order(int n, const std::vector<int>& adjp, const std::vector<int>& adji,
                     std::vector<int>& order, std::vector<int>& starts) {
    starts.clear();
    std::vector<int> part(n, 0), level(n, -1), queue(n);
    int next_part = 1;
    order.clear();
    order.reserve(n);
    struct Job { std::vector<int> verts; int pid; };
    std::vector<Job> stack;
    // Output is assembled back-to-front: separators are appended to "tail" lists.
    std::vector<std::vector<int>> out_blocks;
    std::function<void(std::vector<int>&, int)> rec;
    auto bfs = [&](int src, int pid, std::vector<int>& visited) -> int {
        int qh = 0, qt = 0;
        queue[qt++] = src;
        level[src] = 0;
        visited.push_back(src);
        int last = src;
        while (qh < qt) {
            int v = queue[qh++];
            last = v;
            for (int p = adjp[v]; p < adjp[v + 1]; ++p) {
                int w = adji[p];
                if (part[w] != pid || level[w] >= 0) continue;
                level[w] = level[v] + 1;
                queue[qt++] = w;
                visited.push_back(w);
            }
        }
        return last;
    };
    rec = [&](std::vector<int>& verts, int pid) {
        if (verts.size() <= 48) {
            starts.push_back((int)order.size());
            for (int v : verts) order.push_back(v);
            return;
        }
        std::vector<int> comp;
        int far = bfs(verts[0], pid, comp);
        for (int v : comp) level[v] = -1;
        if (comp.size() < verts.size()) {
            // Disconnected: the components one after another, as peeling off
            // the reached component and recursing on the rest would order
            // them, but found in one pass (linear time, no recursion per
            // component): component i in BFS order from its first vertex,
            // the remaining components as one block once they hold at most 48
            // vertices, the last component from its vertices in verts order.
            std::vector<std::vector<int>> comps;
            std::vector<int> ids;
            ids.push_back(next_part++);
            for (int v : comp) part[v] = ids.back();
            comps.push_back(std::move(comp));
            for (int v : verts) {
                if (part[v] != pid) continue;
                std::vector<int> c;
                bfs(v, pid, c);
                for (int w : c) level[w] = -1;
                ids.push_back(next_part++);
                for (int w : c) part[w] = ids.back();
                comps.push_back(std::move(c));
            }
            size_t remaining = verts.size();
            for (size_t i = 0; i < comps.size(); ++i) {
                if (i > 0 && remaining <= 48) {
                    starts.push_back((int)order.size());
                    for (int v : verts)
                        if (part[v] >= ids[i] && part[v] <= ids.back()) order.push_back(v);
                    return;
                }
                if (i > 0 && i + 1 == comps.size()) {
                    std::vector<int> last;
                    for (int v : verts)
                        if (part[v] == ids[i]) last.push_back(v);
                    rec(last, ids[i]);
                } else {
                    rec(comps[i], ids[i]);
                }
                remaining -= comps[i].size();
            }
            return;
        }
        comp.clear();
        bfs(far, pid, comp);
        int h = 0;
        for (int v : comp) h = std::max(h, level[v]);
        if (h < 2) {
            for (int v : comp) level[v] = -1;
            starts.push_back((int)order.size());
            for (int v : verts) order.push_back(v);
            return;
        }
        std::vector<int> cnt(h + 1, 0);
        for (int v : comp) cnt[level[v]]++;
        int half = (int)verts.size() / 2, acc = 0, m = 1;
        for (int l = 0; l <= h; ++l) {
            acc += cnt[l];
            if (acc >= half) { m = std::max(1, std::min(l, h - 1)); break; }
        }
        std::vector<int> A, S, B;
        for (int v : comp) {
            if (level[v] < m) A.push_back(v);
            else if (level[v] == m) S.push_back(v);
            else B.push_back(v);
            level[v] = -1;
        }
        int pa = next_part++, pb = next_part++;
        for (int v : A) part[v] = pa;
        for (int v : B) part[v] = pb;
        for (int v : S) part[v] = -1;
        rec(A, pa);
        rec(B, pb);
        starts.push_back((int)order.size());
        for (int v : S) order.push_back(v);
    };
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i) all[i] = i;
    rec(all, 0);
}

// Nested dissection by median planes through DOF positions: for each axis
// the cut is at the median position and the separator is the smaller
// one-sided boundary layer; the axis with the smallest separator wins.  Falls
// back to the level-structure split when no axis separates.
static void nd_order_xyz(int n, const std::vector<int>& adjp, const std::vector<int>& adji,
                         const std::vector<std::array<int, 3>>& xyz, std::vector<int>& order,
                         std::vector<int>& starts) {
    starts.clear();
    std::vector<int> part(n, 0);
    int next_part = 1;
    order.clear();
    order.reserve(n);
    std::function<void(std::vector<int>&, int)> rec = [&](std::vector<int>& verts, int pid) {
        if (verts.size() <= 48) {
            starts.push_back((int)order.size());
            for (int v : verts) order.push_back(v);
            return;
        }
        int best_axis = -1, best_cut = 0, best_side = 0;
        size_t best_sep = 0;
        std::vector<int> pos(verts.size());
        for (int ax = 0; ax < 3; ++ax) {
            for (size_t i = 0; i < verts.size(); ++i) pos[i] = xyz[verts[i]][ax];
            const size_t mid = pos.size() / 2;
            std::nth_element(pos.begin(), pos.begin() + mid, pos.end());
            int cut = pos[mid];
            size_t nleft = 0, nle = 0;
            for (int v : verts) { nleft += xyz[v][ax] < cut; nle += xyz[v][ax] <= cut; }
            if (nleft == 0) {
                if (nle == verts.size()) continue;
                cut += 1;
            }
            size_t sl = 0, sr = 0;
            for (int v : verts) {
                const bool left = xyz[v][ax] < cut;
                for (int p = adjp[v]; p < adjp[v + 1]; ++p) {
                    const int w = adji[p];
                    if (part[w] == pid && (xyz[w][ax] < cut) != left) { (left ? sl : sr)++; break; }
                }
            }
            const size_t sep = std::min(sl, sr);
            if (best_axis < 0 || sep < best_sep) { best_axis = ax; best_sep = sep; best_cut = cut; best_side = sl <= sr ? 0 : 1; }
        }
        if (best_axis < 0) {
            starts.push_back((int)order.size());
            for (int v : verts) order.push_back(v);
            return;
        }
        std::vector<int> A, S, B;
        for (int v : verts) {
            const bool left = xyz[v][best_axis] < best_cut;
            bool boundary = false;
            if ((best_side == 0) == left)
                for (int p = adjp[v]; p < adjp[v + 1] && !boundary; ++p) {
                    const int w = adji[p];
                    if (part[w] == pid && (xyz[w][best_axis] < best_cut) != left) boundary = true;
                }
            if (boundary) S.push_back(v);
            else if (left) A.push_back(v);
            else B.push_back(v);
        }
        const int pa = next_part++, pb = next_part++;
        for (int v : A) part[v] = pa;
        for (int v : B) part[v] = pb;
        for (int v : S) part[v] = -1;
        rec(A, pa);
        rec(B, pb);
        starts.push_back((int)order.size());
        for (int v : S) order.push_back(v);
    };
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i) all[i] = i;
    rec(all, 0);
}

template <class T>
void Cholesky::factor(const Csr<T>& A, double eps, const std::vector<std::array<int, 3>>* xyz) {
    n = A.rows;
    // Symmetric pattern without the diagonal.
    std::vector<std::vector<int>> nb(n);
    for (int r = 0; r < n; ++r)
        for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) {
            int c = A.col[p];
            if (c == r) continue;
            nb[r].push_back(c);
            nb[c].push_back(r);
        }
    std::vector<int> adjp(n + 1, 0), adji;
    for (int r = 0; r < n; ++r) {
        std::sort(nb[r].begin(), nb[r].end());
        nb[r].erase(std::unique(nb[r].begin(), nb[r].end()), nb[r].end());
        adjp[r + 1] = adjp[r] + (int)nb[r].size();
    }
    adji.reserve(adjp[n]);
    for (int r = 0; r < n; ++r) adji.insert(adji.end(), nb[r].begin(), nb[r].end());
    // Each group the dissection emits (a leaf block or a separator) is one
    // supernode; the groups come children first.
    std::vector<int> starts;
    if (xyz && (int)xyz->size() == n) nd_order_xyz(n, adjp, adji, *xyz, perm, starts);
    else nd_order(n, adjp, adji, perm, starts);
    starts.push_back(n);
    std::vector<int> iperm(n);
    for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
    const int ns = (int)starts.size() - 1;
    std::vector<int> sn_of(n);
    for (int j = 0; j < ns; ++j)
        for (int c = starts[j]; c < starts[j + 1]; ++c) sn_of[c] = j;
    // Lower triangle of P (A + eps I) P^T by (new) columns.
    std::vector<std::vector<std::pair<int, double>>> lowcol(n);
    for (int r = 0; r < n; ++r)
        for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) {
            const int i = iperm[r], k = iperm[A.col[p]];
            if (i >= k) lowcol[k].push_back({i, (double)A.val[p]});
        }
    for (int k = 0; k < n; ++k) lowcol[k].push_back({k, eps});
    // Symbolic: rows below each supernode, and the assembly tree.
    std::vector<std::vector<int>> rows(ns);
    std::vector<std::vector<int>> kids(ns);
    std::vector<int> mark(n, -1);
    for (int j = 0; j < ns; ++j) {
        const int last = starts[j + 1] - 1;
        std::vector<int>& R = rows[j];
        for (int c = starts[j]; c <= last; ++c)
            for (auto& e : lowcol[c])
                if (e.first > last && mark[e.first] != j) { mark[e.first] = j; R.push_back(e.first); }
        for (int c : kids[j])
            for (int i : rows[c])
                if (i > last && mark[i] != j) { mark[i] = j; R.push_back(i); }
        std::sort(R.begin(), R.end());
        if (!R.empty()) kids[sn_of[R[0]]].push_back(j);
    }
    // Numeric: multifrontal, dense fronts (column-major, lower triangle).
    std::vector<std::vector<double>> upd(ns);
    std::vector<std::vector<double>> Lcols(ns);     // nj x m panel of L^T rows: column a of L in block j
    std::vector<int> pos(n, -1);
    for (int j = 0; j < ns; ++j) {
        const int c0 = starts[j], nj = starts[j + 1] - c0, nr = (int)rows[j].size(), m = nj + nr;
        std::vector<double> F((size_t)m * m, 0.0);
        for (int a = 0; a < nj; ++a) pos[c0 + a] = a;
        for (int k = 0; k < nr; ++k) pos[rows[j][k]] = nj + k;
        for (int a = 0; a < nj; ++a)
            for (auto& e : lowcol[c0 + a]) F[(size_t)a * m + pos[e.first]] += e.second;
        for (int c : kids[j]) {
            const std::vector<int>& rc = rows[c];
            const int mc = (int)rc.size();
            const std::vector<double>& U = upd[c];
            for (int b = 0; b < mc; ++b) {
                const int pb = pos[rc[b]];
                for (int a = b; a < mc; ++a) F[(size_t)pb * m + pos[rc[a]]] += U[(size_t)b * mc + a];
            }
            std::vector<double>().swap(upd[c]);
        }
        // Partial Cholesky of the first nj columns, right-looking in panels of
        // 64 columns: a panel is factored with updates to its own columns,
        // then the columns right of it are updated once with the whole panel.
        // Every entry receives its updates in increasing column order, as in
        // the column-at-a-time form, with 64x less memory traffic.
        constexpr int PB = 64;
        for (int p0 = 0; p0 < nj; p0 += PB) {
            const int pe = std::min(nj, p0 + PB);
            for (int a = p0; a < pe; ++a) {
                double* col = &F[(size_t)a * m];
                const double d = col[a];
                if (!(d > 0)) throw std::runtime_error("oracle Cholesky: matrix not positive definite");
                const double ld = std::sqrt(d);
                col[a] = ld;
                for (int i = a + 1; i < m; ++i) col[i] /= ld;
                for (int b = a + 1; b < pe; ++b) {
                    const double lb = col[b];
                    if (lb == 0.0) continue;
                    double* cb = &F[(size_t)b * m];
                    for (int i = b; i < m; ++i) cb[i] -= col[i] * lb;
                }
            }
#pragma omp parallel for schedule(dynamic, 16) if (m - pe > 128)
            for (int b = pe; b < m; ++b) {
                double* cb = &F[(size_t)b * m];
                for (int a = p0; a < pe; ++a) {
                    const double lb = F[(size_t)a * m + b];
                    if (lb == 0.0) continue;
                    const double* ca = &F[(size_t)a * m];
                    for (int i = b; i < m; ++i) cb[i] -= ca[i] * lb;
                }
            }
        }
        // Update matrix for the parent: the trailing nr x nr lower block.
        if (nr > 0) {
            std::vector<double>& U = upd[j];
            U.assign((size_t)nr * nr, 0.0);
            for (int b = 0; b < nr; ++b)
                for (int a = b; a < nr; ++a) U[(size_t)b * nr + a] = F[(size_t)(nj + b) * m + nj + a];
        }
        std::vector<double>& Lc = Lcols[j];
        Lc.assign((size_t)nj * m, 0.0);
        for (int a = 0; a < nj; ++a)
            for (int i = a; i < m; ++i) Lc[(size_t)a * m + i] = F[(size_t)a * m + i];
    }
    // CSC of L, diagonal first in each column.
    Lp.assign(n + 1, 0);
    for (int j = 0; j < ns; ++j) {
        const int c0 = starts[j], nj = starts[j + 1] - c0, nr = (int)rows[j].size();
        for (int a = 0; a < nj; ++a) Lp[c0 + a + 1] = (nj - a) + nr;
    }
    for (int k = 0; k < n; ++k) Lp[k + 1] += Lp[k];
    Li.resize(Lp[n]);
    Lx.resize(Lp[n]);
    for (int j = 0; j < ns; ++j) {
        const int c0 = starts[j], nj = starts[j + 1] - c0, nr = (int)rows[j].size(), m = nj + nr;
        const std::vector<double>& Lc = Lcols[j];
        for (int a = 0; a < nj; ++a) {
            int p = Lp[c0 + a];
            for (int i = a; i < nj; ++i) { Li[p] = c0 + i; Lx[p] = Lc[(size_t)a * m + i]; ++p; }
            for (int k = 0; k < nr; ++k) { Li[p] = rows[j][k]; Lx[p] = Lc[(size_t)a * m + nj + k]; ++p; }
        }
    }
}

void Cholesky::solve(double* b) const {
    std::vector<double> y(n);
    for (int i = 0; i < n; ++i) y[i] = b[perm[i]];
    for (int j = 0; j < n; ++j) {
        y[j] /= Lx[Lp[j]];
        double yj = y[j];
        for (int p = Lp[j] + 1; p < Lp[j + 1]; ++p) y[Li[p]] -= Lx[p] * yj;
    }
    for (int j = n - 1; j >= 0; --j) {
        double acc = y[j];
        for (int p = Lp[j] + 1; p < Lp[j + 1]; ++p) acc -= Lx[p] * y[Li[p]];
        y[j] = acc / Lx[Lp[j]];
    }
    for (int i = 0; i < n; ++i) b[perm[i]] = y[i];
}

// --------------------------------------------------------------------------
// Adaptive hierarchy (CPU/Interface_Solver/INTERFACE_MATRIX_GENERATOR.h)
// --------------------------------------------------------------------------

// CPU/Interface_Solver/ADAPTIVE_SUBDOMAIN_POISSON_FLAGS.h:11-26.
enum : uint32_t {
    U_NODE_ACTIVE = 0x10u,
    U_NODE_DIRICHLET = 0x20u,
    U_NODE_INTERFACE = 0x40u,
    CELL_INTERIOR = 0x1u,
    NODE_DEGREE = 0x10000000u,
    NODE_TJUNCTION = 0x100u,
    NODE_COARSE_SHARED = 0x200u,
    NODE_ACTIVE = 0x400u,
};

typedef std::array<int, 3> I3;

static inline uint64_t pack3(const I3& c) {
    if (c[0] < 0 || c[1] < 0 || c[2] < 0) throw std::runtime_error("oracle: negative hierarchy index");
    return ((uint64_t)c[0] << 42) | ((uint64_t)c[1] << 21) | (uint64_t)c[2];
}
static inline I3 unpack3(uint64_t k) {
    return {(int)(k >> 42), (int)((k >> 21) & 0x1fffff), (int)(k & 0x1fffff)};
}

// SPGrid page order of a coordinate (PB/Common_Libraries/SPGrid/Core/SPGrid_Mask.h:20-120
// for a 16-byte struct: 4x8x8 pages, bit-interleaved page index, z fastest
// inside a page).  The reference walks hierarchy cells in this order, which
// fixes its DOF numbering.
static inline uint64_t pdep64(uint64_t v, uint64_t mask) {
    uint64_t r = 0;
    for (uint64_t bit = 1; mask; bit <<= 1) {
        uint64_t low = mask & (~mask + 1);
        if (v & bit) r |= low;
        mask &= mask - 1;
    }
    return r;
}
static inline uint64_t page_order_key(const I3& c) {
    const uint64_t XM = 0x9249249249249000ull | 0x300ull;
    const uint64_t YM = 0x4924924924924000ull | 0x0e0ull;
    const uint64_t ZM = 0x2492492492492000ull | 0x01cull;
    return pdep64((uint64_t)c[0], XM) | pdep64((uint64_t)c[1], YM) | pdep64((uint64_t)c[2], ZM);
}

struct Stride1D {
    int lo = 0;
    std::vector<int> q;
    int at(int i) const {
        int k = i - lo;
        if (k < 0 || k >= (int)q.size()) throw std::runtime_error("oracle: stride index out of range");
        return q[k];
    }
};
typedef std::array<Stride1D, 3> Stride3;

// CPU/Interface_Solver/STRIDE_GENERATOR.h:23-54.
// filled (optional): per axis, how many entries the fill wrote (counts + 1
// when the adaptation sequence tiles the range exactly).
static int generate_adaptive_stride(const I3& lo, const I3& hi, Stride3& q, int* filled = nullptr) {
    int level = INT_MAX;
    for (int a = 0; a < 3; ++a) {
        int counts = hi[a] - lo[a], axis_level = 0;
        std::vector<std::pair<int, int>> ad;
        ad.push_back({2, 1});
        int cur = 1, ds = 2;
        int guard = 0;
        while (ds < counts) {
            int quotient = std::min(2, (counts - ds) / cur);
            ad.push_back({quotient, cur});
            ds += quotient * cur;
            if ((counts - ds) % (2 * cur) == 0) { cur *= 2; ++axis_level; }
            if (++guard > 4096) throw std::runtime_error("oracle: stride generator does not terminate");
        }
        q[a].lo = lo[a];
        q[a].q.assign(counts + 1 + 4096, -1);
        int cnt = 1;
        std::vector<int> st;
        auto put = [&](int v) { q[a].q.at(cnt - 1) = v; ++cnt; };
        for (size_t i = 0; i < ad.size(); ++i) {
            for (int k = 0; k < ad[i].second; ++k) put(ad[i].second);
            if (ad[i].first == 1) put(ad[i].second);
            else {
                if (i + 1 == ad.size()) put(ad[i].second);
                st.push_back(ad[i].second);
            }
        }
        while (!st.empty()) {
            int cs = st.back();
            st.pop_back();
            for (int i = 0; i < cs; ++i) put(cs);
        }
        if (filled) filled[a] = cnt - 1;
        q[a].q.resize(counts + 1);
        for (int v : q[a].q)
            if (v <= 0) throw std::runtime_error("oracle: stride array not filled");
        level = std::min(level, axis_level);
    }
    return level;
}

// The strides of the box [lo, hi] per axis, axis 0 first (hi - lo + 1
// entries each), into q_out; filled[3] as above.  Returns the adaptation
// level, or -1 if an axis was not filled.
extern "C" int hddo_adaptive_stride(const int lo[3], const int hi[3], int* q_out, int filled[3]) {
    Stride3 q;
    int level;
    try {
        level = generate_adaptive_stride(I3{lo[0], lo[1], lo[2]}, I3{hi[0], hi[1], hi[2]}, q, filled);
    } catch (const std::exception&) {
        return -1;
    }
    size_t o = 0;
    for (int a = 0; a < 3; ++a)
        for (int v : q[a].q) q_out[o++] = v;
    return level;
}

template <class T>
using Parents = std::vector<std::pair<I3, T>>;

// CPU/Interface_Solver/INTERFACE_MATRIX_GENERATOR.h:81-100 (Embedding_Helper).
template <class T>
static void embed(const I3& idx, Parents<T>& parents, T w, const Stride3& q) {
    int qs = INT_MAX;
    for (int a = 0; a < 3; ++a) qs = std::min(qs, q[a].at(idx[a]));
    for (int a = 0; a < 3; ++a) {
        int cur = idx[a] - q[a].lo;
        if (cur % qs != 0) {
            I3 i1 = idx, i2 = idx;
            i1[a] = (cur / qs) * qs + q[a].lo;
            i2[a] = (cur / qs + 1) * qs + q[a].lo;
            T w1 = w * (T)(i2[a] - idx[a]) / (T)(i2[a] - i1[a]);
            T w2 = w * (T)(idx[a] - i1[a]) / (T)(i2[a] - i1[a]);
            embed(i1, parents, w1, q);
            embed(i2, parents, w2, q);
            return;
        }
    }
    for (auto& p : parents)
        if (p.first == idx) { p.second += w; return; }
    parents.push_back({idx, w});
}

template <class T>
using M8 = std::array<T, 64>;

// CPU/Interface_Solver/CELL_PROLONGATION_BAKER.h:22-50.
template <class T>
static std::array<M8<T>, 8> bake_cell_prolongation() {
    std::array<M8<T>, 8> P;
    for (int mc = 0; mc < 8; ++mc) {
        P[mc].fill(T(0));
        int o[3] = {mc >> 2, (mc >> 1) & 1, mc & 1};
        for (int fi = 0; fi < 8; ++fi) {
            int fn[3] = {(fi >> 2) + o[0], ((fi >> 1) & 1) + o[1], (fi & 1) + o[2]};
            int cn0[3];
            for (int v = 0; v < 3; ++v) cn0[v] = (int)std::floor(fn[v] / 2.0);
            for (int ci = 0; ci < 8; ++ci) {
                int cn[3] = {cn0[0] + (ci >> 2), cn0[1] + ((ci >> 1) & 1), cn0[2] + (ci & 1)};
                T weight = T(1);
                for (int v = 0; v < 3; ++v) weight *= (T(2) - std::abs(cn[v] * 2 - fn[v])) / 2.0;
                if (weight == 0) continue;
                int col = cn[0] * 4 + cn[1] * 2 + cn[2];
                P[mc][fi * 8 + col] = weight;
            }
        }
    }
    return P;
}

// Node-flag view of one subdomain box (the "sub_set" of the reference).
struct SubsetFlags {
    I3 lo, hi;
    std::vector<uint32_t> f;
    uint32_t operator()(const I3& n) const {
        for (int a = 0; a < 3; ++a)
            if (n[a] < lo[a] || n[a] > hi[a]) return 0u;
        int e1 = hi[1] - lo[1] + 1, e2 = hi[2] - lo[2] + 1;
        return f[((size_t)(n[0] - lo[0]) * e1 + (n[1] - lo[1])) * e2 + (n[2] - lo[2])];
    }
};

// CPU/Interface_Solver/GALERKIN_PROCESS.h:27-69.
template <class T>
using GalerkinMemo = std::vector<std::unordered_map<uint64_t, M8<T>>>;

template <class T>
static M8<T> galerkin_coarsen(const SubsetFlags& sf, const std::array<M8<T>, 8>& P, const I3& C,
                              int level, GalerkinMemo<T>& memo) {
    // The coarsened matrix is a pure function of (cell, level): memoised.
    auto hit = memo[level].find(pack3(C));
    if (hit != memo[level].end()) return hit->second;
    M8<T> m;
    m.fill(T(0));
    if (level == 1) {
        const T w = (T)(1.0 / (1 << 2));
        uint32_t nf[8];
        for (int li = 0; li < 8; ++li) {
            I3 node = {C[0] - 1 + (li >> 2), C[1] - 1 + ((li >> 1) & 1), C[2] - 1 + (li & 1)};
            uint32_t s = sf(node);
            nf[li] = (s & (ACTIVE | INTERFACE)) ? ACTIVE : ((s & DIRICHLET) ? DIRICHLET : 0u);
        }
        for (int v = 0; v < 3; ++v) {
            int a = (v == 0) ? 1 : 0, b = (v == 2) ? 1 : 2;
            for (int oa = 0; oa < 2; ++oa)
                for (int ob = 0; ob < 2; ++ob) {
                    int lb[3], ub[3];
                    lb[v] = 0; ub[v] = 1;
                    lb[a] = ub[a] = oa;
                    lb[b] = ub[b] = ob;
                    int l = lb[0] * 4 + lb[1] * 2 + lb[2], u = ub[0] * 4 + ub[1] * 2 + ub[2];
                    if ((nf[l] & ACTIVE) && (nf[u] & ACTIVE)) {
                        m[l * 8 + u] -= w; m[l * 8 + l] += w; m[u * 8 + u] += w; m[u * 8 + l] -= w;
                    }
                    if ((nf[l] & ACTIVE) && (nf[u] & DIRICHLET)) m[l * 8 + l] += w;
                    if ((nf[l] & DIRICHLET) && (nf[u] & ACTIVE)) m[u * 8 + u] += w;
                }
        }
    } else {
        for (int o = 0; o < 8; ++o) {
            I3 child = {2 * C[0] - 1 + (o >> 2), 2 * C[1] - 1 + ((o >> 1) & 1), 2 * C[2] - 1 + (o & 1)};
            M8<T> g = galerkin_coarsen(sf, P, child, level - 1, memo);
            const M8<T>& p = P[o];
            M8<T> t;  // t = g * p
            for (int i = 0; i < 8; ++i)
                for (int j = 0; j < 8; ++j) {
                    T acc = 0;
                    for (int k = 0; k < 8; ++k) acc += g[i * 8 + k] * p[k * 8 + j];
                    t[i * 8 + j] = acc;
                }
            for (int i = 0; i < 8; ++i)
                for (int j = 0; j < 8; ++j) {
                    T acc = 0;
                    for (int k = 0; k < 8; ++k) acc += p[k * 8 + i] * t[k * 8 + j];
                    m[i * 8 + j] += acc;
                }
        }
    }
    memo[level].emplace(pack3(C), m);
    return m;
}

struct NodeRec {
    uint32_t flags = 0;
    int index = 0;
};
typedef std::unordered_map<uint64_t, NodeRec> LevelMap;

template <class T>
struct BuildState {
    int M = 0;
    std::vector<std::unordered_map<uint64_t, int>> iface_hash;   // [level]
    std::vector<int> iface_counter;
    std::vector<std::array<int, 3>> iface_map;
    std::vector<std::unordered_map<uint64_t, T>> Arr;            // [level], key (row<<32|col)
};

static inline uint64_t rc(int r, int c) { return ((uint64_t)(uint32_t)r << 32) | (uint32_t)c; }

// One subdomain's interface contributions with subdomain-local interface
// numbers: the nodes in local first-encounter order and every Arr addition in
// traversal order, so a serial merge in subdomain order reproduces the global
// first-encounter numbering and the per-key summation order exactly.
template <class T>
struct LocalIface {
    int M = 0;
    std::vector<std::unordered_map<uint64_t, int>> hash;     // [level] node -> local id
    std::vector<std::vector<I3>> nodes;                      // [level] local id -> node
    std::vector<std::vector<std::pair<uint64_t, T>>> arr;    // [level] (rc(local, local), value)
};

static bool range_contains(const I3& lo, const I3& hi, const I3& rlo, const I3& rhi) {
    for (int a = 0; a < 3; ++a)
        if (!(lo[a] <= rlo[a] && rhi[a] <= hi[a])) return false;
    return true;
}

// CPU/Interface_Solver/INTERFACE_MATRIX_GENERATOR.h:130-659 for one subdomain.
template <class T>
static void create_subdomain_hierarchy(const SubsetFlags& sf, LocalIface<T>& li,
                                       std::vector<Csr<T>>& Aii_out,
                                       std::vector<std::unordered_map<uint64_t, T>>& Air_out,
                                       std::vector<int>& n_interior_out,
                                       std::vector<std::vector<std::array<int, 3>>>& pos_out) {
    const int M = li.M;
    li.hash.assign(M, {});
    li.nodes.assign(M, {});
    li.arr.assign(M, {});
    const I3 lo = sf.lo, hi = sf.hi;
    static const std::array<M8<T>, 8> P = bake_cell_prolongation<T>();
    Stride3 qtop;
    const int levels = generate_adaptive_stride(lo, hi, qtop);
    if (M > levels) throw std::runtime_error("oracle: sigma_levels exceeds the adaptive levels of a subdomain");
    std::vector<Stride3> q(levels + 1);
    for (int L = 1; L <= levels; ++L) {
        I3 l2, h2;
        for (int a = 0; a < 3; ++a) { l2[a] = lo[a] >> (L - 1); h2[a] = hi[a] >> (L - 1); }
        generate_adaptive_stride(l2, h2, q[L]);
    }
    // H[m][L]: per sigma level m (1..M), per hierarchy level L (1..levels).
    std::vector<std::vector<LevelMap>> H(M + 1, std::vector<LevelMap>(levels + 2));

    // Traversal: activate graded cells (lines 184-239).
    {
        std::unordered_set<uint64_t> traversed;
        auto type = [&](const I3& n) {
            uint32_t s = sf(n), t = 0;
            if (s & (ACTIVE | INTERFACE)) t |= U_NODE_ACTIVE;
            if (s & DIRICHLET) t |= U_NODE_DIRICHLET;
            return t;
        };
        for (int x = lo[0]; x <= hi[0]; ++x)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int z = lo[2]; z <= hi[2]; ++z) {
                    I3 node = {x, y, z};
                    if (sf(node) == 0) continue;
                    for (int ci = 0; ci < 8; ++ci) {
                        I3 c = {x + (ci >> 2), y + ((ci >> 1) & 1), z + (ci & 1)};
                        bool inside = true;
                        for (int a = 0; a < 3; ++a)
                            if (c[a] - 1 < lo[a] || c[a] > hi[a]) inside = false;
                        if (!inside) continue;
                        if (!traversed.insert(pack3(c)).second) continue;
                        bool contributes = false;
                        for (int v = 0; v < 3 && !contributes; ++v) {
                            int a = (v == 0) ? 1 : 0, b = (v == 2) ? 1 : 2;
                            for (int oa = 0; oa < 2 && !contributes; ++oa)
                                for (int ob = 0; ob < 2 && !contributes; ++ob) {
                                    I3 l, u;
                                    l[v] = c[v] - 1; u[v] = c[v];
                                    l[a] = u[a] = c[a] - 1 + oa;
                                    l[b] = u[b] = c[b] - 1 + ob;
                                    uint32_t lt = type(l), ut = type(u);
                                    if ((lt & ut & U_NODE_ACTIVE) ||
                                        (((lt | ut) & U_NODE_ACTIVE) && ((lt | ut) & U_NODE_DIRICHLET)))
                                        contributes = true;
                                }
                        }
                        if (!contributes) continue;
                        I3 cur = c, rlo = {c[0] - 1, c[1] - 1, c[2] - 1}, rhi = c;
                        for (int cl = 1; cl <= levels; ++cl) {
                            for (int m = 1; m <= M; ++m) {
                                int s1 = 1 << cl, s0 = 1 << (cl - 1);
                                I3 a1lo = {lo[0] + s1, lo[1] + s1, lo[2] + s1}, a1hi = {hi[0] - s1, hi[1] - s1, hi[2] - s1};
                                I3 a0lo = {lo[0] + s0, lo[1] + s0, lo[2] + s0}, a0hi = {hi[0] - s0, hi[1] - s0, hi[2] - s0};
                                bool in1 = range_contains(a1lo, a1hi, rlo, rhi);
                                bool in0 = range_contains(a0lo, a0hi, rlo, rhi);
                                if ((cl == m && !in1) || (cl > m && in0 && !in1))
                                    H[m][cl][pack3(cur)].flags |= CELL_INTERIOR;
                            }
                            for (int a = 0; a < 3; ++a) {
                                rlo[a] = (rlo[a] / (1 << cl)) * (1 << cl);
                                rhi[a] = rlo[a] + (1 << cl);
                                cur[a] = (cur[a] + 1) / 2;
                            }
                        }
                    }
                }
    }

    auto sorted_interior_cells = [&](int m, int L) {
        std::vector<std::pair<uint64_t, I3>> cells;
        for (auto& kv : H[m][L])
            if (kv.second.flags & CELL_INTERIOR) {
                I3 c = unpack3(kv.first);
                cells.push_back({page_order_key(c), c});
            }
        std::sort(cells.begin(), cells.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        std::vector<I3> out;
        out.reserve(cells.size());
        for (auto& c : cells) out.push_back(c.second);
        return out;
    };
    auto has = [&](int m, int L, const I3& n, uint32_t mask) {
        auto it = H[m][L].find(pack3(n));
        return it != H[m][L].end() && (it->second.flags & mask);
    };

    Aii_out.assign(M, Csr<T>());
    Air_out.assign(M, {});
    n_interior_out.assign(M, 0);
    std::vector<int> node_counts(M + 1, 0);

    for (int m = 1; m <= M; ++m) {
        // Interface DOFs (lines 249-312).
        auto add_iface = [&](const I3& node, bool) {
            auto& hash = li.hash[m - 1];
            uint64_t key = pack3(node);
            auto it = hash.find(key);
            int id;
            if (it == hash.end()) {
                id = (int)li.nodes[m - 1].size();
                hash.emplace(key, id);
                li.nodes[m - 1].push_back(node);
            } else id = it->second;
            NodeRec& rec = H[m][m][key];
            rec.index = id;
            rec.flags |= U_NODE_INTERFACE | NODE_DEGREE;
        };
        if (m == 1) {
            for (int axis = 0; axis < 3; ++axis)
                for (int face = 0; face <= 1; ++face) {
                    int a = (axis == 0) ? 1 : 0, b = (axis == 2) ? 1 : 2;
                    for (int va = lo[a]; va <= hi[a]; ++va)
                        for (int vb = lo[b]; vb <= hi[b]; ++vb) {
                            I3 node;
                            node[axis] = face ? hi[axis] : lo[axis];
                            node[a] = va;
                            node[b] = vb;
                            uint32_t s = sf(node);
                            if (s & INTERFACE) add_iface(node, true);
                            if (s & ACTIVE) throw std::runtime_error("oracle: active cell on a subdomain face");
                        }
                }
        } else {
            I3 clo, chi;
            for (int a = 0; a < 3; ++a) { clo[a] = lo[a] >> (m - 1); chi[a] = hi[a] >> (m - 1); }
            for (const I3& c : sorted_interior_cells(m, m))
                for (int li = 0; li < 8; ++li) {
                    I3 node = {c[0] - 1 + (li >> 2), c[1] - 1 + ((li >> 1) & 1), c[2] - 1 + (li & 1)};
                    bool is_iface = false;
                    for (int a = 0; a < 3; ++a)
                        if (node[a] == clo[a] || node[a] == chi[a]) is_iface = true;
                    if (is_iface) add_iface(node, false);
                }
        }
        // Interior DOFs (lines 315-375).
        int node_count = 0;
        std::vector<std::array<int, 3>>& pos = pos_out[m - 1];
        for (int L = m; L <= levels; ++L) {
            for (const I3& c : sorted_interior_cells(m, L))
                for (int li = 0; li < 8; ++li) {
                    I3 N = {c[0] - 1 + (li >> 2), c[1] - 1 + ((li >> 1) & 1), c[2] - 1 + (li & 1)};
                    I3 fine = {2 * N[0], 2 * N[1], 2 * N[2]};
                    if (L == 1 && !(sf(N) & ACTIVE)) continue;
                    if (L == m && has(m, L, N, U_NODE_INTERFACE)) continue;
                    int qs = INT_MAX;
                    for (int a = 0; a < 3; ++a) qs = std::min(qs, q[L][a].at(N[a]));
                    bool tj = false;
                    for (int a = 0; a < 3; ++a)
                        if ((N[a] - q[L][a].lo) % qs != 0) tj = true;
                    if (!tj) {
                        if (L > m && has(m, L - 1, fine, NODE_DEGREE)) {
                            NodeRec& rec = H[m][L][pack3(N)];
                            rec.index = H[m][L - 1][pack3(fine)].index;
                            rec.flags |= NODE_DEGREE | NODE_COARSE_SHARED;
                        }
                        NodeRec& rec = H[m][L][pack3(N)];
                        if (!(rec.flags & NODE_DEGREE)) {
                            rec.flags |= NODE_DEGREE | NODE_ACTIVE;
                            rec.index = node_count++;
                            pos.push_back({N[0] << (L - 1), N[1] << (L - 1), N[2] << (L - 1)});
                        }
                    } else {
                        H[m][L][pack3(N)].flags |= NODE_TJUNCTION;
                        Parents<T> par;
                        embed<T>(N, par, T(1), q[L]);
                        for (auto& p : par) {
                            NodeRec& rec = H[m][L][pack3(p.first)];
                            if (!(rec.flags & NODE_DEGREE)) {
                                rec.flags |= NODE_DEGREE | NODE_ACTIVE;
                                rec.index = node_count++;
                                const I3& pn = p.first;
                                pos.push_back({pn[0] << (L - 1), pn[1] << (L - 1), pn[2] << (L - 1)});
                            }
                        }
                    }
                }
        }
        node_counts[m] = node_count;
    }

    // Galerkin assembly (lines 554-655, the compiled #else branch).
    GalerkinMemo<T> memo(levels + 1);
    for (int m = 1; m <= M; ++m) {
        std::unordered_map<uint64_t, T> Aii, Air;
        auto resolve = [&](int L, const I3& p, uint32_t& f, int& id) {
            auto it = H[m][L].find(pack3(p));
            f = (it == H[m][L].end()) ? 0u : it->second.flags;
            id = (it == H[m][L].end()) ? 0 : it->second.index;
            int cur = L;
            I3 idx = p;
            while (!(f & NODE_DEGREE)) {
                ++cur;
                if (cur > levels) throw std::runtime_error("oracle: DOF lookup ran past the coarsest level");
                for (int a = 0; a < 3; ++a) idx[a] /= 2;
                auto jt = H[m][cur].find(pack3(idx));
                f = (jt == H[m][cur].end()) ? 0u : jt->second.flags;
                id = (jt == H[m][cur].end()) ? 0 : jt->second.index;
            }
        };
        for (int L = m; L <= levels; ++L)
            for (const I3& c : sorted_interior_cells(m, L)) {
                M8<T> cm = galerkin_coarsen<T>(sf, P, c, L, memo);
                Parents<T> par[8];
                for (int li = 0; li < 8; ++li) {
                    I3 N = {c[0] - 1 + (li >> 2), c[1] - 1 + ((li >> 1) & 1), c[2] - 1 + (li & 1)};
                    embed<T>(N, par[li], T(1), q[L]);
                }
                for (int n1 = 0; n1 < 8; ++n1)
                    for (int n2 = 0; n2 < 8; ++n2) {
                        T e = cm[n1 * 8 + n2];
                        if (e == 0) continue;
                        for (auto& p1 : par[n1])
                            for (auto& p2 : par[n2]) {
                                uint32_t f1, f2;
                                int id1, id2;
                                resolve(L, p1.first, f1, id1);
                                resolve(L, p2.first, f2, id2);
                                T v = p1.second * p2.second * e;
                                if ((f1 & U_NODE_INTERFACE) && (f2 & U_NODE_INTERFACE))
                                    li.arr[m - 1].push_back({rc(id1, id2), v});
                                if ((f1 & (NODE_ACTIVE | NODE_COARSE_SHARED)) &&
                                    (f2 & (NODE_ACTIVE | NODE_COARSE_SHARED)))
                                    Aii[rc(id1, id2)] += v;
                                if ((f1 & (NODE_ACTIVE | NODE_COARSE_SHARED)) && (f2 & U_NODE_INTERFACE))
                                    Air[rc(id1, id2)] += v;
                            }
                    }
            }
        int ni = node_counts[m];
        n_interior_out[m - 1] = ni;
        Aii_out[m - 1] = csr_from_map<T>(ni, ni, Aii);
        // Columns are local interface numbers until the merge.
        Air_out[m - 1] = std::move(Air);
    }
}

// Subdomain node flags, CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Subdomain_Splitter.h:123-143
// with SPGrid_Subdomain_Rasterizer.h:59-136 and the Domain_Divider pass on the box.
static SubsetFlags extract_subset(const Dims& gd, const uint32_t* gf, const I3& lo, const I3& hi,
                                  const int sub[3]) {
    SubsetFlags s;
    s.lo = lo;
    s.hi = hi;
    int e[3] = {hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1};
    std::vector<uint32_t> t((size_t)e[0] * e[1] * e[2], 0u);
    auto id = [&](int x, int y, int z) { return ((size_t)(x - lo[0]) * e[1] + (y - lo[1])) * e[2] + (z - lo[2]); };
    for (int x = lo[0]; x <= hi[0]; ++x)
        for (int y = lo[1]; y <= hi[1]; ++y)
            for (int z = lo[2]; z <= hi[2]; ++z) {
                uint32_t f0 = flag_at(gd, gf, x, y, z);
                t[id(x, y, z)] = (f0 & ACTIVE) ? ACTIVE : f0;
            }
    // Cells (of any non-zero type) without an Active face neighbour inside the
    // box are dropped.  The reference applies this in place per 4x8x8 page, so an
    // isolated Active cell can also drop a Dirichlet neighbour visited after it;
    // here every decision uses the undropped values.
    s.f.assign(t.size(), 0u);
    for (int x = lo[0]; x <= hi[0]; ++x)
        for (int y = lo[1]; y <= hi[1]; ++y)
            for (int z = lo[2]; z <= hi[2]; ++z) {
                uint32_t v = t[id(x, y, z)];
                if (!v) continue;
                bool nb_active = false;
                for (int face = 0; face < 6; ++face) {
                    int a = x + FACE_D[face][0], b = y + FACE_D[face][1], c = z + FACE_D[face][2];
                    if (a < lo[0] || b < lo[1] || c < lo[2] || a > hi[0] || b > hi[1] || c > hi[2]) continue;
                    if (t[id(a, b, c)] & ACTIVE) nb_active = true;
                }
                if (!nb_active) continue;
                if (v & ACTIVE) {
                    if (x % sub[0] == 0 || y % sub[1] == 0 || z % sub[2] == 0) v = (v - ACTIVE) | INTERFACE;
                }
                s.f[id(x, y, z)] = v;
            }
    return s;
}

template <class T>
void build_interface_system(const Dims& gd, const uint32_t* gflags_in, const int sub[3], int M,
                            InterfaceSystem<T>& out) {
    int ns[3];
    number_of_subdomains(gd.n, sub, ns);
    BuildState<T> st;
    st.M = M;
    st.iface_hash.resize(M);
    st.iface_counter.assign(M, 0);
    st.Arr.resize(M);
    out.M = M;
    out.n_sub = ns[0] * ns[1] * ns[2];
    out.Aii.assign(M, std::vector<Csr<T>>(out.n_sub));
    out.Air.assign(M, std::vector<Csr<T>>(out.n_sub));
    out.n_interior.assign(M, std::vector<int>(out.n_sub, 0));
    out.aii_xyz.assign(M, std::vector<std::vector<std::array<int, 3>>>(out.n_sub));
    // Subdomains are built concurrently in chunks, then merged serially in
    // subdomain order (the reference's traversal order).
    const int nsub = out.n_sub;
    const int chunk = 64;
    for (int s0 = 0; s0 < nsub; s0 += chunk) {
        const int s1 = std::min(nsub, s0 + chunk);
        std::vector<LocalIface<T>> li(s1 - s0);
        std::vector<std::vector<std::unordered_map<uint64_t, T>>> air(s1 - s0);
        std::vector<std::string> err(s1 - s0);
#pragma omp parallel for schedule(dynamic)
        for (int s = s0; s < s1; ++s) {
            try {
                const int i = s / (ns[1] * ns[2]), j = (s / ns[2]) % ns[1], k = s % ns[2];
                I3 lo = {i * sub[0], j * sub[1], k * sub[2]};
                I3 hi = {lo[0] + sub[0], lo[1] + sub[1], lo[2] + sub[2]};
                SubsetFlags sf = extract_subset(gd, gflags_in, lo, hi, sub);
                std::vector<Csr<T>> aii;
                std::vector<int> ni;
                std::vector<std::vector<std::array<int, 3>>> pos(M);
                li[s - s0].M = M;
                create_subdomain_hierarchy<T>(sf, li[s - s0], aii, air[s - s0], ni, pos);
                for (int m = 0; m < M; ++m) {
                    out.aii_xyz[m][s] = std::move(pos[m]);
                    out.Aii[m][s] = std::move(aii[m]);
                    out.n_interior[m][s] = ni[m];
                }
            } catch (const std::exception& e) {
                err[s - s0] = e.what();
            }
        }
        for (auto& e : err)
            if (!e.empty()) throw std::runtime_error(e);
        for (int s = s0; s < s1; ++s) {
            LocalIface<T>& L = li[s - s0];
            for (int m = 0; m < M; ++m) {
                std::vector<int> to_g(L.nodes[m].size());
                for (size_t q = 0; q < L.nodes[m].size(); ++q) {
                    const uint64_t key = pack3(L.nodes[m][q]);
                    auto it = st.iface_hash[m].find(key);
                    if (it == st.iface_hash[m].end()) {
                        it = st.iface_hash[m].emplace(key, st.iface_counter[m]++).first;
                        if (m == 0) st.iface_map.push_back(L.nodes[m][q]);
                    }
                    to_g[q] = it->second;
                }
                for (auto& t : L.arr[m])
                    st.Arr[m][rc(to_g[(int)(t.first >> 32)], to_g[(int)(uint32_t)t.first])] += t.second;
                std::unordered_map<uint64_t, T> ag;
                ag.reserve(air[s - s0][m].size());
                for (auto& kv : air[s - s0][m])
                    ag.emplace(rc((int)(kv.first >> 32), to_g[(int)(uint32_t)kv.first]), kv.second);
                out.Air[m][s] = csr_from_map<T>(out.n_interior[m][s], INT_MAX, ag);
            }
        }
    }
    out.n_iface = st.iface_counter;
    out.iface_map = st.iface_map;
    out.iface_xyz.assign(M, {});
    for (int m = 0; m < M; ++m) {
        out.iface_xyz[m].assign(out.n_iface[m], {0, 0, 0});
        for (auto& kv : st.iface_hash[m]) {
            const I3 nd = unpack3(kv.first);
            out.iface_xyz[m][kv.second] = {nd[0] << m, nd[1] << m, nd[2] << m};
        }
    }
    out.Arr.resize(M);
    for (int m = 0; m < M; ++m) {
        out.Arr[m] = csr_from_map<T>(out.n_iface[m], out.n_iface[m], st.Arr[m]);
        for (int r = 0; r < out.Arr[m].rows; ++r) {
            bool diag = false;
            for (int p = out.Arr[m].ptr[r]; p < out.Arr[m].ptr[r + 1]; ++p)
                if (out.Arr[m].col[p] == r && out.Arr[m].val[p] != T(0)) diag = true;
            if (m == 0 && !diag) throw std::runtime_error("oracle: zero diagonal in Arr (INTERFACE_MATRIX_GENERATOR.h:679-680)");
        }
        for (int sd = 0; sd < out.n_sub; ++sd) out.Air[m][sd].cols = out.n_iface[m];
    }
    // Prr (CPU/Interface_Solver/PROLONGATION_MATRIX_HELPER.cpp:13-40).
    out.Prr.resize(M > 1 ? M - 1 : 0);
    for (int m = 0; m + 1 < M; ++m) {
        std::unordered_map<uint64_t, T> P;
        for (auto& kv : st.iface_hash[m]) {
            I3 F = unpack3(kv.first);
            int cn0[3];
            for (int v = 0; v < 3; ++v) cn0[v] = (int)std::floor(F[v] / 2.0);
            for (int ci = 0; ci < 8; ++ci) {
                I3 C = {cn0[0] + (ci >> 2), cn0[1] + ((ci >> 1) & 1), cn0[2] + (ci & 1)};
                T weight = T(1);
                for (int v = 0; v < 3; ++v) weight *= (T(2) - std::abs(C[v] * 2 - F[v])) / 2.0;
                if (weight > 0) {
                    auto it = st.iface_hash[m + 1].find(pack3(C));
                    if (it == st.iface_hash[m + 1].end()) continue;
                    P[rc(kv.second, it->second)] += weight;
                }
            }
        }
        out.Prr[m] = csr_from_map<T>(out.n_iface[m], out.n_iface[m + 1], P);
    }
}

// --------------------------------------------------------------------------
// Sigma V-cycle (CPU/Interface_Solver/SIGMA_SMOOTHER.cpp, SIGMA_MULTIGRID_SOLVER.cpp)
// --------------------------------------------------------------------------
template <class T>
void SigmaSolver<T>::initialize(const InterfaceSystem<T>& s, int smoothing_iterations) {
    sys = &s;
    smoothing = smoothing_iterations;
    const double eps = 1e-5;  // Eigen_To_Pardiso default epsilon, SIGMA_SMOOTHER.cpp:176
    arr.resize(s.M);
    aii.assign(s.M, std::vector<Cholesky>(s.n_sub));
    const bool verbose = std::getenv("HDDO_VERBOSE") != nullptr;
    auto t0 = std::chrono::steady_clock::now();
    auto stamp = [&](const char* what, int l) {
        if (!verbose) return;
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(stderr, "[oracle setup]   level %d %s at %.2f s\n", l, what, sec);
    };
    for (int l = 0; l < s.M; ++l) {
        arr[l].factor(s.Arr[l], eps, &s.iface_xyz[l]);
        stamp("interface factor", l);
#pragma omp parallel for schedule(dynamic)
        for (int sd = 0; sd < s.n_sub; ++sd)
            if (s.n_interior[l][sd] > 0) aii[l][sd].factor(s.Aii[l][sd], eps, &s.aii_xyz[l][sd]);
        stamp("subdomain factors", l);
    }
    u.resize(s.M);
    r.resize(s.M);
    b.resize(s.M);
    for (int l = 0; l < s.M; ++l) {
        u[l].assign(s.n_iface[l], T(0));
        r[l].assign(s.n_iface[l], T(0));
        b[l].assign(s.n_iface[l], T(0));
    }
}

template <class T>
static void schur_accumulate(const InterfaceSystem<T>& s, const std::vector<std::vector<Cholesky>>& aii,
                             int l, const std::vector<T>& u, std::vector<T>& acc) {
    // The subdomain solves are independent; their contributions are added
    // in subdomain order afterwards.
    std::vector<std::vector<T>> vxt(s.n_sub);
#pragma omp parallel for schedule(dynamic)
    for (int sd = 0; sd < s.n_sub; ++sd) {
        int ni = s.n_interior[l][sd];
        if (ni == 0) continue;
        std::vector<T> vb(ni, T(0));
        s.Air[l][sd].spmv(u.data(), vb.data());
        std::vector<double> vx(vb.begin(), vb.end());
        aii[l][sd].solve(vx.data());
        vxt[sd].assign(vx.begin(), vx.end());
    }
    for (int sd = 0; sd < s.n_sub; ++sd)
        if (s.n_interior[l][sd] > 0) s.Air[l][sd].spmv_t_add(vxt[sd].data(), acc.data());
}

template <class T>
void SigmaSolver<T>::smooth(int l, std::vector<T>& uu, std::vector<T>& tmp, const std::vector<T>& bb) const {
    tmp = bb;
    schur_accumulate(*sys, aii, l, uu, tmp);
    std::vector<double> x(tmp.begin(), tmp.end());
    arr[l].solve(x.data());
    for (size_t i = 0; i < x.size(); ++i) uu[i] = (T)x[i];
}

template <class T>
void SigmaSolver<T>::compute_residual(int l, const std::vector<T>& uu, std::vector<T>& rr,
                                      const std::vector<T>& bb) const {
    rr = bb;
    schur_accumulate(*sys, aii, l, uu, rr);
    std::vector<T> au(uu.size());
    sys->Arr[l].spmv(uu.data(), au.data());
    for (size_t i = 0; i < rr.size(); ++i) rr[i] -= au[i];
}

template <class T>
void SigmaSolver<T>::v_cycle() {
    const int M = sys->M;
    for (int l = 0; l < M - 1; ++l) {
        for (int i = 0; i < smoothing; ++i) smooth(l, u[l], r[l], b[l]);
        compute_residual(l, u[l], r[l], b[l]);
        std::fill(u[l + 1].begin(), u[l + 1].end(), T(0));
        std::fill(b[l + 1].begin(), b[l + 1].end(), T(0));
        sys->Prr[l].spmv_t_add(r[l].data(), b[l + 1].data());
    }
    for (int i = 0; i < 200; ++i) smooth(M - 1, u[M - 1], r[M - 1], b[M - 1]);
    for (int l = M - 2; l >= 0; --l) {
        std::vector<T> pu(u[l].size());
        sys->Prr[l].spmv(u[l + 1].data(), pu.data());
        for (size_t i = 0; i < pu.size(); ++i) u[l][i] += pu[i];
        for (int i = 0; i < smoothing; ++i) smooth(l, u[l], r[l], b[l]);
    }
}

template struct Csr<float>;
template struct Csr<double>;
template void Cholesky::factor<float>(const Csr<float>&, double, const std::vector<std::array<int, 3>>*);
template void Cholesky::factor<double>(const Csr<double>&, double, const std::vector<std::array<int, 3>>*);
template void build_interface_system<float>(const Dims&, const uint32_t*, const int*, int, InterfaceSystem<float>&);
template void build_interface_system<double>(const Dims&, const uint32_t*, const int*, int, InterfaceSystem<double>&);
template struct SigmaSolver<float>;
template struct SigmaSolver<double>;

}  // namespace oracle
