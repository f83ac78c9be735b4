// Interface system assembly (host, parallel over subdomains).
//
// Restates CPU/Interface_Solver/INTERFACE_MATRIX_GENERATOR.h:130-735 with its
// helpers STRIDE_GENERATOR.h:23-54, CELL_PROLONGATION_BAKER.h:22-50,
// GALERKIN_PROCESS.h:27-69 and PROLONGATION_MATRIX_HELPER.cpp:13-40, and
// the subdomain flag extraction of SPGrid_Subdomain_Splitter.h:123-154 /
// SPGrid_Subdomain_Rasterizer.h:59-136.
//
// Data structures differ from the reference: every subdomain works on dense
// box-local arrays per hierarchy level instead of SPGrid allocators and hash
// tables, Galerkin-coarsened element matrices are computed once per cell type,
// and subdomains are processed concurrently.  Global interface DOF numbers are
// then assigned in the reference's first-encounter order over (subdomain, local
// index), and interface-interface contributions are summed per key in the
// reference's (subdomain, cell) order, so the assembled matrices follow the
// reference's numbering and float summation order.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <deque>
#include <functional>
#include <parallel/algorithm>
#include <string>
#include <unordered_map>

#include "host_setup.h"
#include "sigma.h"

namespace hdd {
namespace {

// Adaptive-hierarchy flags, CPU/Interface_Solver/ADAPTIVE_SUBDOMAIN_POISSON_FLAGS.h:11-26.
enum : uint32_t {
    N_INTERFACE = 0x40u,
    CELL_INTERIOR = 0x1u,
    N_DEGREE = 0x10000000u,
    N_TJUNCTION = 0x100u,
    N_COARSE_SHARED = 0x200u,
    N_ACTIVE = 0x400u,
};

typedef std::array<int, 3> I3;
typedef std::array<float, 64> M8;

// SPGrid page order: the order in which the reference walks hierarchy cells.
inline uint64_t page_key(const I3& c) { return spgrid_address(c[0], c[1], c[2]); }

struct Stride {
    int lo[3];
    std::vector<int> q[3];
    int at(int axis, int i) const { return q[axis][i - lo[axis]]; }
};

// STRIDE_GENERATOR::Generate_Adaptive_Stride: graded node spacing per axis
// (1 next to the box faces, doubling toward the centre); returns the number
// of adaptation levels.
int adaptive_stride(const I3& lo, const I3& hi, Stride& st) {
    int level = INT_MAX;
    for (int a = 0; a < 3; ++a) {
        const int count = hi[a] - lo[a];
        int axis_level = 0;
        std::vector<std::pair<int, int>> steps{{2, 1}};
        int cur = 1, covered = 2;
        while (covered < count) {
            const int qn = std::min(2, (count - covered) / cur);
            if (qn <= 0) throw Error(HDD_ERR_UNSUPPORTED, "adaptive stride: subdomain size must be a power of two");
            steps.push_back({qn, cur});
            covered += qn * cur;
            if ((count - covered) % (2 * cur) == 0) { cur *= 2; ++axis_level; }
        }
        st.lo[a] = lo[a];
        std::vector<int>& q = st.q[a];
        q.clear();
        std::vector<int> pending;
        for (size_t i = 0; i < steps.size(); ++i) {
            q.insert(q.end(), steps[i].second, steps[i].second);
            if (steps[i].first == 1 || i + 1 == steps.size()) q.push_back(steps[i].second);
            if (steps[i].first != 1) pending.push_back(steps[i].second);
        }
        while (!pending.empty()) {
            q.insert(q.end(), pending.back(), pending.back());
            pending.pop_back();
        }
        if ((int)q.size() != count + 1) throw Error(HDD_ERR_INTERNAL, "adaptive stride length mismatch");
        level = std::min(level, axis_level);
    }
    return level;
}

typedef std::vector<std::pair<I3, float>> Parents;

// Embedding_Helper: hanging nodes are linear interpolants of the aligned nodes
// on either side, recursively.
void embed(const I3& idx, Parents& out, float w, const Stride& q) {
    int qs = INT_MAX;
    for (int a = 0; a < 3; ++a) qs = std::min(qs, q.at(a, idx[a]));
    for (int a = 0; a < 3; ++a) {
        const int cur = idx[a] - q.lo[a];
        if (cur % qs != 0) {
            I3 i1 = idx, i2 = idx;
            i1[a] = (cur / qs) * qs + q.lo[a];
            i2[a] = (cur / qs + 1) * qs + q.lo[a];
            const float w1 = w * (float)(i2[a] - idx[a]) / (float)(i2[a] - i1[a]);
            const float w2 = w * (float)(idx[a] - i1[a]) / (float)(i2[a] - i1[a]);
            embed(i1, out, w1, q);
            embed(i2, out, w2, q);
            return;
        }
    }
    for (auto& p : out)
        if (p.first == idx) { p.second += w; return; }
    out.push_back({idx, w});
}

// Trilinear node prolongation of one cell to its 8 children, indexed by the
// child offset o = 4*ox+2*oy+oz; rows are the child's local nodes, columns the
// parent's local nodes (both 4*x+2*y+z).
std::array<M8, 8> bake_prolongation() {
    std::array<M8, 8> P;
    for (int o = 0; o < 8; ++o) {
        P[o].fill(0.0f);
        const int off[3] = {o >> 2, (o >> 1) & 1, o & 1};
        for (int fi = 0; fi < 8; ++fi) {
            const int fn[3] = {(fi >> 2) + off[0], ((fi >> 1) & 1) + off[1], (fi & 1) + off[2]};
            int base[3];
            for (int v = 0; v < 3; ++v) base[v] = (int)std::floor(fn[v] / 2.0);
            for (int ci = 0; ci < 8; ++ci) {
                const int cn[3] = {base[0] + (ci >> 2), base[1] + ((ci >> 1) & 1), base[2] + (ci & 1)};
                float w = 1.0f;
                for (int v = 0; v < 3; ++v) w *= (2.0f - std::abs(cn[v] * 2 - fn[v])) / 2.0;
                if (w == 0) continue;
                P[o][fi * 8 + cn[0] * 4 + cn[1] * 2 + cn[2]] = w;
            }
        }
    }
    return P;
}

struct BoxWork {
    I3 lo, hi;
    int levels = 0;
    std::vector<uint32_t> sub_flags;       // (sub+1)^3 node flags of the box
    int e1[3];
    uint32_t sf(const I3& n) const {
        for (int a = 0; a < 3; ++a)
            if (n[a] < lo[a] || n[a] > hi[a]) return 0u;
        return sub_flags[((size_t)(n[0] - lo[0]) * e1[1] + (n[1] - lo[1])) * e1[2] + (n[2] - lo[2])];
    }
    // Results per sigma level m (0-based).
    std::vector<std::vector<I3>> iface_nodes;   // first-encounter list of interface nodes (level coords)
    std::vector<std::vector<std::pair<std::pair<int, int>, float>>> arr_terms;  // (local iface ids), value
    std::vector<CsrF> aii;
    std::vector<std::vector<std::pair<std::pair<int, int>, float>>> air_terms;  // (row, local iface id)
    std::vector<int> n_int;
    std::vector<std::vector<I3>> int_xyz;       // interior DOF -> position in finest-level units
};

struct LevelArrays {
    int lo[3], e[3];
    std::vector<uint32_t> flags;
    std::vector<int> index;
    bool inside(const I3& n) const {
        for (int a = 0; a < 3; ++a)
            if (n[a] < lo[a] || n[a] >= lo[a] + e[a]) return false;
        return true;
    }
    size_t at(const I3& n) const {
        if (!inside(n)) throw Error(HDD_ERR_INTERNAL, "hierarchy index outside its subdomain box");
        return ((size_t)(n[0] - lo[0]) * e[1] + (n[1] - lo[1])) * e[2] + (n[2] - lo[2]);
    }
};

// m += P^T (G P) for one child (CELL_PROLONGATION_BAKER / GALERKIN_PROCESS):
// t = G P, then m_ij += sum_k P_ki t_kj.  Every sum starts at 0 and adds its
// eight products in k order; the loops run over j innermost so they vectorise
// without changing that order (no FMA contraction: -ffp-contract=off).
__attribute__((target_clones("avx2", "default")))
void galerkin_add(const M8& g, const M8& p, M8& m) {
    M8 t;
    for (int i = 0; i < 8; ++i) {
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 8; ++k) {
            const float gik = g[i * 8 + k];
            for (int j = 0; j < 8; ++j) acc[j] += gik * p[k * 8 + j];
        }
        for (int j = 0; j < 8; ++j) t[i * 8 + j] = acc[j];
    }
    for (int i = 0; i < 8; ++i) {
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 8; ++k) {
            const float pki = p[k * 8 + i];
            for (int j = 0; j < 8; ++j) acc[j] += pki * t[k * 8 + j];
        }
        for (int j = 0; j < 8; ++j) m[i * 8 + j] += acc[j];
    }
}

void process_box(BoxWork& W, int M, const std::array<M8, 8>& P) {
    const I3 lo = W.lo, hi = W.hi;
    Stride qtop;
    const int levels = adaptive_stride(lo, hi, qtop);
    if (M > levels) throw Error(HDD_ERR_INVALID_ARGUMENT, "sigma_levels exceeds the adaptive levels of a subdomain");
    W.levels = levels;
    // A box without Active or Interface cells has no interface and no interior
    // DOFs at any level (no cell is activated below), so its matrices are
    // empty; sparse domains have many such boxes.
    bool solvable = false;
    for (uint32_t f : W.sub_flags)
        if (f & (F_ACTIVE | F_INTERFACE)) { solvable = true; break; }
    if (!solvable) {
        W.iface_nodes.assign(M, {});
        W.arr_terms.assign(M, {});
        W.air_terms.assign(M, {});
        W.aii.assign(M, CsrF());
        for (CsrF& A : W.aii) A.ptr.assign(1, 0);
        W.n_int.assign(M, 0);
        W.int_xyz.assign(M, {});
        return;
    }
    std::vector<Stride> q(levels + 1);
    for (int L = 1; L <= levels; ++L) {
        I3 l2, h2;
        for (int a = 0; a < 3; ++a) { l2[a] = lo[a] >> (L - 1); h2[a] = hi[a] >> (L - 1); }
        adaptive_stride(l2, h2, q[L]);
    }
    // H[m][L] for m = 1..M, L = 1..levels.
    std::vector<std::vector<LevelArrays>> H(M + 1, std::vector<LevelArrays>(levels + 1));
    for (int m = 1; m <= M; ++m)
        for (int L = 1; L <= levels; ++L) {
            LevelArrays& A = H[m][L];
            size_t cnt = 1;
            for (int a = 0; a < 3; ++a) {
                A.lo[a] = lo[a] >> (L - 1);
                A.e[a] = (hi[a] >> (L - 1)) - A.lo[a] + 1;
                cnt *= (size_t)A.e[a];
            }
            A.flags.assign(cnt, 0u);
            A.index.assign(cnt, 0);
        }

    // Graded cell activation (INTERFACE_MATRIX_GENERATOR.h:184-239).
    {
        const int ec[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
        std::vector<uint8_t> traversed((size_t)ec[0] * ec[1] * ec[2], 0);
        auto ntype = [&](const I3& n) {
            const uint32_t s = W.sf(n);
            return (uint32_t)(((s & (F_ACTIVE | F_INTERFACE)) ? 1u : 0u) | ((s & F_DIRICHLET) ? 2u : 0u));
        };
        for (int x = lo[0]; x <= hi[0]; ++x)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int z = lo[2]; z <= hi[2]; ++z) {
                    if (W.sf({x, y, z}) == 0) continue;
                    for (int ci = 0; ci < 8; ++ci) {
                        const I3 c = {x + (ci >> 2), y + ((ci >> 1) & 1), z + (ci & 1)};
                        if (c[0] > hi[0] || c[1] > hi[1] || c[2] > hi[2]) continue;
                        if (c[0] - 1 < lo[0] || c[1] - 1 < lo[1] || c[2] - 1 < lo[2]) continue;
                        uint8_t& tv = traversed[((size_t)(c[0] - lo[0] - 1) * ec[1] + (c[1] - lo[1] - 1)) * ec[2] +
                                                (c[2] - lo[2] - 1)];
                        if (tv) continue;
                        tv = 1;
                        bool contributes = false;
                        for (int v = 0; v < 3 && !contributes; ++v) {
                            const int a = (v == 0) ? 1 : 0, b = (v == 2) ? 1 : 2;
                            for (int e = 0; e < 4 && !contributes; ++e) {
                                I3 l, u;
                                l[v] = c[v] - 1; u[v] = c[v];
                                l[a] = u[a] = c[a] - 1 + (e >> 1);
                                l[b] = u[b] = c[b] - 1 + (e & 1);
                                const uint32_t lt = ntype(l), ut = ntype(u);
                                if ((lt & ut & 1u) || (((lt | ut) & 1u) && ((lt | ut) & 2u))) contributes = true;
                            }
                        }
                        if (!contributes) continue;
                        I3 cur = c, rlo = {c[0] - 1, c[1] - 1, c[2] - 1}, rhi = c;
                        for (int cl = 1; cl <= levels; ++cl) {
                            const int s1 = 1 << cl, s0 = 1 << (cl - 1);
                            bool in1 = true, in0 = true;
                            for (int a = 0; a < 3; ++a) {
                                if (!(lo[a] + s1 <= rlo[a] && rhi[a] <= hi[a] - s1)) in1 = false;
                                if (!(lo[a] + s0 <= rlo[a] && rhi[a] <= hi[a] - s0)) in0 = false;
                            }
                            for (int m = 1; m <= M; ++m)
                                if ((cl == m && !in1) || (cl > m && in0 && !in1))
                                    H[m][cl].flags[H[m][cl].at(cur)] |= CELL_INTERIOR;
                            for (int a = 0; a < 3; ++a) {
                                rlo[a] = (rlo[a] / s1) * s1;
                                rhi[a] = rlo[a] + s1;
                                cur[a] = (cur[a] + 1) / 2;
                            }
                        }
                    }
                }
    }

    // Interior cells of (m, L) in SPGrid page order.  Their CELL_INTERIOR marks
    // are final after the activation above (the DOF numbering only adds node
    // bits), so each list is built once and reused.
    std::vector<std::vector<std::vector<I3>>> cell_lists(M + 1, std::vector<std::vector<I3>>(levels + 1));
    std::vector<std::vector<char>> cell_listed(M + 1, std::vector<char>(levels + 1, 0));
    auto interior_cells = [&](int m, int L) -> const std::vector<I3>& {
        if (cell_listed[m][L]) return cell_lists[m][L];
        const LevelArrays& A = H[m][L];
        std::vector<std::pair<uint64_t, I3>> cells;
        for (int x = 0; x < A.e[0]; ++x)
            for (int y = 0; y < A.e[1]; ++y)
                for (int z = 0; z < A.e[2]; ++z)
                    if (A.flags[((size_t)x * A.e[1] + y) * A.e[2] + z] & CELL_INTERIOR) {
                        const I3 c = {A.lo[0] + x, A.lo[1] + y, A.lo[2] + z};
                        cells.push_back({page_key(c), c});
                    }
        std::sort(cells.begin(), cells.end(), [](const auto& p, const auto& r) { return p.first < r.first; });
        std::vector<I3>& out = cell_lists[m][L];
        out.resize(cells.size());
        for (size_t i = 0; i < cells.size(); ++i) out[i] = cells[i].second;
        cell_listed[m][L] = 1;
        return out;
    };

    W.iface_nodes.assign(M, {});
    W.arr_terms.assign(M, {});
    W.air_terms.assign(M, {});
    W.aii.assign(M, CsrF());
    W.n_int.assign(M, 0);
    W.int_xyz.assign(M, {});
    std::vector<int> node_count(M + 1, 0);
    Parents tj_par;  // parents of a T-junction node (reused)

    for (int m = 1; m <= M; ++m) {
        // Interface DOFs (lines 249-312), numbered locally in encounter order.
        std::unordered_map<uint64_t, int> local_id;
        auto add_iface = [&](const I3& node) {
            const uint64_t key = ((uint64_t)node[0] << 42) | ((uint64_t)node[1] << 21) | (uint64_t)node[2];
            auto it = local_id.find(key);
            int id;
            if (it == local_id.end()) {
                id = (int)W.iface_nodes[m - 1].size();
                local_id.emplace(key, id);
                W.iface_nodes[m - 1].push_back(node);
            } else id = it->second;
            LevelArrays& A = H[m][m];
            const size_t p = A.at(node);
            A.index[p] = id;
            A.flags[p] |= N_INTERFACE | N_DEGREE;
        };
        if (m == 1) {
            for (int axis = 0; axis < 3; ++axis)
                for (int face = 0; face <= 1; ++face) {
                    const int a = (axis == 0) ? 1 : 0, b = (axis == 2) ? 1 : 2;
                    for (int va = lo[a]; va <= hi[a]; ++va)
                        for (int vb = lo[b]; vb <= hi[b]; ++vb) {
                            I3 node;
                            node[axis] = face ? hi[axis] : lo[axis];
                            node[a] = va;
                            node[b] = vb;
                            if (W.sf(node) & F_INTERFACE) add_iface(node);
                        }
                }
        } else {
            I3 clo, chi;
            for (int a = 0; a < 3; ++a) { clo[a] = lo[a] >> (m - 1); chi[a] = hi[a] >> (m - 1); }
            for (const I3& c : interior_cells(m, m))
                for (int li = 0; li < 8; ++li) {
                    const I3 node = {c[0] - 1 + (li >> 2), c[1] - 1 + ((li >> 1) & 1), c[2] - 1 + (li & 1)};
                    bool on_face = false;
                    for (int a = 0; a < 3; ++a)
                        if (node[a] == clo[a] || node[a] == chi[a]) on_face = true;
                    if (on_face) add_iface(node);
                }
        }
        // Interior DOFs (lines 315-375).
        int count = 0;
        for (int L = m; L <= levels; ++L) {
            LevelArrays& A = H[m][L];
            for (const I3& c : interior_cells(m, L))
                for (int li = 0; li < 8; ++li) {
                    const I3 N = {c[0] - 1 + (li >> 2), c[1] - 1 + ((li >> 1) & 1), c[2] - 1 + (li & 1)};
                    if (L == 1 && !(W.sf(N) & F_ACTIVE)) continue;
                    const size_t pn = A.at(N);
                    if (L == m && (A.flags[pn] & N_INTERFACE)) continue;
                    int qs = INT_MAX;
                    for (int a = 0; a < 3; ++a) qs = std::min(qs, q[L].at(a, N[a]));
                    bool tj = false;
                    for (int a = 0; a < 3; ++a)
                        if ((N[a] - q[L].lo[a]) % qs != 0) tj = true;
                    if (!tj) {
                        if (L > m) {
                            const LevelArrays& F = H[m][L - 1];
                            const I3 fine = {2 * N[0], 2 * N[1], 2 * N[2]};
                            const size_t pf = F.at(fine);
                            if (F.flags[pf] & N_DEGREE) {
                                A.index[pn] = F.index[pf];
                                A.flags[pn] |= N_DEGREE | N_COARSE_SHARED;
                            }
                        }
                        if (!(A.flags[pn] & N_DEGREE)) {
                            A.flags[pn] |= N_DEGREE | N_ACTIVE;
                            A.index[pn] = count++;
                            W.int_xyz[m - 1].push_back({N[0] << (L - 1), N[1] << (L - 1), N[2] << (L - 1)});
                        }
                    } else {
                        A.flags[pn] |= N_TJUNCTION;
                        tj_par.clear();
                        embed(N, tj_par, 1.0f, q[L]);
                        const Parents& par = tj_par;
                        for (auto& p : par) {
                            const size_t pp = A.at(p.first);
                            if (!(A.flags[pp] & N_DEGREE)) {
                                A.flags[pp] |= N_DEGREE | N_ACTIVE;
                                A.index[pp] = count++;
                                const I3& q2 = p.first;
                                W.int_xyz[m - 1].push_back({q2[0] << (L - 1), q2[1] << (L - 1), q2[2] << (L - 1)});
                            }
                        }
                    }
                }
        }
        node_count[m] = count;
    }

    // Galerkin-coarsened cell matrices.  A cell's matrix depends only on its
    // type: at level 1 the kinds of its 8 nodes (Active/Interface, Dirichlet or
    // neither), at coarser levels the types of its 8 children.  Each distinct
    // type is computed once per subdomain, by the same operations in the same
    // order as for any cell of that type; cells keep a type id, in a dense
    // box-local table per level (reused by the thread from box to box) with a
    // hash table for any cell outside it.
    struct MemoRange { int lo[3], e[3]; size_t base; };
    std::vector<MemoRange> mr(levels + 1);
    size_t memo_cells = 0;
    for (int L = 1; L <= levels; ++L) {
        size_t cnt = 1;
        for (int a = 0; a < 3; ++a) {
            mr[L].lo[a] = (lo[a] >> (L - 1)) - 1;
            mr[L].e[a] = (hi[a] >> (L - 1)) + 2 - mr[L].lo[a];
            cnt *= (size_t)mr[L].e[a];
        }
        mr[L].base = memo_cells;
        memo_cells += cnt;
    }
    static thread_local std::vector<int> memo_type;
    memo_type.assign(memo_cells, -1);
    std::vector<std::unordered_map<uint64_t, int>> memo(levels + 1);
    std::deque<M8> mats;                              // matrix of each type id
    std::vector<int> node_types(6561, -1);            // level 1: 3^8 node-kind codes
    struct ChildHash {
        size_t operator()(const std::array<int, 8>& k) const {
            uint64_t h = 1469598103934665603ull;
            for (int v : k) h = (h ^ (uint32_t)v) * 1099511628211ull;
            return (size_t)h;
        }
    };
    std::vector<std::unordered_map<std::array<int, 8>, int, ChildHash>> child_types(levels + 1);
    std::function<int(const I3&, int)> cell_type = [&](const I3& C, int level) -> int {
        const MemoRange& R = mr[level];
        bool dense = true;
        for (int a = 0; a < 3; ++a)
            if (C[a] < R.lo[a] || C[a] >= R.lo[a] + R.e[a]) dense = false;
        const size_t slot =
            dense ? R.base + ((size_t)(C[0] - R.lo[0]) * R.e[1] + (C[1] - R.lo[1])) * R.e[2] + (C[2] - R.lo[2]) : 0;
        const uint64_t key = ((uint64_t)C[0] << 42) | ((uint64_t)C[1] << 21) | (uint64_t)C[2];
        if (dense) {
            if (memo_type[slot] >= 0) return memo_type[slot];
        } else {
            auto it = memo[level].find(key);
            if (it != memo[level].end()) return it->second;
        }
        int id;
        if (level == 1) {
            uint32_t nf[8];
            int code = 0;
            for (int li = 7; li >= 0; --li) {
                const I3 node = {C[0] - 1 + (li >> 2), C[1] - 1 + ((li >> 1) & 1), C[2] - 1 + (li & 1)};
                const uint32_t s = W.sf(node);
                nf[li] = (s & (F_ACTIVE | F_INTERFACE)) ? 1u : ((s & F_DIRICHLET) ? 2u : 0u);
                code = code * 3 + (int)nf[li];
            }
            id = node_types[code];
            if (id < 0) {
                M8 m;
                m.fill(0.0f);
                const float w = (float)(1.0 / (1 << 2));
                for (int v = 0; v < 3; ++v) {
                    const int a = (v == 0) ? 1 : 0, b = (v == 2) ? 1 : 2;
                    for (int e = 0; e < 4; ++e) {
                        int lb[3], ub[3];
                        lb[v] = 0; ub[v] = 1;
                        lb[a] = ub[a] = e >> 1;
                        lb[b] = ub[b] = e & 1;
                        const int l = lb[0] * 4 + lb[1] * 2 + lb[2], u = ub[0] * 4 + ub[1] * 2 + ub[2];
                        if (nf[l] == 1u && nf[u] == 1u) {
                            m[l * 8 + u] -= w; m[l * 8 + l] += w; m[u * 8 + u] += w; m[u * 8 + l] -= w;
                        }
                        if (nf[l] == 1u && nf[u] == 2u) m[l * 8 + l] += w;
                        if (nf[l] == 2u && nf[u] == 1u) m[u * 8 + u] += w;
                    }
                }
                id = (int)mats.size();
                mats.push_back(m);
                node_types[code] = id;
            }
        } else {
            std::array<int, 8> ch;
            for (int o = 0; o < 8; ++o) {
                const I3 child = {2 * C[0] - 1 + (o >> 2), 2 * C[1] - 1 + ((o >> 1) & 1), 2 * C[2] - 1 + (o & 1)};
                ch[o] = cell_type(child, level - 1);
            }
            auto it = child_types[level].find(ch);
            if (it != child_types[level].end()) {
                id = it->second;
            } else {
                M8 m;
                m.fill(0.0f);
                for (int o = 0; o < 8; ++o) galerkin_add(mats[ch[o]], P[o], m);
                id = (int)mats.size();
                mats.push_back(m);
                child_types[level].emplace(ch, id);
            }
        }
        if (dense) memo_type[slot] = id;
        else memo[level].emplace(key, id);
        return id;
    };
    auto galerkin = [&](const I3& C, int level) -> const M8& { return mats[cell_type(C, level)]; };

    // Assembly (lines 554-655).  Each cell's node parents are resolved once;
    // the entries are then summed in the reference's (cell, n1, n2, parent1,
    // parent2) order, so every Aii / Air sum adds its terms in that order.
    for (int m = 1; m <= M; ++m) {
        // Per interior row: its Aii entries (column, sum) and its Air entries
        // (interface column, index into air_terms), in first-encounter order.
        const int nrow = node_count[m];
        std::vector<std::vector<std::pair<int, float>>> aii_rows(nrow);
        std::vector<std::vector<std::pair<int, size_t>>> air_rows(nrow);
        // Walks up the hierarchy to the level that owns node p; false when no
        // level does (an error only if an entry with this parent is used).
        auto resolve = [&](int L, const I3& p, uint32_t& f, int& id) {
            I3 idx = p;
            int cur = L;
            {
                const LevelArrays& A = H[m][cur];
                const size_t pp = A.at(idx);
                f = A.flags[pp];
                id = A.index[pp];
            }
            while (!(f & N_DEGREE)) {
                if (++cur > levels) return false;
                for (int a = 0; a < 3; ++a) idx[a] /= 2;
                const LevelArrays& A = H[m][cur];
                const size_t pp = A.at(idx);
                f = A.flags[pp];
                id = A.index[pp];
            }
            return true;
        };
        struct Resolved { uint32_t f; int id; float w; bool ok; };
        // Resolved parents of each node of level L, computed once per node
        // (a node is shared by up to 8 cells): node_first[node] indexes pool.
        std::vector<Resolved> pool;
        std::vector<int> node_first, node_n;
        int rb[8], rn[8];
        Parents par;
        for (int L = m; L <= levels; ++L) {
            const LevelArrays& AL = H[m][L];
            node_first.assign(AL.flags.size(), -1);
            node_n.assign(AL.flags.size(), 0);
            pool.clear();
            for (const I3& c : interior_cells(m, L)) {
                const M8& cm = galerkin(c, L);
                for (int li = 0; li < 8; ++li) {
                    const I3 N = {c[0] - 1 + (li >> 2), c[1] - 1 + ((li >> 1) & 1), c[2] - 1 + (li & 1)};
                    const size_t nidx = AL.at(N);
                    if (node_first[nidx] < 0) {
                        par.clear();
                        embed(N, par, 1.0f, q[L]);
                        node_first[nidx] = (int)pool.size();
                        node_n[nidx] = (int)par.size();
                        for (auto& p : par) {
                            Resolved r;
                            r.ok = resolve(L, p.first, r.f, r.id);
                            r.w = p.second;
                            pool.push_back(r);
                        }
                    }
                    rb[li] = node_first[nidx];
                    rn[li] = node_n[nidx];
                }
                for (int n1 = 0; n1 < 8; ++n1)
                    for (int n2 = 0; n2 < 8; ++n2) {
                        const float e = cm[n1 * 8 + n2];
                        if (e == 0) continue;
                        for (int i1 = 0; i1 < rn[n1]; ++i1)
                            for (int i2 = 0; i2 < rn[n2]; ++i2) {
                                const Resolved& p1 = pool[(size_t)rb[n1] + i1];
                                const Resolved& p2 = pool[(size_t)rb[n2] + i2];
                                if (!p1.ok || !p2.ok)
                                    throw Error(HDD_ERR_INTERNAL, "interface DOF lookup past the coarsest level");
                                const uint32_t f1 = p1.f, f2 = p2.f;
                                const int id1 = p1.id, id2 = p2.id;
                                const float v = p1.w * p2.w * e;
                                const bool a1 = f1 & (N_ACTIVE | N_COARSE_SHARED), a2 = f2 & (N_ACTIVE | N_COARSE_SHARED);
                                if ((f1 & N_INTERFACE) && (f2 & N_INTERFACE))
                                    W.arr_terms[m - 1].push_back({{id1, id2}, v});
                                if (a1 && (id1 < 0 || id1 >= nrow))
                                    throw Error(HDD_ERR_INTERNAL, "interior DOF number out of range");
                                if (a1 && a2) {
                                    auto& row = aii_rows[id1];
                                    size_t k = 0;
                                    while (k < row.size() && row[k].first != id2) ++k;
                                    if (k == row.size()) row.push_back({id2, 0.0f});
                                    row[k].second += v;
                                }
                                if (a1 && (f2 & N_INTERFACE)) {
                                    auto& row = air_rows[id1];
                                    size_t k = 0;
                                    while (k < row.size() && row[k].first != id2) ++k;
                                    if (k == row.size()) {
                                        row.push_back({id2, W.air_terms[m - 1].size()});
                                        W.air_terms[m - 1].push_back({{id1, id2}, v});
                                    } else W.air_terms[m - 1][row[k].second].second += v;
                                }
                            }
                    }
            }
        }
        const int ni = node_count[m];
        W.n_int[m - 1] = ni;
        // Aii in CSR with explicit zeros dropped (Convert_To_Eigen, lines 687-705).
        CsrF& A = W.aii[m - 1];
        A.rows = A.cols = ni;
        A.ptr.assign(ni + 1, 0);
        A.col.clear();
        A.val.clear();
        for (int r = 0; r < ni; ++r) {
            auto& row = aii_rows[r];
            std::sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            for (const auto& t : row)
                if (t.second != 0.0f) { A.col.push_back(t.first); A.val.push_back(t.second); }
            A.ptr[r + 1] = (int)A.col.size();
        }
    }
}

CsrF csr_from_pairs(int rows, int cols, std::vector<std::pair<uint64_t, float>>& e) {
    e.erase(std::remove_if(e.begin(), e.end(), [](const auto& t) { return t.second == 0.0f; }), e.end());
    std::sort(e.begin(), e.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    CsrF A;
    A.rows = rows;
    A.cols = cols;
    A.ptr.assign(rows + 1, 0);
    for (auto& t : e) A.ptr[(int)(t.first >> 32) + 1]++;
    for (int r = 0; r < rows; ++r) A.ptr[r + 1] += A.ptr[r];
    A.col.resize(e.size());
    A.val.resize(e.size());
    for (size_t i = 0; i < e.size(); ++i) { A.col[i] = (int)(uint32_t)e[i].first; A.val[i] = e[i].second; }
    return A;
}

}  // namespace

void build_interface(const DomainLayout& L, int M, InterfaceHost& out) {
    const int* size = L.opt.size;
    const int* sub = L.opt.sub;
    int ns[3];
    number_of_subdomains(size, sub, ns);
    const int nsub = ns[0] * ns[1] * ns[2];
    static const std::array<M8, 8> P = bake_prolongation();
    std::vector<BoxWork> work(nsub);
    std::vector<std::string> errors(nsub);
#pragma omp parallel for schedule(dynamic)
    for (int s = 0; s < nsub; ++s) {
        try {
            const int i = s / (ns[1] * ns[2]), j = (s / ns[2]) % ns[1], k = s % ns[2];
            BoxWork& W = work[s];
            W.lo = {i * sub[0], j * sub[1], k * sub[2]};
            W.hi = {W.lo[0] + sub[0], W.lo[1] + sub[1], W.lo[2] + sub[2]};
            for (int a = 0; a < 3; ++a) W.e1[a] = sub[a] + 1;
            // Subdomain node flags: Active cells of the box (the splitter's temporary
            // Boundary marks), other non-zero flags kept; cells without an Active
            // face neighbour inside the box dropped; box-face Active cells become
            // Interface (Domain_Divider on the box).
            std::vector<uint32_t> t((size_t)W.e1[0] * W.e1[1] * W.e1[2], 0u);
            auto lid = [&](int x, int y, int z) { return ((size_t)x * W.e1[1] + y) * W.e1[2] + z; };
            for (int x = 0; x < W.e1[0]; ++x)
                for (int y = 0; y < W.e1[1]; ++y)
                    for (int z = 0; z < W.e1[2]; ++z) {
                        const int gi = W.lo[0] + x, gj = W.lo[1] + y, gk = W.lo[2] + z;
                        uint32_t f0 = 0;
                        if (gi < size[0] && gj < size[1] && gk < size[2]) f0 = L.flags_in[L.dense_index(gi, gj, gk)];
                        t[lid(x, y, z)] = (f0 & F_ACTIVE) ? F_ACTIVE : f0;
                    }
            W.sub_flags.assign(t.size(), 0u);
            for (int x = 0; x < W.e1[0]; ++x)
                for (int y = 0; y < W.e1[1]; ++y)
                    for (int z = 0; z < W.e1[2]; ++z) {
                        uint32_t v = t[lid(x, y, z)];
                        if (!v) continue;
                        bool nb = false;
                        const int d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
                        for (int f = 0; f < 6 && !nb; ++f) {
                            const int a = x + d[f][0], b = y + d[f][1], c = z + d[f][2];
                            if (a < 0 || b < 0 || c < 0 || a >= W.e1[0] || b >= W.e1[1] || c >= W.e1[2]) continue;
                            if (t[lid(a, b, c)] & F_ACTIVE) nb = true;
                        }
                        if (!nb) continue;
                        const int gi = W.lo[0] + x, gj = W.lo[1] + y, gk = W.lo[2] + z;
                        if ((v & F_ACTIVE) && (gi % sub[0] == 0 || gj % sub[1] == 0 || gk % sub[2] == 0))
                            v = (v - F_ACTIVE) | F_INTERFACE;
                        W.sub_flags[lid(x, y, z)] = v;
                    }
            process_box(W, M, P);
            std::vector<uint32_t>().swap(W.sub_flags);  // not needed by the merge below
        } catch (const std::exception& e) {
            errors[s] = e.what();
        }
    }
    for (auto& e : errors)
        if (!e.empty()) throw Error(HDD_ERR_UNSUPPORTED, "interface assembly: " + e);

    // Serial merge in subdomain order: global interface numbering (first
    // encounter) and the per-key summation of Arr across subdomains.
    out.M = M;
    out.n_sub = nsub;
    out.n_iface.assign(M, 0);
    out.iface_map.clear();
    out.Arr.assign(M, CsrF());
    out.Aii.assign(M, std::vector<CsrF>(nsub));
    out.Air.assign(M, std::vector<CsrF>(nsub));
    out.iface_xyz.assign(M, {});
    out.aii_xyz.assign(M, std::vector<std::vector<std::array<int, 3>>>(nsub));
    // Per level: (node key, global number) of every interface DOF, sorted by key
    // (the prolongation below looks coarse DOFs up in it).
    std::vector<std::vector<std::pair<uint64_t, int>>> gkeys(M);
    auto node_key = [](const I3& nd) {
        return ((uint64_t)nd[0] << 42) | ((uint64_t)nd[1] << 21) | (uint64_t)nd[2];
    };
    for (int m = 0; m < M; ++m) {
        // Global numbers in first-encounter order over (subdomain, local
        // index): the entries sorted by (key, position) give each key's first
        // encounter, and numbering the first encounters in position order gives
        // the reference's order.
        std::vector<long long> off((size_t)nsub + 1, 0);
        for (int s = 0; s < nsub; ++s) off[(size_t)s + 1] = off[s] + (long long)work[s].iface_nodes[m].size();
        const long long T = off[nsub];
        std::vector<std::pair<uint64_t, long long>> ent((size_t)T);
#pragma omp parallel for schedule(dynamic, 16)
        for (int s = 0; s < nsub; ++s) {
            const std::vector<I3>& nodes = work[s].iface_nodes[m];
            for (size_t i = 0; i < nodes.size(); ++i) ent[(size_t)off[s] + i] = {node_key(nodes[i]), off[s] + (long long)i};
        }
        __gnu_parallel::sort(ent.begin(), ent.end());
        std::vector<char> first((size_t)T, 0);
        for (long long k = 0; k < T; ++k)
            if (k == 0 || ent[k].first != ent[k - 1].first) first[(size_t)ent[k].second] = 1;
        std::vector<int> number((size_t)T, -1);  // the DOF number at its first encounter
        int nfirst = 0;
        for (long long e = 0; e < T; ++e)
            if (first[(size_t)e]) number[(size_t)e] = nfirst++;
        out.n_iface[m] = nfirst;
        std::vector<int> flat((size_t)T);
        gkeys[m].reserve((size_t)nfirst);
        for (long long k = 0, cur = -1; k < T; ++k) {
            if (k == 0 || ent[k].first != ent[k - 1].first) {
                cur = number[(size_t)ent[k].second];
                gkeys[m].push_back({ent[k].first, (int)cur});
            }
            flat[(size_t)ent[k].second] = (int)cur;
        }
        std::vector<std::pair<uint64_t, long long>>().swap(ent);
        if (m == 0) out.iface_map.resize((size_t)nfirst);
        out.iface_xyz[m].resize((size_t)nfirst);
        std::vector<std::vector<int>> to_g(nsub);
#pragma omp parallel for schedule(dynamic, 16)
        for (int s = 0; s < nsub; ++s) {
            const std::vector<I3>& nodes = work[s].iface_nodes[m];
            to_g[s].assign(flat.begin() + off[s], flat.begin() + off[(size_t)s + 1]);
            for (size_t i = 0; i < nodes.size(); ++i) {
                const long long e = off[s] + (long long)i;
                if (!first[(size_t)e]) continue;
                const I3& nd = nodes[i];
                if (m == 0) out.iface_map[(size_t)number[(size_t)e]] = nd;
                out.iface_xyz[m][(size_t)number[(size_t)e]] = {nd[0] << m, nd[1] << m, nd[2] << m};
            }
        }
        const int nif = out.n_iface[m];
        // Arr: each entry is the float sum of its terms in (subdomain, term)
        // order, starting from 0.  The terms are bucketed by row in that order
        // (a serial fill), then every row sums its columns on its own.
        std::vector<long long> row_ptr((size_t)nif + 1, 0);
        for (int s = 0; s < nsub; ++s)
            for (const auto& tv : work[s].arr_terms[m]) row_ptr[(size_t)to_g[s][tv.first.first] + 1]++;
        for (int r = 0; r < nif; ++r) row_ptr[r + 1] += row_ptr[r];
        std::vector<std::pair<int, float>> bucket((size_t)row_ptr[nif]);
        {
            std::vector<long long> fill(row_ptr.begin(), row_ptr.end() - 1);
            for (int s = 0; s < nsub; ++s) {
                for (const auto& tv : work[s].arr_terms[m])
                    bucket[(size_t)fill[to_g[s][tv.first.first]]++] = {to_g[s][tv.first.second], tv.second};
                std::vector<std::pair<std::pair<int, int>, float>>().swap(work[s].arr_terms[m]);
            }
        }
        std::vector<int> row_nnz(nif, 0);
#pragma omp parallel for schedule(dynamic, 256)
        for (int r = 0; r < nif; ++r) {
            auto* b = bucket.data() + row_ptr[r];
            auto* e = bucket.data() + row_ptr[r + 1];
            std::stable_sort(b, e, [](const auto& x, const auto& y) { return x.first < y.first; });
            int w = 0;  // compacted (column, sum) pairs written from b
            for (auto* p = b; p != e;) {
                const int c = p->first;
                float acc = 0.0f;
                for (; p != e && p->first == c; ++p) acc += p->second;
                if (acc != 0.0f) b[w++] = {c, acc};  // explicit zeros dropped, as csr_from_pairs does
            }
            row_nnz[r] = w;
        }
        CsrF& A = out.Arr[m];
        A.rows = A.cols = nif;
        A.ptr.assign((size_t)nif + 1, 0);
        for (int r = 0; r < nif; ++r) A.ptr[r + 1] = A.ptr[r] + row_nnz[r];
        A.col.resize((size_t)A.ptr[nif]);
        A.val.resize((size_t)A.ptr[nif]);
#pragma omp parallel for schedule(dynamic, 256)
        for (int r = 0; r < nif; ++r) {
            const auto* b = bucket.data() + row_ptr[r];
            for (int i = 0; i < row_nnz[r]; ++i) {
                A.col[(size_t)A.ptr[r] + i] = b[i].first;
                A.val[(size_t)A.ptr[r] + i] = b[i].second;
            }
        }
        std::vector<std::pair<int, float>>().swap(bucket);
        // Air and Aii per subdomain (independent).
#pragma omp parallel for schedule(dynamic)
        for (int s = 0; s < nsub; ++s) {
            BoxWork& W = work[s];
            std::vector<std::pair<uint64_t, float>> ap;
            ap.reserve(W.air_terms[m].size());
            for (auto& tv : W.air_terms[m])
                ap.push_back({((uint64_t)(uint32_t)tv.first.first << 32) | (uint32_t)to_g[s][tv.first.second], tv.second});
            out.Air[m][s] = csr_from_pairs(W.n_int[m], nif, ap);
            out.Aii[m][s] = std::move(W.aii[m]);
            out.aii_xyz[m][s] = std::move(W.int_xyz[m]);
        }
        if (m == 0)
            for (int r = 0; r < out.Arr[0].rows; ++r) {
                bool diag = false;
                for (int p = out.Arr[0].ptr[r]; p < out.Arr[0].ptr[r + 1]; ++p)
                    if (out.Arr[0].col[p] == r) diag = true;
                if (!diag) throw Error(HDD_ERR_INTERNAL, "zero diagonal in the level-0 interface matrix");
            }
    }
    // Interface prolongation Prr[m]: fine level m -> coarse level m+1.  Row id
    // holds fine DOF id's (at most 8) coarse parents with positive trilinear
    // weight, columns ascending: the fine DOFs are visited in parallel, each
    // filling its own row.
    out.Prr.assign(M > 1 ? M - 1 : 0, CsrF());
    for (int m = 0; m + 1 < M; ++m) {
        const int nf = out.n_iface[m];
        std::vector<std::array<std::pair<int, float>, 8>> ent(nf);
        std::vector<int> cnt(nf, 0);
#pragma omp parallel for schedule(static)
        for (int id = 0; id < nf; ++id) {
            const std::array<int, 3>& X = out.iface_xyz[m][id];
            const I3 F = {X[0] >> m, X[1] >> m, X[2] >> m};
            int base[3];
            for (int v = 0; v < 3; ++v) base[v] = (int)std::floor(F[v] / 2.0);
            int k = 0;
            for (int ci = 0; ci < 8; ++ci) {
                const I3 C = {base[0] + (ci >> 2), base[1] + ((ci >> 1) & 1), base[2] + (ci & 1)};
                float w = 1.0f;
                for (int v = 0; v < 3; ++v) w *= (2.0f - std::abs(C[v] * 2 - F[v])) / 2.0;
                if (!(w > 0)) continue;
                const uint64_t ck = ((uint64_t)C[0] << 42) | ((uint64_t)C[1] << 21) | (uint64_t)C[2];
                const auto& keys = gkeys[m + 1];
                auto it = std::lower_bound(keys.begin(), keys.end(), std::make_pair(ck, INT_MIN));
                if (it == keys.end() || it->first != ck) continue;
                ent[id][k++] = {it->second, w};
            }
            std::sort(ent[id].begin(), ent[id].begin() + k,
                      [](const auto& x, const auto& y) { return x.first < y.first; });
            cnt[id] = k;
        }
        CsrF& P = out.Prr[m];
        P.rows = nf;
        P.cols = out.n_iface[m + 1];
        P.ptr.assign((size_t)nf + 1, 0);
        for (int id = 0; id < nf; ++id) P.ptr[id + 1] = P.ptr[id] + cnt[id];
        P.col.resize((size_t)P.ptr[nf]);
        P.val.resize((size_t)P.ptr[nf]);
#pragma omp parallel for schedule(static)
        for (int id = 0; id < nf; ++id)
            for (int k = 0; k < cnt[id]; ++k) {
                P.col[(size_t)P.ptr[id] + k] = ent[id][k].first;
                P.val[(size_t)P.ptr[id] + k] = ent[id][k].second;
            }
    }
}

void build_second_level(const DomainLayout& L, const int sub[3], int M, InterfaceHost& out) {
    // Two-level DD (TWO/SPGrid_Domain_Decomposition_Solver/SPGrid_Subdomain_Splitter.h:168-193):
    // every first-level subdomain box [lo, lo + sub] gets its own interface
    // system, from the caller's flags with the Active cells on the
    // first-level planes made Dirichlet (Domain_Divider with clear_flag),
    // split at sub/2.  Each box is assembled as a grid of its own (origin lo,
    // a multiple of sub, so the plane tests are the global ones); the
    // systems with a level-0 interface are then stacked in box order (x
    // slowest) into one block-diagonal system.  They are not assembled as
    // one grid: coarse interface nodes on a first-level plane would then be
    // shared by the boxes on either side.
    const int* size = L.opt.size;
    int ns[3], sub2[3];
    number_of_subdomains(size, sub, ns);
    for (int a = 0; a < 3; ++a) sub2[a] = sub[a] / 2;
    const int nbox = ns[0] * ns[1] * ns[2];
    std::vector<InterfaceHost> part(nbox);
    std::vector<std::array<int, 3>> lo(nbox);
    std::vector<std::string> errors(nbox);
#pragma omp parallel for schedule(dynamic)
    for (int s = 0; s < nbox; ++s) {
        try {
            const int b[3] = {s / (ns[1] * ns[2]), (s / ns[2]) % ns[1], s % ns[2]};
            DomainLayout Ls;
            Ls.opt = L.opt;
            for (int a = 0; a < 3; ++a) {
                lo[s][a] = b[a] * sub[a];
                Ls.opt.size[a] = std::min(sub[a] + 1, size[a] - lo[s][a]);
                Ls.opt.sub[a] = sub2[a];
            }
            const int* ld = Ls.opt.size;
            Ls.flags_in.assign((size_t)ld[0] * ld[1] * ld[2], 0u);
            for (int x = 0; x < ld[0]; ++x)
                for (int y = 0; y < ld[1]; ++y)
                    for (int z = 0; z < ld[2]; ++z)
                        Ls.flags_in[((size_t)x * ld[1] + y) * ld[2] + z] =
                            L.flags_in[L.dense_index(lo[s][0] + x, lo[s][1] + y, lo[s][2] + z)];
            clear_planes(ld, sub, Ls.flags_in.data());
            build_interface(Ls, M, part[s]);
        } catch (const std::exception& e) {
            errors[s] = e.what();
        }
    }
    for (auto& e : errors)
        if (!e.empty()) throw Error(HDD_ERR_UNSUPPORTED, "second-level interface assembly: " + e);
    out = InterfaceHost();
    out.M = M;
    out.n_iface.assign(M, 0);
    out.Arr.assign(M, CsrF());
    out.Aii.assign(M, {});
    out.Air.assign(M, {});
    out.iface_xyz.assign(M, {});
    out.aii_xyz.assign(M, {});
    out.Prr.assign(M > 1 ? M - 1 : 0, CsrF());
    auto append = [](CsrF& A, const CsrF& B, int col0) {
        // B's rows appended to A's, its columns shifted by col0.
        if (A.ptr.empty()) A.ptr.assign(1, 0);
        for (int r = 0; r < B.rows; ++r) {
            for (int p = B.ptr[r]; p < B.ptr[r + 1]; ++p) {
                A.col.push_back(B.col[p] + col0);
                A.val.push_back(B.val[p]);
            }
            A.ptr.push_back((int)A.col.size());
        }
    };
    for (int s = 0; s < nbox; ++s) {
        const InterfaceHost& P = part[s];
        if (P.n_iface.empty() || P.n_iface[0] == 0) continue;
        if (P.M != M) throw Error(HDD_ERR_INTERNAL, "second-level system with another level count");
        const std::array<int, 3>& o = lo[s];
        std::vector<int> off(M);
        for (int m = 0; m < M; ++m) off[m] = out.n_iface[m];
        for (const auto& c : P.iface_map) out.iface_map.push_back({c[0] + o[0], c[1] + o[1], c[2] + o[2]});
        for (int m = 0; m < M; ++m) {
            append(out.Arr[m], P.Arr[m], off[m]);
            if (m + 1 < M) append(out.Prr[m], P.Prr[m], off[m + 1]);
            for (const auto& x : P.iface_xyz[m]) out.iface_xyz[m].push_back({x[0] + o[0], x[1] + o[1], x[2] + o[2]});
            for (int b = 0; b < P.n_sub; ++b) {
                out.Aii[m].push_back(P.Aii[m][b]);
                CsrF air;
                air.rows = P.Air[m][b].rows;
                append(air, P.Air[m][b], off[m]);
                out.Air[m].push_back(std::move(air));
                std::vector<std::array<int, 3>> xyz;
                for (const auto& x : P.aii_xyz[m][b]) xyz.push_back({x[0] + o[0], x[1] + o[1], x[2] + o[2]});
                out.aii_xyz[m].push_back(std::move(xyz));
            }
            out.n_iface[m] += P.n_iface[m];
        }
        out.n_sub += P.n_sub;
    }
    for (int m = 0; m < M; ++m) {
        out.Arr[m].rows = out.Arr[m].cols = out.n_iface[m];
        if (out.Arr[m].ptr.empty()) out.Arr[m].ptr.assign(1, 0);
        for (auto& A : out.Air[m]) A.cols = out.n_iface[m];
        if (m + 1 < M) {
            CsrF& Pm = out.Prr[m];
            Pm.rows = out.n_iface[m];
            Pm.cols = out.n_iface[m + 1];
            if (Pm.ptr.empty()) Pm.ptr.assign(1, 0);
        }
    }
}

}  // namespace hdd
