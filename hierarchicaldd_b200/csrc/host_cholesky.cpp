// Supernodal multifrontal Cholesky of (A + eps I) on the host.
//
// Stands in for MKL PARDISO (SPD, mtype 2) that the reference uses for the
// interface matrix and every subdomain interior matrix
// (CPU/Interface_Solver/SIGMA_SMOOTHER.cpp:175-237 builds A + 1e-5 I with a
// 1e-5 diagonal for empty rows; phases 11/22 factor it).  The ordering is a
// nested dissection: median planes through the DOF positions when they are
// known, breadth-first level structures otherwise; every separator (and every
// leaf block) is one dense front, so the factor is a tree of dense blocks that
// the GPU solves level by level.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <functional>
#include <numeric>
#include <string>

#include <omp.h>

#include "sigma.h"

namespace hdd {

namespace {
constexpr int kLeaf = 32;

// Trailing update of a front after a panel of kb columns starting at k0: for
// the columns c in [c0, c0 + kColBlock) (clipped to f) and every row i >= c,
//   F(i, c) -= sum_{kk < kb} F(i, k0 + kk) * F(c, k0 + kk),
// F column-major with leading dimension f.  The panel rows t0..f-1 are read
// from P, packed by pack_panel in blocks of kRowBlock rows so that each kk
// step reads one contiguous run.  Each sum starts at 0 and adds its products
// in kk order, whatever the blocking, so the result does not depend on the
// instruction set or the thread that runs it (no FMA contraction: the library
// is built with -ffp-contract=off).  kColBlock x kRowBlock independent
// accumulators vectorise over the rows; the AVX-512 or AVX2 clone is picked at
// load time where the CPU has it.  c0 - t0 is a multiple of kColBlock.
constexpr int kColBlock = 4;
constexpr int kRowBlock = 8;

// P[(r * kb + kk) * kRowBlock + a] = F(t0 + r * kRowBlock + a, k0 + kk), zero
// past row f - 1.
void pack_panel(const double* F, int f, int k0, int kb, int t0, std::vector<double>& P) {
    const int nrb = (f - t0 + kRowBlock - 1) / kRowBlock;
    P.assign((size_t)nrb * kb * kRowBlock, 0.0);
    for (int kk = 0; kk < kb; ++kk) {
        const double* col = F + (size_t)(k0 + kk) * f;
        for (int i = t0; i < f; ++i) {
            const int r = (i - t0) / kRowBlock, a = (i - t0) % kRowBlock;
            P[((size_t)r * kb + kk) * kRowBlock + a] = col[i];
        }
    }
}

__attribute__((target_clones("avx512f", "avx2", "default")))
void trailing_update(double* F, int f, const double* P, int kb, int t0, int c0) {
    const int cn = std::min(kColBlock, f - c0);
    const int rc = (c0 - t0) / kRowBlock, ac = (c0 - t0) % kRowBlock;
    const int nrb = (f - t0 + kRowBlock - 1) / kRowBlock;
    const double* Pc = P + (size_t)rc * kb * kRowBlock + ac;
    for (int r = rc; r < nrb; ++r) {
        const double* Pr = P + (size_t)r * kb * kRowBlock;
        double acc[kColBlock][kRowBlock];
        for (int b = 0; b < kColBlock; ++b)
            for (int a = 0; a < kRowBlock; ++a) acc[b][a] = 0.0;
        for (int kk = 0; kk < kb; ++kk) {
            double l[kColBlock];
            for (int b = 0; b < kColBlock; ++b) l[b] = Pc[(size_t)kk * kRowBlock + b];
            const double* pr = Pr + (size_t)kk * kRowBlock;
            for (int b = 0; b < kColBlock; ++b)
                for (int a = 0; a < kRowBlock; ++a) acc[b][a] += pr[a] * l[b];
        }
        const int i0 = t0 + r * kRowBlock;
        for (int b = 0; b < cn; ++b) {
            double* col = F + (size_t)(c0 + b) * f;
            for (int a = 0; a < kRowBlock; ++a) {
                const int i = i0 + a;
                if (i >= c0 + b && i < f) col[i] -= acc[b][a];
            }
        }
    }
}
}

void SnFactor::analyze(const CsrF& A, const std::vector<std::array<int, 3>>* xyz) {
    n = A.rows;
    // Symmetric adjacency without self loops: every off-diagonal entry (r, c)
    // gives c to r's list and r to c's; each list is then sorted and
    // deduplicated, so the fill order (parallel, atomic slots) does not matter.
    std::vector<int> adjp(n + 1, 0), adj;
    {
        std::vector<int> deg(n, 0);
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; ++r)
            for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) {
                const int c = A.col[p];
                if (c == r) continue;
#pragma omp atomic
                deg[r]++;
#pragma omp atomic
                deg[c]++;
            }
        std::vector<long long> start((size_t)n + 1, 0);
        for (int r = 0; r < n; ++r) start[(size_t)r + 1] = start[r] + deg[r];
        std::vector<int> raw((size_t)start[n]);
        std::vector<int> fill(n, 0);
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; ++r)
            for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) {
                const int c = A.col[p];
                if (c == r) continue;
                int kr, kc;
#pragma omp atomic capture
                kr = fill[r]++;
#pragma omp atomic capture
                kc = fill[c]++;
                raw[(size_t)start[r] + kr] = c;
                raw[(size_t)start[c] + kc] = r;
            }
#pragma omp parallel for schedule(dynamic, 1024)
        for (int r = 0; r < n; ++r) {
            int* b = raw.data() + start[r];
            int* e = raw.data() + start[(size_t)r + 1];
            std::sort(b, e);
            deg[r] = (int)(std::unique(b, e) - b);
        }
        for (int r = 0; r < n; ++r) adjp[r + 1] = adjp[r] + deg[r];
        adj.resize((size_t)adjp[n]);
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; ++r)
            std::copy(raw.data() + start[r], raw.data() + start[r] + deg[r], adj.data() + adjp[r]);
    }

    perm.clear();
    perm.reserve(n);
    col0.clear(); ncol.clear(); parent.clear(); rows.clear();
    // The recursion splits a vertex set into parts ordered first and a
    // separator ordered after them.  Each call returns the supernodes of its
    // set in post-order (its own list, so large parts run as OpenMP tasks);
    // the caller appends the lists in the order the serial recursion creates
    // them (first part, second part, separator), so the ordering is the same
    // for any number of threads.  part[] marks which set a vertex belongs to
    // (ids are unique; a task only writes the ids of its own vertices, and it
    // only compares a neighbour's id with its own, so it reads them relaxed);
    // level[] is only touched for vertices of the caller's own set.
    struct Node { std::vector<int> cols, kids; };
    struct Sub { std::vector<Node> nodes; std::vector<int> roots; };
    auto append = [](Sub& to, Sub&& from) {
        const int off = (int)to.nodes.size();
        for (Node& nd : from.nodes) {
            for (int& k : nd.kids) k += off;
            to.nodes.push_back(std::move(nd));
        }
        for (int r : from.roots) to.roots.push_back(r + off);
    };
    auto leaf = [](std::vector<int> cols) {
        Sub s;
        s.nodes.push_back({std::move(cols), {}});
        s.roots.push_back(0);
        return s;
    };
    // Separator node over the roots of `s` (appended last).
    auto close = [](Sub& s, std::vector<int> cols) {
        Node nd{std::move(cols), s.roots};
        s.nodes.push_back(std::move(nd));
        s.roots.assign(1, (int)s.nodes.size() - 1);
    };
    std::vector<int> part(n, 0), level(n, -1);
    std::atomic<int> next_part{1};
    auto get_part = [&](int v) { return __atomic_load_n(&part[v], __ATOMIC_RELAXED); };
    auto set_part = [&](int v, int id) { __atomic_store_n(&part[v], id, __ATOMIC_RELAXED); };
    auto bfs = [&](int src, int pid, std::vector<int>& seen) {
        // seen doubles as the queue: vertices are appended in visiting order.
        size_t qh = seen.size();
        int last = src;
        level[src] = 0;
        seen.push_back(src);
        while (qh < seen.size()) {
            const int v = seen[qh++];
            last = v;
            for (int p = adjp[v]; p < adjp[v + 1]; ++p) {
                const int w = adj[p];
                if (get_part(w) != pid || level[w] >= 0) continue;
                level[w] = level[v] + 1;
                seen.push_back(w);
            }
        }
        return last;
    };
    constexpr size_t kTaskMin = 16384;  // parts at least this large run as tasks
    std::function<Sub(std::vector<int>&, int)> rec = [&](std::vector<int>& verts, int pid) -> Sub {
        if ((int)verts.size() <= kLeaf) return leaf(verts);
        std::vector<int> comp;
        const int far = bfs(verts[0], pid, comp);
        for (int v : comp) level[v] = -1;
        if (comp.size() < verts.size()) {
            // Disconnected: order the components one after another.  All
            // components are found in one pass over verts (each breadth-first
            // from its first vertex in verts order), so a set of many small
            // components costs linear time and no recursion depth.  Component
            // i is ordered on its own (BFS order), except that once the
            // remaining components hold at most kLeaf vertices they form one
            // leaf, and the last component is ordered from its vertices in
            // verts order: the ordering of peeling one component at a time.
            std::vector<std::vector<int>> comps;
            std::vector<int> ids;
            ids.push_back(next_part++);
            for (int v : comp) set_part(v, ids.back());
            comps.push_back(std::move(comp));
            for (int v : verts) {
                if (get_part(v) != pid) continue;
                std::vector<int> c;
                bfs(v, pid, c);
                for (int w : c) level[w] = -1;
                ids.push_back(next_part++);
                for (int w : c) set_part(w, ids.back());
                comps.push_back(std::move(c));
            }
            Sub out;
            size_t remaining = verts.size();
            for (size_t i = 0; i < comps.size(); ++i) {
                if (i > 0 && remaining <= (size_t)kLeaf) {
                    std::vector<int> rest;
                    for (int v : verts) {
                        const int pv = get_part(v);
                        if (pv >= ids[i] && pv <= ids.back()) rest.push_back(v);
                    }
                    append(out, leaf(std::move(rest)));
                    break;
                }
                if (i > 0 && i + 1 == comps.size()) {
                    std::vector<int> last;
                    for (int v : verts)
                        if (get_part(v) == ids[i]) last.push_back(v);
                    append(out, rec(last, ids[i]));
                } else {
                    append(out, rec(comps[i], ids[i]));
                }
                remaining -= comps[i].size();
            }
            return out;
        }
        // Orders the two parts (the first as a task when both are large) and
        // closes them with the separator.
        auto split = [&](std::vector<int>& Av, std::vector<int>& Sv, std::vector<int>& Bv) -> Sub {
            const int pa = next_part++, pb = next_part++;
            for (int v : Av) set_part(v, pa);
            for (int v : Bv) set_part(v, pb);
            for (int v : Sv) set_part(v, -1);
            Sub ra, rb;
            if (Av.size() >= kTaskMin && Bv.size() >= kTaskMin && omp_in_parallel()) {
#pragma omp task shared(ra, Av)
                ra = rec(Av, pa);
                rb = rec(Bv, pb);
#pragma omp taskwait
            } else {
                ra = rec(Av, pa);
                rb = rec(Bv, pb);
            }
            append(ra, std::move(rb));
            close(ra, std::move(Sv));
            return ra;
        };
        if (xyz) {
            // Geometric split: for each axis, cut at the median position; the
            // separator is the smaller of the two one-sided boundary layers.
            // Keep the axis with the smallest separator.
            int best_axis = -1;
            size_t best_sep = 0;
            int best_cut = 0, best_side = 0;
            std::vector<int> pos(verts.size());
            for (int ax = 0; ax < 3; ++ax) {
                for (size_t i = 0; i < verts.size(); ++i) pos[i] = (*xyz)[verts[i]][ax];
                const size_t mid = pos.size() / 2;
                std::nth_element(pos.begin(), pos.begin() + mid, pos.end());
                int cut = pos[mid];
                size_t nleft = 0, nle = 0;
                for (int v : verts) {
                    nleft += (*xyz)[v][ax] < cut;
                    nle += (*xyz)[v][ax] <= cut;
                }
                if (nleft == 0) {
                    if (nle == verts.size()) continue;  // all at one position along this axis
                    cut += 1;                           // left = positions <= median
                }
                size_t sl = 0, sr = 0;
                for (int v : verts) {
                    const bool left = (*xyz)[v][ax] < cut;
                    for (int p = adjp[v]; p < adjp[v + 1]; ++p) {
                        const int w = adj[p];
                        if (get_part(w) != pid) continue;
                        if (((*xyz)[w][ax] < cut) != left) {
                            (left ? sl : sr)++;
                            break;
                        }
                    }
                }
                const size_t sep = std::min(sl, sr);
                if (best_axis < 0 || sep < best_sep) {
                    best_axis = ax;
                    best_sep = sep;
                    best_cut = cut;
                    best_side = sl <= sr ? 0 : 1;
                }
            }
            if (best_axis >= 0) {
                // best_side 0: separator taken from the left layer.
                std::vector<int> Av, Sv, Bv;
                for (int v : verts) {
                    const bool left = (*xyz)[v][best_axis] < best_cut;
                    const bool on_sep_side = (best_side == 0) == left;
                    bool boundary = false;
                    if (on_sep_side)
                        for (int p = adjp[v]; p < adjp[v + 1] && !boundary; ++p) {
                            const int w = adj[p];
                            if (get_part(w) == pid && ((*xyz)[w][best_axis] < best_cut) != left) boundary = true;
                        }
                    if (boundary) Sv.push_back(v);
                    else if (left) Av.push_back(v);
                    else Bv.push_back(v);
                }
                if (!Av.empty() && !Bv.empty()) return split(Av, Sv, Bv);
            }
        }
        comp.clear();
        bfs(far, pid, comp);
        int h = 0;
        for (int v : comp) h = std::max(h, level[v]);
        if (h < 2) {
            for (int v : comp) level[v] = -1;
            return leaf(verts);
        }
        std::vector<int> cnt(h + 1, 0);
        for (int v : comp) cnt[level[v]]++;
        // Separator level: the smallest level set in the middle half.
        const int total = (int)verts.size();
        int best = -1, best_size = 0, acc = 0;
        for (int l = 1; l < h; ++l) {
            acc += cnt[l - 1];
            if (acc < total / 4 || acc > (3 * total) / 4) continue;
            if (best < 0 || cnt[l] < best_size) { best = l; best_size = cnt[l]; }
        }
        if (best < 0) {
            acc = 0;
            for (int l = 0; l <= h; ++l) {
                acc += cnt[l];
                if (acc >= total / 2) { best = std::max(1, std::min(l, h - 1)); break; }
            }
        }
        std::vector<int> Av, Sv, Bv;
        for (int v : comp) {
            if (level[v] < best) Av.push_back(v);
            else if (level[v] == best) Sv.push_back(v);
            else Bv.push_back(v);
            level[v] = -1;
        }
        return split(Av, Sv, Bv);
    };
    std::vector<int> all(n);
    std::iota(all.begin(), all.end(), 0);
    Sub top;
    if (n > 0) {
#pragma omp parallel if (n >= (int)(4 * kTaskMin) && !omp_in_parallel())
#pragma omp single
        top = rec(all, 0);
    }
    for (size_t k = 0; k < top.nodes.size(); ++k) {
        col0.push_back((int)perm.size());
        ncol.push_back((int)top.nodes[k].cols.size());
        parent.push_back(-1);
        perm.insert(perm.end(), top.nodes[k].cols.begin(), top.nodes[k].cols.end());
    }
    for (size_t k = 0; k < top.nodes.size(); ++k)
        for (int c : top.nodes[k].kids) parent[c] = (int)k;

    // Row structure of every front (symbolic factorisation).
    std::vector<int> iperm(n);
    for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
    const int ns = (int)col0.size();
    rows.assign(ns, {});
    std::vector<std::vector<int>> kids(ns);
    for (int j = 0; j < ns; ++j)
        if (parent[j] >= 0) kids[parent[j]].push_back(j);
    std::vector<int> mark(n, -1);
    for (int j = 0; j < ns; ++j) {
        const int last = col0[j] + ncol[j] - 1;
        std::vector<int>& R = rows[j];
        for (int c = col0[j]; c <= last; ++c) {
            const int old = perm[c];
            for (int p = A.ptr[old]; p < A.ptr[old + 1]; ++p) {
                const int i = iperm[A.col[p]];
                if (i > last && mark[i] != j) { mark[i] = j; R.push_back(i); }
            }
        }
        for (int c : kids[j])
            for (int i : rows[c])
                if (i > last && mark[i] != j) { mark[i] = j; R.push_back(i); }
        std::sort(R.begin(), R.end());
    }
}

namespace {
// Columns c0 .. c0+cn-1 (cn <= kSolveGroup) of Fw = [L^{-1}; -L_RJ L^{-1}] for
// one front, column c at Fw + c*m with m = nj + nr (cleared here): forward
// substitution of e_c through L (nj x nj, col-major), then w = -R x with
// R = L_RJ (nr x nj, col-major).  The columns of a group share every column of
// L and R they read (a front's L and R are read once per group, not once per
// column), and each column receives its updates in the order of the
// one-column algorithm (axpy loops only), so the grouping and the vectorised
// clones give the same values.
constexpr int kSolveGroup = 8;
__attribute__((target_clones("avx512f", "avx2", "default")))
void solve_block_columns(const double* L, const double* R, int nj, int nr, int c0, int cn, double* Fw, int m) {
    double* x[kSolveGroup];
    for (int g = 0; g < cn; ++g) {
        x[g] = Fw + (size_t)(c0 + g) * m;
        std::fill(x[g], x[g] + m, 0.0);
        x[g][c0 + g] = 1.0;
    }
    for (int jj = c0; jj < nj; ++jj) {
        const double* Lc = L + (size_t)jj * nj;
        for (int g = 0; g < cn && c0 + g <= jj; ++g) {
            double* xg = x[g];
            const double xj = xg[jj] / Lc[jj];
            xg[jj] = xj;
            if (xj == 0.0) continue;
            for (int i = jj + 1; i < nj; ++i) xg[i] -= Lc[i] * xj;
        }
    }
    for (int a = c0; a < nj; ++a) {
        const double* Ra = R + (size_t)a * nr;
        for (int g = 0; g < cn && c0 + g <= a; ++g) {
            const double la = x[g][a];
            if (la == 0.0) continue;
            double* w = x[g] + nj;
            for (int k = 0; k < nr; ++k) w[k] -= Ra[k] * la;
        }
    }
}
}  // namespace

namespace {
struct FrontScratch {
    std::vector<int> pos;
    std::vector<double> front, panel;
};
}  // namespace

void SnFactor::factor(const CsrF& A, double eps) {
    const int ns = (int)col0.size();
    std::vector<int> iperm(n);
    for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
    std::vector<std::vector<int>> kids(ns);
    for (int j = 0; j < ns; ++j)
        if (parent[j] >= 0) kids[parent[j]].push_back(j);
    Ljj.assign(ns, {});
    Lrj.assign(ns, {});
    std::vector<BlockVec> upd(ns);
    // One front: assemble A's columns and the children's update matrices (in
    // child order), partial dense Cholesky, keep L_JJ, L_RJ and the update
    // matrix for the parent.  `scratch.pos` is an n-long map (all -1 on entry
    // and on exit); the front and panel buffers are reused from front to front.  The arithmetic of a front does not depend on which thread
    // runs it or on `inner_par`, so the factor is the same for any schedule.
    auto factor_front = [&](int j, FrontScratch& scratch, bool inner_par) {
        const int nj = ncol[j], nr = (int)rows[j].size(), f = nj + nr;
        // Large fronts (the separators near the root) split their clearing,
        // assembly, panel rows and copies over the threads too; every value is
        // computed by the same operations in the same order either way.
        const bool big = inner_par && (size_t)f * f > ((size_t)1 << 20);
        std::vector<int>& pos = scratch.pos;
        std::vector<double>& F = scratch.front;  // col-major, lower triangle used
        if (F.size() < (size_t)f * f) F.resize((size_t)f * f);
#pragma omp parallel for schedule(dynamic, 64) if (big)
        for (int a = 0; a < f; ++a) std::fill(F.begin() + (size_t)a * f + a, F.begin() + (size_t)(a + 1) * f, 0.0);
        for (int a = 0; a < nj; ++a) pos[col0[j] + a] = a;
        for (int k = 0; k < nr; ++k) pos[rows[j][k]] = nj + k;
        for (int a = 0; a < nj; ++a) {
            const int cnew = col0[j] + a, old = perm[cnew];
            for (int p = A.ptr[old]; p < A.ptr[old + 1]; ++p) {
                const int i = iperm[A.col[p]];
                if (i < cnew) continue;
                F[(size_t)a * f + pos[i]] += (double)A.val[p];
            }
            F[(size_t)a * f + a] += eps;
        }
        for (int c : kids[j]) {
            const std::vector<int>& rc = rows[c];
            const int m = (int)rc.size();
            const BlockVec& U = upd[c];
            // Column b of the child's update goes to front column pos[rc[b]]:
            // distinct columns, so the columns of one child run in parallel.
#pragma omp parallel for schedule(dynamic, 16) if (big)
            for (int b = 0; b < m; ++b) {
                const int pb = pos[rc[b]];
                for (int a = b; a < m; ++a) {
                    const int pa = pos[rc[a]];
                    // U is lower (a >= b); the front position order is monotone in the
                    // new index, so pa >= pb.
                    F[(size_t)pb * f + pa] += U[(size_t)b * m + a];
                }
            }
            upd[c].clear();
            upd[c].shrink_to_fit();
        }
        // Dense partial Cholesky of the front (first nj columns), blocked in
        // panels of kPanel columns: factor the panel's diagonal block, then
        // the panel rows below it (each row on its own), then update the
        // trailing columns (trailing_update).
        constexpr int kPanel = 48;
        std::vector<double>& Pk = scratch.panel;
        for (int k0 = 0; k0 < nj; k0 += kPanel) {
            const int kb = std::min(kPanel, nj - k0);
            const int t0 = k0 + kb;
            for (int k = k0; k < t0; ++k) {
                double d = F[(size_t)k * f + k];
                if (!(d > 0)) throw Error(HDD_ERR_INTERNAL, "interface matrix is not positive definite");
                d = std::sqrt(d);
                F[(size_t)k * f + k] = d;
                for (int i = k + 1; i < t0; ++i) F[(size_t)k * f + i] /= d;
                for (int c = k + 1; c < t0; ++c) {
                    const double lck = F[(size_t)k * f + c];
                    if (lck == 0.0) continue;
                    double* colc = &F[(size_t)c * f];
                    const double* colk = &F[(size_t)k * f];
                    for (int i = c; i < t0; ++i) colc[i] -= colk[i] * lck;
                }
            }
            if (t0 >= f) continue;
            constexpr int kRows = 256;
            const int nchunk = (f - t0 + kRows - 1) / kRows;
#pragma omp parallel for schedule(dynamic, 1) if (big)
            for (int q = 0; q < nchunk; ++q) {
                const int r0 = t0 + q * kRows, r1 = std::min(f, r0 + kRows);
                for (int k = k0; k < t0; ++k) {
                    const double d = F[(size_t)k * f + k];
                    double* colk = &F[(size_t)k * f];
                    for (int i = r0; i < r1; ++i) colk[i] /= d;
                    for (int c = k + 1; c < t0; ++c) {
                        const double lck = F[(size_t)k * f + c];
                        if (lck == 0.0) continue;
                        double* colc = &F[(size_t)c * f];
                        for (int i = r0; i < r1; ++i) colc[i] -= colk[i] * lck;
                    }
                }
            }
            pack_panel(F.data(), f, k0, kb, t0, Pk);
            const int nblk = (f - t0 + kColBlock - 1) / kColBlock;
            const double* P = Pk.data();
#pragma omp parallel for schedule(dynamic, 2) if (inner_par && (size_t)(f - t0) * (f - t0) * kb > 4000000)
            for (int cb = 0; cb < nblk; ++cb) trailing_update(F.data(), f, P, kb, t0, t0 + cb * kColBlock);
        }
        // Only the parts read later are written: the lower triangle of L_JJ and
        // of the update matrix, all of L_RJ.
        Ljj[j].resize((size_t)nj * nj);
        Lrj[j].resize((size_t)nr * nj);
        if (nr > 0) upd[j].resize((size_t)nr * nr);
        BlockVec& Lj = Ljj[j];
        BlockVec& Rj = Lrj[j];
        BlockVec& Uj = upd[j];
#pragma omp parallel if (big)
        {
#pragma omp for schedule(dynamic, 16) nowait
            for (int a = 0; a < nj; ++a) {
                for (int i = a; i < nj; ++i) Lj[(size_t)a * nj + i] = F[(size_t)a * f + i];
                for (int k = 0; k < nr; ++k) Rj[(size_t)a * nr + k] = F[(size_t)a * f + nj + k];
            }
#pragma omp for schedule(dynamic, 16)
            for (int b = 0; b < nr; ++b)
                for (int a = b; a < nr; ++a) Uj[(size_t)b * nr + a] = F[(size_t)(nj + b) * f + nj + a];
        }
        for (int a = 0; a < nj; ++a) pos[col0[j] + a] = -1;
        for (int k = 0; k < nr; ++k) pos[rows[j][k]] = -1;
    };

    // Schedule over the elimination tree.  Fronts are in post-order, so the
    // subtree of front j is the index range [first[j], j].  Subtrees whose work
    // is at most 1/(8 * threads) of the total (and whose parent's is not) run
    // in parallel, each in post-order on one thread; the remaining top fronts
    // (the large separators near the root) then run in post-order with the
    // trailing updates of big fronts split over the threads.
    std::vector<double> work(ns, 0.0);
    std::vector<int> first(ns);
    for (int j = 0; j < ns; ++j) first[j] = j;
    double total = 0;
    for (int j = 0; j < ns; ++j) {
        const double f = (double)ncol[j] + (double)rows[j].size();
        work[j] += (double)ncol[j] * f * f + f;
        total += (double)ncol[j] * f * f + f;
        if (parent[j] >= 0) {
            work[parent[j]] += work[j];
            first[parent[j]] = std::min(first[parent[j]], first[j]);
        }
    }
    const int threads = std::max(1, omp_get_max_threads());
    const double cut = total / (8.0 * threads);
    std::vector<int> roots;
    std::vector<char> in_subtree(ns, 0);
    for (int j = 0; j < ns; ++j)
        if (work[j] <= cut && (parent[j] < 0 || work[parent[j]] > cut)) roots.push_back(j);
    for (int r : roots)
        for (int j = first[r]; j <= r; ++j) in_subtree[j] = 1;
    std::sort(roots.begin(), roots.end(), [&](int a, int b) { return work[a] > work[b]; });
    std::string err;
#pragma omp parallel if (roots.size() > 1 && !omp_in_parallel())
    {
        FrontScratch sc;
        sc.pos.assign(n, -1);
#pragma omp for schedule(dynamic, 1)
        for (long t = 0; t < (long)roots.size(); ++t) {
            try {
                for (int j = first[roots[t]]; j <= roots[t]; ++j) factor_front(j, sc, false);
            } catch (const std::exception& e) {
#pragma omp critical(hdd_factor_err)
                err = e.what();
            }
        }
    }
    if (!err.empty()) throw Error(HDD_ERR_INTERNAL, err);
    FrontScratch sc;
    sc.pos.assign(n, -1);
    for (int j = 0; j < ns; ++j)
        if (!in_subtree[j]) factor_front(j, sc, true);
}

void SnFactor::build_solve_blocks() {
    // Per front: Fw = [Linv; -W] ((nj+nr) x nj, col-major) with Linv = L_JJ^{-1}
    // (lower triangular) and W = L_RJ Linv, so that the forward substitution of a
    // front is one product [y_J; v_J] = Fw f_J (+ f_R on the update rows) and the
    // backward substitution is x_J = Fw^T [y_J; x_R].  Column c of Fw needs only
    // column c of L^{-1}, so columns are computed independently.
    const int ns = (int)col0.size();
    Fw.assign(ns, {});
    auto work = [&](int j, bool inner_par) {
        const int nj = ncol[j], nr = (int)rows[j].size(), m = nj + nr;
        BlockVec& F = Fw[j];
        F.resize((size_t)m * nj);  // every column is cleared and written by solve_block_columns
        const BlockVec& L = Ljj[j];
        const BlockVec& R = Lrj[j];
        const int ngroups = (nj + kSolveGroup - 1) / kSolveGroup;
#pragma omp parallel for schedule(dynamic, 1) if (inner_par)
        for (int gi = 0; gi < ngroups; ++gi) {
            const int c0 = gi * kSolveGroup;
            solve_block_columns(L.data(), R.data(), nj, nr, c0, std::min(kSolveGroup, nj - c0), F.data(), m);
        }
    };
    std::vector<int> small;
    for (int j = 0; j < ns; ++j)
        if (ncol[j] >= 128) work(j, true);
        else small.push_back(j);
#pragma omp parallel for schedule(dynamic)
    for (long t = 0; t < (long)small.size(); ++t) work(small[t], false);
}

void SnFactor::solve(double* x) const {
    const int ns = (int)col0.size();
    std::vector<double> y(n);
    for (int i = 0; i < n; ++i) y[i] = x[perm[i]];
    for (int j = 0; j < ns; ++j) {
        const int nj = ncol[j], nr = (int)rows[j].size();
        double* yj = &y[col0[j]];
        for (int a = 0; a < nj; ++a) {
            yj[a] /= Ljj[j][(size_t)a * nj + a];
            for (int i = a + 1; i < nj; ++i) yj[i] -= Ljj[j][(size_t)a * nj + i] * yj[a];
            for (int k = 0; k < nr; ++k) y[rows[j][k]] -= Lrj[j][(size_t)a * nr + k] * yj[a];
        }
    }
    for (int j = ns - 1; j >= 0; --j) {
        const int nj = ncol[j], nr = (int)rows[j].size();
        double* yj = &y[col0[j]];
        for (int a = nj - 1; a >= 0; --a) {
            double acc = yj[a];
            for (int k = 0; k < nr; ++k) acc -= Lrj[j][(size_t)a * nr + k] * y[rows[j][k]];
            for (int i = a + 1; i < nj; ++i) acc -= Ljj[j][(size_t)a * nj + i] * yj[i];
            yj[a] = acc / Ljj[j][(size_t)a * nj + a];
        }
    }
    for (int i = 0; i < n; ++i) x[perm[i]] = y[i];
}

}  // namespace hdd
