// Host reference of the supernodal solve plans (sn_solve.cu): the fronts of a
// batch of factorisations with concatenated unknowns, the FP32 blocks
// Fw = [L_JJ^{-1}; -L_RJ L_JJ^{-1}] exactly as the device plan stores them,
// and a front-by-front solve with the device kernels' arithmetic (FP64
// accumulation of the FP32 x FP32 products, FP64 vectors between fronts, one
// rounding to FP32 at the output).  It lets the CPU tests check a plan
// against the factorisation's own FP64 solve without a GPU, and the GPU tests
// check the device solve against it.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "sigma.h"

namespace hdd {

void PlanHost::build(const std::vector<const SnFactor*>& factors, const std::vector<int>& offsets) {
    *this = PlanHost();
    for (size_t f = 0; f < factors.size(); ++f) n = std::max(n, offsets[f] + factors[f]->n);
    perm.assign(n, 0);
    long long fw_total = 0;
    for (size_t f = 0; f < factors.size(); ++f) {
        const SnFactor& F = *factors[f];
        if (F.Fw.size() != F.col0.size()) throw Error(HDD_ERR_INTERNAL, "solve blocks not built");
        const int off = offsets[f], base = nsn;
        for (int i = 0; i < F.n; ++i) perm[off + i] = off + F.perm[i];
        for (size_t j = 0; j < F.col0.size(); ++j) {
            const int nj = F.ncol[j], nr = (int)F.rows[j].size(), m = nj + nr;
            col0.push_back(off + F.col0[j]);
            ncol.push_back(nj);
            nrow.push_back(nr);
            parent.push_back(F.parent[j] >= 0 ? base + F.parent[j] : -1);
            rows_off.push_back((long long)rows.size());
            for (int r : F.rows[j]) rows.push_back(off + r);
            fw_off.push_back(fw_total);
            fw_total += (long long)((m + 3) & ~3) * nj;
            ++nsn;
        }
    }
    fw.assign((size_t)std::max<long long>(fw_total, 4), 0.0f);
    int g = 0;
    for (size_t f = 0; f < factors.size(); ++f) {
        const SnFactor& F = *factors[f];
        for (size_t j = 0; j < F.col0.size(); ++j, ++g) {
            const BlockVec& W = F.Fw[j];
            const int nj = ncol[g], m = nj + nrow[g], ld = (m + 3) & ~3;
            float* dst = &fw[(size_t)fw_off[g]];
            for (int c = 0; c < nj; ++c)
                for (int r = 0; r < m; ++r) dst[(size_t)c * ld + r] = (float)W[(size_t)c * m + r];
        }
    }
}

void PlanHost::emulate(const float* b_old, float* x_old) const {
    // Fronts are stored in post-order (children before parents), so a forward
    // sweep in index order and a backward sweep in reverse order respect the
    // elimination tree; a front's update lands on its rows, which belong to
    // its ancestors.
    std::vector<double> y(n, 0.0), x(n, 0.0), f;
    for (int i = 0; i < n; ++i) y[i] = (double)b_old[perm[i]];
    for (int J = 0; J < nsn; ++J) {
        const int nj = ncol[J], m = nj + nrow[J], c0 = col0[J];
        const size_t ld = (size_t)((m + 3) & ~3);
        const float* A = &fw[(size_t)fw_off[J]];
        f.assign(y.begin() + c0, y.begin() + c0 + nj);
        for (int r = 0; r < m; ++r) {
            double acc = 0.0;
            for (int c = 0; c < std::min(nj, r + 1); ++c) acc = std::fma((double)A[(size_t)c * ld + r], f[c], acc);
            if (r < nj) y[c0 + r] = acc;
            else y[rows[rows_off[J] + (r - nj)]] += acc;
        }
    }
    for (int J = nsn - 1; J >= 0; --J) {
        const int nj = ncol[J], m = nj + nrow[J], c0 = col0[J];
        const size_t ld = (size_t)((m + 3) & ~3);
        const float* A = &fw[(size_t)fw_off[J]];
        for (int a = 0; a < nj; ++a) {
            double acc = 0.0;
            for (int r = a; r < m; ++r) {
                const double g = r < nj ? y[c0 + r] : x[rows[rows_off[J] + (r - nj)]];
                acc = std::fma((double)A[(size_t)a * ld + r], g, acc);
            }
            x[c0 + a] = acc;
        }
    }
    for (int i = 0; i < n; ++i) x_old[perm[i]] = (float)x[i];
}

const std::vector<std::array<int, 3>>* interface_positions(const InterfaceHost& ih, int l) {
    if (l < (int)ih.iface_xyz.size() && (int)ih.iface_xyz[l].size() == ih.Arr[l].rows) return &ih.iface_xyz[l];
    return nullptr;
}

const std::vector<std::array<int, 3>>* interior_positions(const InterfaceHost& ih, int l, int sd) {
    if (l >= (int)ih.aii_xyz.size() || sd >= (int)ih.aii_xyz[l].size()) return nullptr;
    if ((int)ih.aii_xyz[l][sd].size() != ih.Aii[l][sd].rows) return nullptr;
    return &ih.aii_xyz[l][sd];
}

void interface_solve_plan(const InterfaceHost& ih, int kind, int l, std::vector<SnFactor>& factors, PlanHost& plan) {
    const double eps = 1e-5;
    std::vector<const SnFactor*> fs;
    std::vector<int> offs;
    if (kind == 0) {
        factors.assign(1, SnFactor());
        factors[0].analyze(ih.Arr[l], interface_positions(ih, l));
        factors[0].factor(ih.Arr[l], eps);
        factors[0].build_solve_blocks();
        fs.push_back(&factors[0]);
        offs.push_back(0);
    } else {
        factors.assign(ih.n_sub, SnFactor());
        int off = 0;
        for (int sd = 0; sd < ih.n_sub; ++sd) {
            const CsrF& A = ih.Aii[l][sd];
            if (A.rows > 0) {
                factors[sd].analyze(A, interior_positions(ih, l, sd));
                factors[sd].factor(A, eps);
                factors[sd].build_solve_blocks();
                fs.push_back(&factors[sd]);
                offs.push_back(off);
            }
            off += A.rows;
        }
    }
    plan.build(fs, offs);
}

}  // namespace hdd
