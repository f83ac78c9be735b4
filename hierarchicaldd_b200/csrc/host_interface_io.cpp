// Interface-system dump and reload: the reference's -iomode output / input.
//
// The reference's CPU solver writes its assembled interface matrices after the
// split and reads them back instead of assembling
// (CPU/SPGrid_Domain_Decomposition_Solver/SPGrid_Domain_Decomposition_Solver.h:121-161,
// CPU/Interface_Solver/INTERFACE_SOLVER_DATA.h:177-212 and
// INTERFACE_MATRIX_GENERATOR.h:66-80).  The directory layout is the same:
//   levels, number_of_subdomains      one int32 each
//   Aii_<l>_<s>, Arr_<l>              Matrix Market, column-major entry order
//   Air_<l>_<s>, Prr_<l>              Matrix Market, row-major entry order
//   interface_map                     uint64 n, then n x 3 int32 cell indices
// Matrix Market files are "%%MatrixMarket matrix coordinate real general",
// a "rows cols nnz" line and 1-based "row col value" lines, the values with
// nine significant digits so a float reads back unchanged.  This library adds
// positions_<l> (its own binary: the DOF positions its nested-dissection
// ordering uses); without it a reload orders the factorisations by
// breadth-first level sets instead.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include <omp.h>

#include "host_setup.h"
#include "sigma.h"

namespace hdd {

namespace {

struct FileCloser {
    void operator()(FILE* f) const { if (f) std::fclose(f); }
};
using File = std::unique_ptr<FILE, FileCloser>;

File open_file(const std::string& path, const char* mode) {
    File f(std::fopen(path.c_str(), mode));
    if (!f) throw Error(HDD_ERR_IO, "cannot open " + path + ": " + std::strerror(errno));
    return f;
}

// Entries of a CSR matrix in column-major order (column, then row).
void transpose_order(const CsrF& A, std::vector<int>& ptr, std::vector<int>& idx, std::vector<float>& val) {
    ptr.assign((size_t)A.cols + 1, 0);
    for (int c : A.col) ptr[(size_t)c + 1]++;
    for (int c = 0; c < A.cols; ++c) ptr[(size_t)c + 1] += ptr[c];
    idx.resize(A.col.size());
    val.resize(A.col.size());
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (int r = 0; r < A.rows; ++r)
        for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) {
            const int q = fill[A.col[p]]++;
            idx[q] = r;
            val[q] = A.val[p];
        }
}

void write_market(const std::string& path, const CsrF& A, bool column_major) {
    std::vector<char> buf(1 << 20);  // outlives f, which flushes through it on close
    File f = open_file(path, "w");
    std::setvbuf(f.get(), buf.data(), _IOFBF, buf.size());
    std::fprintf(f.get(), "%%%%MatrixMarket matrix coordinate real general\n%d %d %zu\n", A.rows, A.cols,
                 A.col.size());
    if (column_major) {
        std::vector<int> ptr, idx;
        std::vector<float> val;
        transpose_order(A, ptr, idx, val);
        for (int c = 0; c < A.cols; ++c)
            for (int p = ptr[c]; p < ptr[c + 1]; ++p)
                std::fprintf(f.get(), "%d %d %.8e\n", idx[p] + 1, c + 1, (double)val[p]);
    } else {
        for (int r = 0; r < A.rows; ++r)
            for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p)
                std::fprintf(f.get(), "%d %d %.8e\n", r + 1, A.col[p] + 1, (double)A.val[p]);
    }
    if (std::ferror(f.get())) throw Error(HDD_ERR_IO, "write failed: " + path);
}

// Reads a real coordinate Matrix Market file into CSR (rows sorted by column;
// duplicate entries summed in file order, as Eigen's loadMarket does through
// setFromTriplets).  A "symmetric" header mirrors the stored triangle.
void read_market(const std::string& path, CsrF& A) {
    std::ifstream in(path);
    if (!in) throw Error(HDD_ERR_IO, "cannot open " + path);
    std::string line;
    bool symmetric = false, have_size = false;
    long long rows = 0, cols = 0, nnz = 0;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        if (line[0] == '%') {
            if (line.rfind("%%MatrixMarket", 0) == 0) {
                if (line.find("coordinate") == std::string::npos || line.find("complex") != std::string::npos)
                    throw Error(HDD_ERR_IO, path + ": only real coordinate Matrix Market files are read");
                symmetric = line.find("symmetric") != std::string::npos;
            }
            continue;
        }
        if (std::sscanf(line.c_str(), "%lld %lld %lld", &rows, &cols, &nnz) != 3)
            throw Error(HDD_ERR_IO, path + ": bad size line");
        have_size = true;
        break;
    }
    if (!have_size || rows < 0 || cols < 0 || nnz < 0 || rows > (1ll << 31) - 2 || cols > (1ll << 31) - 2)
        throw Error(HDD_ERR_IO, path + ": bad size line");
    struct T { int r, c; float v; };
    std::vector<T> t;
    // The size line is not trusted for the allocation: a short file fails below.
    t.reserve((size_t)std::min<long long>(nnz, 1ll << 22) * (symmetric ? 2 : 1));
    for (long long k = 0; k < nnz; ++k) {
        if (!std::getline(in, line)) throw Error(HDD_ERR_IO, path + ": fewer entries than its size line says");
        char* p = const_cast<char*>(line.c_str());
        char* e;
        const long long r = std::strtoll(p, &e, 10);
        if (e == p) throw Error(HDD_ERR_IO, path + ": bad entry line");
        p = e;
        const long long c = std::strtoll(p, &e, 10);
        if (e == p) throw Error(HDD_ERR_IO, path + ": bad entry line");
        p = e;
        const float v = std::strtof(p, &e);
        if (e == p) throw Error(HDD_ERR_IO, path + ": bad entry line");
        if (r < 1 || r > rows || c < 1 || c > cols) throw Error(HDD_ERR_IO, path + ": entry outside the matrix");
        t.push_back({(int)r - 1, (int)c - 1, v});
        if (symmetric && r != c) t.push_back({(int)c - 1, (int)r - 1, v});
    }
    A.rows = (int)rows;
    A.cols = (int)cols;
    A.ptr.assign((size_t)rows + 1, 0);
    for (const T& x : t) A.ptr[(size_t)x.r + 1]++;
    for (long long r = 0; r < rows; ++r) A.ptr[(size_t)r + 1] += A.ptr[(size_t)r];
    std::vector<int> col(t.size());
    std::vector<float> val(t.size());
    {
        std::vector<int> fill(A.ptr.begin(), A.ptr.end() - 1);
        for (const T& x : t) {
            const int q = fill[x.r]++;
            col[q] = x.c;
            val[q] = x.v;
        }
    }
    // Per row: stable sort by column, then merge duplicates.
    A.col.clear();
    A.val.clear();
    std::vector<int> np((size_t)rows + 1, 0);
    std::vector<std::pair<int, float>> row;
    for (long long r = 0; r < rows; ++r) {
        row.clear();
        for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) row.push_back({col[p], val[p]});
        std::stable_sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (size_t k = 0; k < row.size();) {
            const int c = row[k].first;
            float s = 0.0f;
            for (; k < row.size() && row[k].first == c; ++k) s += row[k].second;
            A.col.push_back(c);
            A.val.push_back(s);
        }
        np[(size_t)r + 1] = (int)A.col.size();
    }
    A.ptr.swap(np);
}

void write_int(const std::string& path, int v) {
    File f = open_file(path, "wb");
    if (std::fwrite(&v, sizeof(v), 1, f.get()) != 1) throw Error(HDD_ERR_IO, "write failed: " + path);
}

int read_int(const std::string& path) {
    File f = open_file(path, "rb");
    int v = 0;
    if (std::fread(&v, sizeof(v), 1, f.get()) != 1) throw Error(HDD_ERR_IO, "short file: " + path);
    return v;
}

typedef std::vector<std::array<int, 3>> Points;

void write_points(FILE* f, const Points& p) {
    const long long n = (long long)p.size();
    std::fwrite(&n, sizeof(n), 1, f);
    if (n) std::fwrite(p.data(), sizeof(int) * 3, (size_t)n, f);
}

bool read_points(FILE* f, Points& p) {
    long long n = 0;
    if (std::fread(&n, sizeof(n), 1, f) != 1 || n < 0 || n > (1ll << 34)) return false;
    p.resize((size_t)n);
    return n == 0 || std::fread(p.data(), sizeof(int) * 3, (size_t)n, f) == (size_t)n;
}

std::string name(const std::string& dir, const char* stem, int l, int s = -1) {
    std::string n = dir + "/" + stem + "_" + std::to_string(l);
    if (s >= 0) n += "_" + std::to_string(s);
    return n;
}

// Runs fn(k) for k in [0, n) over the host threads; the first exception wins.
template <class Fn>
void parallel_files(int n, Fn fn) {
    std::string err;
    hdd_status st = HDD_OK;
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < n; ++k) {
        try {
            fn(k);
        } catch (const Error& e) {
#pragma omp critical(hdd_io_err)
            if (err.empty()) { err = e.what(); st = e.status; }
        } catch (const std::exception& e) {
#pragma omp critical(hdd_io_err)
            if (err.empty()) { err = e.what(); st = HDD_ERR_IO; }
        }
    }
    if (!err.empty()) throw Error(st, err);
}

}  // namespace

void write_interface_dir(const InterfaceHost& ih, const std::string& dir) {
    write_int(dir + "/levels", ih.M);
    write_int(dir + "/number_of_subdomains", ih.n_sub);
    const int M = ih.M, ns = ih.n_sub;
    parallel_files(M * (2 * ns + 2), [&](int k) {
        const int l = k / (2 * ns + 2), r = k % (2 * ns + 2);
        if (r < ns) write_market(name(dir, "Aii", l, r), ih.Aii[l][r], true);
        else if (r < 2 * ns) write_market(name(dir, "Air", l, r - ns), ih.Air[l][r - ns], false);
        else if (r == 2 * ns) write_market(name(dir, "Arr", l), ih.Arr[l], true);
        else if (l + 1 < M) write_market(name(dir, "Prr", l), ih.Prr[l], false);
    });
    {
        File f = open_file(dir + "/interface_map", "wb");
        const uint64_t n = ih.iface_map.size();
        std::fwrite(&n, sizeof(n), 1, f.get());
        if (n) std::fwrite(ih.iface_map.data(), sizeof(int) * 3, n, f.get());
        if (std::ferror(f.get())) throw Error(HDD_ERR_IO, "write failed: " + dir + "/interface_map");
    }
    parallel_files(M, [&](int l) {
        File f = open_file(name(dir, "positions", l), "wb");
        write_points(f.get(), l < (int)ih.iface_xyz.size() ? ih.iface_xyz[l] : Points());
        const long long n = ns;
        std::fwrite(&n, sizeof(n), 1, f.get());
        for (int s = 0; s < ns; ++s)
            write_points(f.get(), l < (int)ih.aii_xyz.size() ? ih.aii_xyz[l][s] : Points());
        if (std::ferror(f.get())) throw Error(HDD_ERR_IO, "write failed: " + name(dir, "positions", l));
    });
}

void read_interface_dir(const std::string& dir, InterfaceHost& ih) {
    InterfaceHost in;
    in.M = read_int(dir + "/levels");
    in.n_sub = read_int(dir + "/number_of_subdomains");
    const int M = in.M, ns = in.n_sub;
    if (M < 1 || M > 32 || ns < 1) throw Error(HDD_ERR_IO, dir + ": bad levels / number_of_subdomains");
    in.Arr.assign(M, CsrF());
    in.Prr.assign(M - 1, CsrF());
    in.Aii.assign(M, std::vector<CsrF>(ns));
    in.Air.assign(M, std::vector<CsrF>(ns));
    parallel_files(M * (2 * ns + 2), [&](int k) {
        const int l = k / (2 * ns + 2), r = k % (2 * ns + 2);
        if (r < ns) read_market(name(dir, "Aii", l, r), in.Aii[l][r]);
        else if (r < 2 * ns) read_market(name(dir, "Air", l, r - ns), in.Air[l][r - ns]);
        else if (r == 2 * ns) read_market(name(dir, "Arr", l), in.Arr[l]);
        else if (l + 1 < M) read_market(name(dir, "Prr", l), in.Prr[l]);
    });
    {
        File f = open_file(dir + "/interface_map", "rb");
        uint64_t n = 0;
        if (std::fread(&n, sizeof(n), 1, f.get()) != 1 || n > (1ull << 34))
            throw Error(HDD_ERR_IO, dir + "/interface_map: bad header");
        in.iface_map.resize(n);
        if (n && std::fread(in.iface_map.data(), sizeof(int) * 3, n, f.get()) != n)
            throw Error(HDD_ERR_IO, dir + "/interface_map: short file");
    }
    in.n_iface.resize(M);
    for (int l = 0; l < M; ++l) in.n_iface[l] = in.Arr[l].rows;
    // DOF positions: this library's own file when present, else the level-0
    // interface cells (the ordering of the other blocks falls back to level sets).
    in.iface_xyz.assign(M, Points());
    in.aii_xyz.assign(M, std::vector<Points>(ns));
    for (int l = 0; l < M; ++l) {
        FILE* raw = std::fopen(name(dir, "positions", l).c_str(), "rb");
        File f(raw);
        bool ok = raw != nullptr;
        Points ip;
        long long n = 0;
        std::vector<Points> sp;
        if (ok) ok = read_points(raw, ip) && std::fread(&n, sizeof(n), 1, raw) == 1 && n == ns;
        if (ok) {
            sp.resize(ns);
            for (int s = 0; s < ns && ok; ++s) ok = read_points(raw, sp[s]);
        }
        if (ok) {
            in.iface_xyz[l].swap(ip);
            in.aii_xyz[l].swap(sp);
        } else if (l == 0) {
            in.iface_xyz[0] = in.iface_map;
        }
    }
    ih = std::move(in);
}

void check_interface(const DomainLayout& L, int sigma_levels, const InterfaceHost& ih) {
    int ns[3];
    number_of_subdomains(L.opt.size, L.opt.sub, ns);
    const int nsub = ns[0] * ns[1] * ns[2];
    auto bad = [](const std::string& what) { throw Error(HDD_ERR_INVALID_ARGUMENT, "interface dump: " + what); };
    if (ih.M != sigma_levels) bad("it holds " + std::to_string(ih.M) + " levels, sigma_levels is " + std::to_string(sigma_levels));
    if (ih.n_sub != nsub) bad("it holds " + std::to_string(ih.n_sub) + " subdomains, the domain has " + std::to_string(nsub));
    for (int l = 0; l < ih.M; ++l) {
        const CsrF& R = ih.Arr[l];
        if (R.rows != R.cols) bad("Arr is not square");
        for (int s = 0; s < ih.n_sub; ++s) {
            const CsrF& I = ih.Aii[l][s];
            const CsrF& X = ih.Air[l][s];
            if (I.rows != I.cols || X.rows != I.rows || (X.rows > 0 && X.cols != R.rows))
                bad("Aii / Air sizes disagree at level " + std::to_string(l));
        }
        if (l + 1 < ih.M && (ih.Prr[l].rows != R.rows || ih.Prr[l].cols != ih.Arr[l + 1].rows))
            bad("Prr sizes disagree at level " + std::to_string(l));
    }
    if ((int)ih.iface_map.size() != ih.Arr[0].rows) bad("interface_map length differs from Arr");
    for (const auto& c : ih.iface_map) {
        for (int a = 0; a < 3; ++a)
            if (c[a] < 0 || c[a] >= L.opt.size[a]) bad("interface_map cell outside the grid");
        if (!(L.flags0[L.dense_index(c[0], c[1], c[2])] & F_INTERFACE)) bad("interface_map cell is not an Interface cell");
    }
}

}  // namespace hdd
