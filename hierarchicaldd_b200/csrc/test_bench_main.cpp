// hdd_test_bench: the reference's Test_Bench_3D command line over the C ABI.
//
// Same flags, defaults and meaning as
// demos/Domain_Decomposition_CPU_Only/Test_Bench_3D/main.cpp:236-301 (-size,
// -threads, -vlevels, -sigma_levels, -sigma_smoothing, -sigma_mg,
// -interior_smoothing, -boundary_smoothing, -nVcycles, -frame, -origin,
// -sub_size, -d, -o, -mode, -iomode), so a run script of the reference's CPU
// dd_pcg drives this solver unchanged.  "-mode no_convertion" reads the
// Write_SPGrid directory given by -d (main.cpp:307-316); the "velocity" and
// "rhs" modes read the fluids simulation format, which this library does not
// implement, and exit with HDD_ERR_UNSUPPORTED.  -iomode output / input dump
// or reload the interface matrices in the -o directory (main.cpp:315).
// -multilevel yes|no is the two-level demo's flag
// (demos/Domain_Decomposition_CPU_Only_Two_Levels/Test_Bench_3D/main.cpp:251-257):
// "yes" solves every subdomain by a DD at sub_size/2; that demo has no
// -iomode, so with -multilevel yes it defaults to neither.
//
// Flags of this library only: -tol x and -relative_tol 0|1 (the stop test;
// default 1e-6 relative, the reference's is -tol 1e-5 -relative_tol 0),
// -precision reference|mixed, -max_iters n, -device n, and -solution file
// (writes x as raw float32 in the dense layout of hdd.h, z fastest).
//
// Exit status: 0 on a converged solve, 1 when the solve did not converge, 2 on
// a usage error, 3 when a library call fails (its status and message are
// printed).
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "hdd.h"

namespace {

struct Args {
    int size[3] = {257, 257, 257};
    int sub[3] = {64, 64, 64};
    int threads = 0, vlevels = 3, sigma_levels = 3, sigma_smoothing = 3, sigma_mg = 1;
    int interior = 1, boundary = 3, nvcycles = 1, frame = 0;
    int origin[3] = {0, 0, 0};
    std::string dir, out = "output", mode = "velocity", iomode = "output", multilevel = "no";
    bool iomode_given = false;
    double tol = 1e-6;
    int relative_tol = 1, max_iters = 5000, device = 0;
    std::string precision = "reference", solution;
};

void usage(FILE* f) {
    std::fprintf(f,
                 "usage: hdd_test_bench [-size n n n] [-sub_size n n n] [-vlevels n] [-sigma_levels n]\n"
                 "       [-sigma_smoothing n] [-sigma_mg n] [-interior_smoothing n] [-boundary_smoothing n]\n"
                 "       [-nVcycles n] [-threads n] [-frame n] [-origin n n n] -d dir [-o dir]\n"
                 "       [-mode no_convertion|velocity|rhs] [-iomode output|input|neither]\n"
                 "       [-tol x] [-relative_tol 0|1] [-precision reference|mixed] [-max_iters n]\n"
                 "       [-device n] [-solution file] [-multilevel yes|no]\n");
}

bool parse_int(const char* s, int& v) {
    char* e = nullptr;
    const long x = std::strtol(s, &e, 10);
    if (!*s || *e || x < -2147483647L || x > 2147483647L) return false;
    v = (int)x;
    return true;
}

// Vector flags take three values (PARSE_ARGS::Add_Vector_3D_Argument); like
// the reference they are read as numbers and truncated to int.
bool parse_vec(char** argv, int argc, int& i, int v[3]) {
    if (i + 3 >= argc) return false;
    for (int a = 0; a < 3; ++a) {
        char* e = nullptr;
        const double x = std::strtod(argv[i + 1 + a], &e);
        if (*e || x < 0 || x > 1e9) return false;
        v[a] = (int)x;
    }
    i += 3;
    return true;
}

// 0 ok, 1 help printed, 2 usage error.
int parse(int argc, char** argv, Args& a) {
    for (int i = 1; i < argc; ++i) {
        const std::string f = argv[i];
        auto next = [&](std::string& s) {
            if (i + 1 >= argc) return false;
            s = argv[++i];
            return true;
        };
        auto next_int = [&](int& v) { return i + 1 < argc && parse_int(argv[++i], v); };
        bool ok = true;
        if (f == "-help" || f == "--help" || f == "-h") return 1;
        else if (f == "-size") ok = parse_vec(argv, argc, i, a.size);
        else if (f == "-sub_size") ok = parse_vec(argv, argc, i, a.sub);
        else if (f == "-origin") ok = parse_vec(argv, argc, i, a.origin);
        else if (f == "-threads") ok = next_int(a.threads);
        else if (f == "-vlevels") ok = next_int(a.vlevels);
        else if (f == "-sigma_levels") ok = next_int(a.sigma_levels);
        else if (f == "-sigma_smoothing") ok = next_int(a.sigma_smoothing);
        else if (f == "-sigma_mg") ok = next_int(a.sigma_mg);
        else if (f == "-interior_smoothing") ok = next_int(a.interior);
        else if (f == "-boundary_smoothing") ok = next_int(a.boundary);
        else if (f == "-nVcycles") ok = next_int(a.nvcycles);
        else if (f == "-frame") ok = next_int(a.frame);
        else if (f == "-d") ok = next(a.dir);
        else if (f == "-o") ok = next(a.out);
        else if (f == "-mode") ok = next(a.mode);
        else if (f == "-iomode") {
            ok = next(a.iomode);
            a.iomode_given = true;
        }
        else if (f == "-multilevel") ok = next(a.multilevel);
        else if (f == "-relative_tol") ok = next_int(a.relative_tol);
        else if (f == "-max_iters") ok = next_int(a.max_iters);
        else if (f == "-device") ok = next_int(a.device);
        else if (f == "-precision") ok = next(a.precision);
        else if (f == "-solution") ok = next(a.solution);
        else if (f == "-tol") {
            std::string s;
            char* e = nullptr;
            ok = next(s) && (a.tol = std::strtod(s.c_str(), &e), !s.empty() && !*e && a.tol > 0);
        } else {
            std::fprintf(stderr, "unknown flag %s\n", f.c_str());
            return 2;
        }
        if (!ok) {
            std::fprintf(stderr, "bad or missing value for %s\n", f.c_str());
            return 2;
        }
    }
    if (a.multilevel != "yes" && a.multilevel != "no") {
        std::fprintf(stderr, "-multilevel must be yes or no\n");
        return 2;
    }
    if (a.multilevel == "yes" && !a.iomode_given) a.iomode = "neither";
    if (a.iomode != "output" && a.iomode != "input" && a.iomode != "neither") {
        std::fprintf(stderr, "-iomode must be output, input or neither\n");
        return 2;
    }
    if (a.precision != "reference" && a.precision != "mixed") {
        std::fprintf(stderr, "-precision must be reference or mixed\n");
        return 2;
    }
    if (a.relative_tol != 0 && a.relative_tol != 1) {
        std::fprintf(stderr, "-relative_tol must be 0 or 1\n");
        return 2;
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    Args a;
    const int p = parse(argc, argv, a);
    if (p == 1) {
        usage(stdout);
        return 0;
    }
    if (p == 2) {
        usage(stderr);
        return 2;
    }
    std::printf("Size of 3D grid          : %d %d %d\n", a.size[0], a.size[1], a.size[2]);
    std::printf("Size of subdomain        : %d %d %d\n", a.sub[0], a.sub[1], a.sub[2]);
    std::printf("V cycle levels           : %d\n", a.vlevels);
    std::printf("Sigma MG levels          : %d\n", a.sigma_levels);
    std::printf("Sigma smoothing iteration: %d\n", a.sigma_smoothing);
    std::printf("Sigma MG iteration       : %d\n", a.sigma_mg);
    std::printf("Interior smoothing iteration: %d\n", a.interior);
    std::printf("boundary smoothing iteration: %d\n", a.boundary);
    std::printf("V cycle iterations in DD : %d\n", a.nvcycles);
    if (a.mode != "no_convertion") {
        std::fprintf(stderr,
                     "%s: -mode %s reads the fluids simulation format, which this solver does not read; "
                     "write the domain with Write_SPGrid and use -mode no_convertion\n",
                     hdd_status_string(HDD_ERR_UNSUPPORTED), a.mode.c_str());
        return 3;
    }
    if (a.dir.empty()) {
        std::fprintf(stderr, "-mode no_convertion needs -d <SPGrid directory>\n");
        usage(stderr);
        return 2;
    }
    if (a.threads > 0) omp_set_num_threads(a.threads);

    hdd_options o;
    hdd_options_default(&o);
    for (int k = 0; k < 3; ++k) { o.size[k] = a.size[k]; o.sub_size[k] = a.sub[k]; }
    o.vlevels = a.vlevels;
    o.nVcycles = a.nvcycles;
    o.interior_smoothing = a.interior;
    o.boundary_smoothing = a.boundary;
    o.sigma_levels = a.sigma_levels;
    o.sigma_smoothing = a.sigma_smoothing;
    o.sigma_mg = a.sigma_mg;
    o.tol = a.tol;
    o.relative_tol = a.relative_tol;
    o.max_iters = a.max_iters;
    o.precision_mode = a.precision == "mixed" ? HDD_PRECISION_MIXED : HDD_PRECISION_REFERENCE;
    o.device = a.device;
    o.multilevel = a.multilevel == "yes" ? 1 : 0;

    hdd_solver* h = nullptr;
    auto fail = [&](const char* what, hdd_status st) {
        std::fprintf(stderr, "%s failed: %s: %s\n", what, hdd_status_string(st), h ? hdd_last_error(h) : "");
        hdd_destroy(h);
        return 3;
    };
    hdd_status st = hdd_create(&o, &h);
    if (st != HDD_OK) return fail("hdd_create", st);
    if ((st = hdd_load_spgrid_dir(h, a.dir.c_str())) != HDD_OK) return fail("Read_SPGrid", st);
    std::printf("Finished Reading SPGrid\n");
    const int io = a.iomode == "output" ? HDD_IOMODE_OUTPUT : a.iomode == "input" ? HDD_IOMODE_INPUT
                                                                                    : HDD_IOMODE_NEITHER;
    if ((st = hdd_set_iomode(h, io, a.out.c_str())) != HDD_OK) return fail("iomode", st);
    if ((st = hdd_initialize_preconditioner(h)) != HDD_OK) return fail("Initialize_Preconditioner", st);
    double phase_ms[4];
    if (hdd_get_setup_timing(h, phase_ms) == HDD_OK)
        std::printf("setup ms: layout %.1f, interface system %.1f, interface solver %.1f, total %.1f\n",
                    phase_ms[0], phase_ms[1], phase_ms[2], phase_ms[3]);
    hdd_result r;
    st = hdd_solve(h, &r);
    if (st != HDD_OK && st != HDD_ERR_NOT_CONVERGED) return fail("Solve", st);
    std::printf("cg iterations            : %d\n", r.iterations);
    std::printf("converged                : %d\n", r.converged);
    std::printf("residual max|r|          : %.9e\n", r.final_norm);
    std::printf("true residual inf / l2   : %.9e %.9e\n", r.true_residual_inf, r.true_residual_l2);
    std::printf("setup ms / solve ms      : %.3f %.3f\n", r.setup_ms, r.solve_ms);
    if (!a.solution.empty()) {
        const size_t n = (size_t)a.size[0] * a.size[1] * a.size[2];
        std::vector<float> x(n);
        const hdd_status sx = hdd_get_solution_dense(h, x.data());
        if (sx != HDD_OK) return fail("solution", sx);
        FILE* f = std::fopen(a.solution.c_str(), "wb");
        if (!f || std::fwrite(x.data(), sizeof(float), n, f) != n) {
            if (f) std::fclose(f);
            std::fprintf(stderr, "cannot write %s\n", a.solution.c_str());
            hdd_destroy(h);
            return 3;
        }
        std::fclose(f);
    }
    hdd_destroy(h);
    return r.converged ? 0 : 1;
}
