// spaqr: the command-line driver with the reference's flags and flow
// (spaQR.cpp:26-323), on the B200 library through its C ABI.
//
//   spaqr -m A.mtx [-l L] [-n N -d D | --coordinates X.mtx] [-t tol] [--skip s]
//         [--scale 1] [--order 1|1.5] [--hsl 0] [-i iters] [--res r] [--rhs b.mtx]
//         [--precision fp64|fp32] [--target r] [--device k]
//
// Flow as in the reference: read the MatrixMarket matrix (transposed when it
// has fewer rows than columns), scale its columns to norm 10, build the tree
// (geometric partition from a tensor grid or a coordinate file; without
// coordinates, the library's recursive bisection of the A^T A graph in the
// place of the reference's METIS / PaToH partition), partition,
// assemble, factorize (per-level lines), one solve with the seeded random
// right-hand side (mt19937 seed 2021, uniform on [-1, 1], src/util.cpp:943-952)
// and its residual, then GMRES (square) or CGLS (more rows than columns) with
// b = that random vector or --rhs.
//
// Flags the reference has and this build does not run: --hsl != 0 (the library
// returns SPQ_ERR_UNSUPPORTED) and the Eigen comparison solvers --useEigenLSCG /
// --useEigenQR / --useCholesky. --scale 0 runs on square systems; on least
// squares the driver switches it to 1, as the reference's does.
// Added: --precision fp32 (FP32 factorization, FP64 Krylov), --target r (the
// time-to-residual driver: refinement with GMRES corrections until the true
// ||Ax - b|| / ||b|| <= r; square systems), --device k.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <map>
#include <random>
#include <string>
#include <vector>

#include "mm_io.hpp"
#include "spaqr_b200.h"

namespace {

using Clock = std::chrono::steady_clock;
double since(Clock::time_point a) { return std::chrono::duration<double>(Clock::now() - a).count(); }

struct Opt {
    const char* longname;
    const char* shortname;
    bool takes_value;
    const char* help;
};

const Opt kOpts[] = {
    {"help", nullptr, false, "Print help"},
    {"matrix", "m", true, "Matrix file in MatrixMarket format"},
    {"lvl", "l", true, "Number of levels (default ceil(log2(ncols/64)))"},
    {"coordinates", nullptr, true, "Coordinates MatrixMarket array file (d x N): geometric partitioning"},
    {"coordinates_n", "n", true, "Tensor grid n^d coordinates (with -d); overrides --coordinates"},
    {"coordinates_d", "d", true, "Tensor grid dimension (with -n)"},
    {"hsl", nullptr, true, "HSL bipartite row matching (0 only in this build)"},
    {"tol", "t", true, "Sparsification tolerance (default 1e-1)"},
    {"skip", nullptr, true, "Levels without sparsification (default 0)"},
    {"order", nullptr, true, "Scheme order: 1 (default) or 1.5 (keeps the E2 term: more accurate, more memory)"},
    {"scale", nullptr, true, "Block scaling (default 1)"},
    {"iterations", "i", true, "Iterative solver iterations (default 300)"},
    {"rhs", nullptr, true, "Right-hand side in MatrixMarket array format"},
    {"res", nullptr, true, "Relative residual of the iterative solver (default 1e-12)"},
    {"useEigenLSCG", nullptr, true, "Eigen comparison solver (not built)"},
    {"useEigenQR", nullptr, true, "Eigen comparison solver (not built)"},
    {"useCholesky", nullptr, true, "Eigen comparison solver (not built)"},
    {"precision", nullptr, true, "fp64 (default) or fp32: FP32 factorization with FP64 Krylov"},
    {"target", nullptr, true, "Time-to-residual driver: refine until ||Ax-b||/||b|| <= target (square)"},
    {"device", nullptr, true, "CUDA device (default 0)"},
};

void usage() {
    std::cout << "spaQR-B200: sparsified QR for general sparse matrices\nUsage:\n  spaqr [OPTION...]\n\n";
    for (const Opt& o : kOpts) {
        std::string s = "  ";
        s += o.shortname ? std::string("-") + o.shortname + ", " : std::string("    ");
        s += std::string("--") + o.longname + (o.takes_value ? " arg" : "");
        if (s.size() < 32) s.resize(32, ' ');
        std::cout << s << " " << o.help << "\n";
    }
}

// --name value, --name=value, -x value. Returns false (with a message) on an
// unknown option or a missing value.
bool parse(int argc, char** argv, std::map<std::string, std::string>& out) {
    for (int a = 1; a < argc; ++a) {
        std::string arg = argv[a];
        const Opt* hit = nullptr;
        std::string val;
        bool has_val = false;
        if (arg.rfind("--", 0) == 0) {
            std::string name = arg.substr(2);
            const size_t eq = name.find('=');
            if (eq != std::string::npos) {
                val = name.substr(eq + 1);
                name = name.substr(0, eq);
                has_val = true;
            }
            for (const Opt& o : kOpts)
                if (name == o.longname) hit = &o;
        } else if (arg.size() >= 2 && arg[0] == '-') {
            const std::string name = arg.substr(1);
            for (const Opt& o : kOpts)
                if (o.shortname && name == o.shortname) hit = &o;
        }
        if (!hit) {
            std::cerr << "unknown option " << arg << "\n";
            return false;
        }
        if (hit->takes_value && !has_val) {
            if (a + 1 >= argc) {
                std::cerr << "option " << arg << " needs a value\n";
                return false;
            }
            val = argv[++a];
        }
        out[hit->longname] = hit->takes_value ? val : "1";
    }
    return true;
}

int check(int rc, const char* what) {
    if (rc != SPQ_OK) std::cerr << what << " failed (" << rc << "): " << spq_last_error() << "\n";
    return rc;
}

// Seeded right-hand side of the reference: mt19937(seed), uniform on [-1, 1].
std::vector<double> random_vector(int size, int seed) {
    std::mt19937 rng;
    rng.seed(seed);
    std::uniform_real_distribution<double> dist(-1.0, 1.0);
    std::vector<double> x(size);
    for (int i = 0; i < size; ++i) x[i] = dist(rng);
    return x;
}

double norm(const std::vector<double>& v) {
    double s = 0;
    for (double x : v) s += x * x;
    return std::sqrt(s);
}

}  // namespace

int main(int argc, char** argv) {
    std::map<std::string, std::string> o;
    if (!parse(argc, argv, o)) return 1;
    auto has = [&](const char* k) { return o.count(k) > 0; };
    auto geti = [&](const char* k, int d) { return has(k) ? std::atoi(o[k].c_str()) : d; };
    auto getd = [&](const char* k, double d) { return has(k) ? std::atof(o[k].c_str()) : d; };
    if (has("help")) {
        usage();
        return 0;
    }
    if (!has("matrix")) {
        std::cout << "--matrix is mandatory" << std::endl;
        return 0;
    }
    for (const char* k : {"useEigenLSCG", "useEigenQR", "useCholesky"})
        if (geti(k, 0)) {
            std::cerr << "--" << k << ": the Eigen comparison solvers are not part of this build\n";
            return 1;
        }
    const std::string matrix = o["matrix"];
    const int cn = geti("coordinates_n", -1), cd = geti("coordinates_d", -1);
    const bool geo_file = has("coordinates");
    if ((cn == -1 && cd >= 0) || (cd == -1 && cn >= 0)) {
        std::cout << "cn and cd should be both provided, or none should be provided" << std::endl;
        return 1;
    }
    const bool geo_tensor = cn >= 0 && cd >= 0;
    const bool geo = geo_file || geo_tensor;

    spq::mm::Csc A;
    try {
        A = spq::mm::read_sparse(matrix);
    } catch (const std::exception& e) {
        std::cerr << "cannot read " << matrix << ": " << e.what() << "\n";
        return 1;
    }
    if (A.m < A.n) {
        std::cout << " <<< Warning!!! nrows < ncols. Finding QR on A.transpose() instead. " << std::endl;
        A = spq::mm::transpose(A);
    }
    const int nrows = A.m, ncols = A.n;
    std::cout << "Matrix " << matrix << " with " << nrows << " rows,  " << ncols << " columns loaded" << std::endl;
    const bool useGMRES = nrows == ncols, useCGLS = nrows > ncols;
    const int iterations = geti("iterations", 300);
    const double residual = getd("res", 1e-12);
    int nlevels;
    if (!has("lvl")) {
        std::cout << "--Levels not provided" << std::endl;
        nlevels = (int)std::ceil(std::log2((double)(ncols / 64)));
        std::cout << " Levels set to ceil(log2(ncols/64)) =  " << nlevels << std::endl;
    } else {
        nlevels = geti("lvl", 1);
    }
    const int hsl = geti("hsl", 0);
    int scale = geti("scale", 1);
    if (nrows != ncols && scale == 0) {
        std::cout << "Scaling necessary for rectangular matrices" << std::endl;
        std::cout << "Setting scale to 1" << std::endl;
        scale = 1;
    }
    const double tol = getd("tol", 1e-1);
    const float order = (float)getd("order", 1.0);

    auto p0 = Clock::now();
    if (check(spq_column_normalize(A.m, A.n, A.colptr.data(), A.rowind.data(), A.val.data()), "normalization"))
        return 1;
    std::cout << "Pre-process time: " << since(p0) << std::endl;

    const int skip = tol == 0 ? nlevels - 1 : geti("skip", 0);
    std::vector<double> X;
    int xd = 0;
    if (geo_tensor) {
        if (std::pow((double)cn, (double)cd) != (double)ncols) {
            std::cout << "Error: cn and cd where both provided, but cn^cd != N where A is NxN" << std::endl;
            return 1;
        }
        std::cout << "Tensor coordinate matrix of size " << cn << "^" << cd << " built" << std::endl;
    } else if (geo_file) {
        int xr = 0, xc = 0;
        try {
            X = spq::mm::read_dense(o["coordinates"], xr, xc);
        } catch (const std::exception& e) {
            std::cerr << "cannot read " << o["coordinates"] << ": " << e.what() << "\n";
            return 1;
        }
        std::cout << "Coordinate file " << xr << "x" << xc << " loaded from " << o["coordinates"] << std::endl;
        if (xc != ncols) {
            std::cout << "Error: coordinate file should hold a matrix of size d x N" << std::endl;
            return 1;
        }
        xd = xr;
    }

    spq_tree* t = nullptr;
    if (check(spq_create(&t, nlevels, skip), "create")) return 1;
    const std::string prec = has("precision") ? o["precision"] : "fp64";
    if (prec != "fp64" && prec != "fp32") {
        std::cerr << "--precision must be fp64 or fp32\n";
        return 1;
    }
    int rc = 0;
    rc = rc ? rc : check(spq_set_device(t, geti("device", 0)), "device");
    rc = rc ? rc : check(spq_set_precision(t, prec == "fp32" ? SPQ_FP32 : SPQ_FP64), "precision");
    rc = rc ? rc : check(spq_set_scale(t, scale), "scale");
    rc = rc ? rc : check(spq_set_tol(t, tol), "tol");
    rc = rc ? rc : check(spq_set_order(t, order), "order");
    rc = rc ? rc : check(spq_set_hsl(t, hsl), "hsl");
    if (!rc && nrows == ncols) rc = check(spq_set_square(t, 1), "square");
    if (!rc && geo_tensor) rc = check(spq_set_coords_grid(t, cn, cd), "coordinates");
    if (!rc && geo_file) rc = check(spq_set_coords(t, xd, ncols, X.data()), "coordinates");
    if (!rc) {  // Tree::partition's banner (src/tree.cpp:605-616)
        if (geo) std::cout << "Using GeometricPartition... " << std::endl;
        else std::cout << "Using graph bisection partition (A^T A)... " << std::endl;
    }
    rc = rc ? rc : check(spq_set_verbose(t, 1), "verbose");
    const int* cp = A.colptr.data();
    const int* ri = A.rowind.data();
    const double* va = A.val.data();
    rc = rc ? rc : check(spq_partition(t, A.m, A.n, cp, ri, va), "partition");
    rc = rc ? rc : check(spq_assemble(t, A.m, A.n, cp, ri, va), "assemble");
    rc = rc ? rc : check(spq_factorize(t), "factorize");
    if (rc) {
        spq_destroy(t);
        return 1;
    }

    auto spmv = [&](const std::vector<double>& x) {  // A x
        std::vector<double> y(nrows, 0.0);
        for (int j = 0; j < ncols; ++j)
            for (int q = cp[j]; q < cp[j + 1]; ++q) y[ri[q]] += va[q] * x[j];
        return y;
    };
    auto spmv_t = [&](const std::vector<double>& y) {  // A^T y
        std::vector<double> x(ncols, 0.0);
        for (int j = 0; j < ncols; ++j) {
            double s = 0;
            for (int q = cp[j]; q < cp[j + 1]; ++q) s += va[q] * y[ri[q]];
            x[j] = s;
        }
        return x;
    };
    auto minus = [](std::vector<double> a, const std::vector<double>& b) {
        for (size_t i = 0; i < a.size(); ++i) a[i] -= b[i];
        return a;
    };

    {  // one solve with the seeded random right-hand side
        const std::vector<double> b = random_vector(nrows, 2021);
        std::vector<double> x(ncols, 0.0);
        auto s0 = Clock::now();
        if (nrows == ncols) {
            rc = check(spq_solve(t, b.data(), x.data()), "solve");
            std::cout << "<<<<tsolv=" << since(s0) << std::endl;
            std::cout << "One-time solve (Random b):" << std::endl;
            std::cout << "<<<<|(Ax-b)|/|b| : " << std::scientific << norm(minus(spmv(x), b)) / norm(b) << std::endl;
        } else {
            const std::vector<double> atb = spmv_t(b);
            rc = check(spq_solve_nrml(t, atb.data(), x.data()), "solve_nrml");
            std::cout << "<<<<tsolv=" << since(s0) << std::endl;
            std::cout << "One-time solve (Random b):" << std::endl;
            std::cout << "<<<<|A'(Ax-b)|/|A'b| : " << std::scientific
                      << norm(spmv_t(minus(spmv(x), b))) / norm(atb) << std::endl;
        }
    }
    if (rc) {
        spq_destroy(t);
        return 1;
    }

    std::vector<double> b;
    if (!has("rhs")) {
        b = random_vector(nrows, 2021);
    } else {
        int br = 0, bc = 0;
        try {
            b = spq::mm::read_dense(o["rhs"], br, bc);
        } catch (const std::exception& e) {
            std::cerr << "cannot read " << o["rhs"] << ": " << e.what() << "\n";
            spq_destroy(t);
            return 1;
        }
        if (bc != 1 || br != nrows) {
            std::cerr << "--rhs must be a " << nrows << " x 1 array\n";
            spq_destroy(t);
            return 1;
        }
    }
    std::vector<double> x(ncols, 0.0);
    int its = 0;
    double res = 0;
    if (useGMRES && has("target")) {
        auto g0 = Clock::now();
        const double target = getd("target", 1e-10);
        const double inner = prec == "fp32" ? 1e-5 : target;  // FP32 factor: loose corrections, refined
        rc = spq_solve_to_residual(t, A.m, A.n, cp, ri, va, b.data(), x.data(), target, inner, 20, iterations, &its,
                                   &res);
        const double tt = since(g0);
        if (rc != SPQ_OK && rc != SPQ_ERR_NOCONV) {
            check(rc, "solve_to_residual");
        } else {
            std::cout << "Refined GMRES: #iterations: " << its << ", residual |Ax-b|/|b|: "
                      << norm(minus(spmv(x), b)) / norm(b) << (rc == SPQ_ERR_NOCONV ? " (target not reached)" : "")
                      << std::endl;
            std::cout << "  Time to residual (GMRES): " << tt << " s." << std::endl;
            std::cout << "<<<<GMRES=" << its << std::endl;
            rc = 0;
        }
    } else if (useGMRES) {
        auto g0 = Clock::now();
        rc = spq_gmres(t, A.m, A.n, cp, ri, va, b.data(), x.data(), iterations, iterations, residual, &its, &res);
        const double tt = since(g0);
        if (rc != SPQ_OK && rc != SPQ_ERR_NOCONV) {
            check(rc, "gmres");
        } else {
            std::cout << "GMRES: #iterations: " << its << ", residual |Ax-b|/|b|: " << norm(minus(spmv(x), b)) / norm(b)
                      << std::endl;
            std::cout << "  GMRES: " << tt << " s." << std::endl;
            std::cout << "<<<<GMRES=" << its << std::endl;
            rc = 0;
        }
    } else if (useCGLS) {
        auto c0 = Clock::now();
        rc = spq_cgls(t, A.m, A.n, cp, ri, va, b.data(), x.data(), iterations, residual, &its, &res);
        if (rc != SPQ_OK && rc != SPQ_ERR_NOCONV) {
            check(rc, "cgls");
        } else {
            std::cout << "CGLS: #iterations: " << its << ", residual |A'(Ax-b)|/|A'(b)|: "
                      << norm(spmv_t(minus(spmv(x), b))) / norm(spmv_t(b)) << std::endl;
            std::cout << "  CGLS: " << since(c0) << " s." << std::endl;
            std::cout << "<<<<CGLS=" << its << std::endl;
            rc = 0;
        }
    }
    spq_destroy(t);
    return rc ? 1 : 0;
}
